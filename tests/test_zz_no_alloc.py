"""The IMat builder that allocates no device memory, against the ordinary one.

pbsam_imat_build_static exists for callers that cannot call cudaMalloc (their own
pool allocator owns the device memory, or their device footprint must stay fixed
after the library loads).  It keeps its work buffers in one fixed device array
shared by every call, so it is checked here on two calls in a row: the second
call must not see anything the first one left in the array.  The file sorts last
so that a run stopping at the first failure has run every other test before it.
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import golden_dir

pytestmark = pytest.mark.gpu
TOL = 1e-8   # relative, as the other GPU parity tests


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _call_static(ctx, cen, rad, n_points, out):
    import pbsam_b200 as pb
    dp = ctypes.POINTER(ctypes.c_double)
    return pb.lib().pbsam_imat_build_static(ctx.handle, len(rad), cen.ctypes.data_as(dp), rad.ctypes.data_as(dp),
                                            n_points, out.ctypes.data_as(dp))


def test_static_imat_matches_allocating_builder_twice():
    import pbsam_b200 as pb
    from pbsam_b200 import synth
    cen, rad, _, _ = synth.read_pqr(os.path.join(golden_dir("cfg0"), "molA.pqr"))
    cen = np.ascontiguousarray(cen, dtype=np.float64)
    rad = np.ascontiguousarray(rad, dtype=np.float64)
    ctx = pb.CSystem(poles=10, salt=0.05)
    try:
        n_points = 250000
        ref = ctx.build_imats(cen, rad, n_points=n_points)
        for call in range(2):
            out = np.full(ref.shape, np.nan)
            assert _call_static(ctx, cen, rad, n_points, out) == 0, pb.lib().pbsam_last_error()
            assert np.all(np.isfinite(out)), "call %d" % call
            assert rel(out, ref) < TOL, "call %d: %.3e" % (call, rel(out, ref))
        # a different molecule through the same array, then the first one again
        cen_b, rad_b, _, _ = synth.read_pqr(os.path.join(golden_dir("cfg0"), "molB.pqr"))
        cen_b = np.ascontiguousarray(cen_b, dtype=np.float64)
        rad_b = np.ascontiguousarray(rad_b, dtype=np.float64)
        ref_b = ctx.build_imats(cen_b, rad_b, n_points=n_points)
        out_b = np.zeros_like(ref_b)
        assert _call_static(ctx, cen_b, rad_b, n_points, out_b) == 0
        assert rel(out_b, ref_b) < TOL
        out = np.zeros_like(ref)
        assert _call_static(ctx, cen, rad, n_points, out) == 0
        assert rel(out, ref) < TOL
    finally:
        ctx.close()


def test_static_imat_at_its_maximum_order():
    """p = 16 fills the fixed array's Gram and IMat buffers exactly; two calls in a
    row still agree with the allocating builder."""
    import pbsam_b200 as pb
    from pbsam_b200 import synth
    cen, rad, _, _ = synth.read_pqr(os.path.join(golden_dir("cfg0"), "molA.pqr"))
    cen = np.ascontiguousarray(cen[:4], dtype=np.float64)
    rad = np.ascontiguousarray(rad[:4], dtype=np.float64)
    ctx = pb.CSystem(poles=16, salt=0.05)
    try:
        n_points = 30000
        ref = ctx.build_imats(cen, rad, n_points=n_points)
        assert ref.shape == (4, 16 ** 4)
        for call in range(2):
            out = np.full(ref.shape, np.nan)
            assert _call_static(ctx, cen, rad, n_points, out) == 0, pb.lib().pbsam_last_error()
            assert np.all(np.isfinite(out)), "call %d" % call
            assert rel(out, ref) < TOL, "call %d: %.3e" % (call, rel(out, ref))
    finally:
        ctx.close()


def test_static_imat_rejects_orders_beyond_its_buffer():
    import pbsam_b200 as pb
    ctx = pb.CSystem(poles=20, salt=0.05)
    try:
        cen = np.zeros((1, 3))
        rad = np.array([3.0])
        out = np.zeros(20 ** 4)
        rc = _call_static(ctx, cen, rad, 1000, out)
        assert rc == -1   # PBSAM_E_BADARG
        assert b"exceeds the maximum" in pb.lib().pbsam_last_error()
    finally:
        ctx.close()
