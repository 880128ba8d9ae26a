"""Failure statuses of the C ABI, provoked on the host (no GPU fault is involved).

The reference reports these cases by printing and exiting, or not at all:
  * a missing or short IMat / expansion file makes readMats / readExpansionsP exit
    (src/readutil.cpp:290-294, 406-410); here pbsam_moltype_load returns PBSAM_E_IO;
  * a non-finite or blown-up expansion (CExpan::isBlownup, src/expansion.h:216-221)
    goes unnoticed; here the system reports PBSAM_SYS_NAN;
  * a sweep loop that stops at MAX_POL_ROUNDS prints "Polarization does not
    converge" (src/molecule.cpp:1963-1967) and carries on; here the system reports
    PBSAM_SYS_NOT_CONVERGED and still returns its forces.
Every case is an ordinary call with bad input: the kernels run to completion.
"""
import os
import shutil

import numpy as np
import pytest

import oracle
from conftest import golden_dir
from test_gpu_parity import frame_arrays, make_ctx, poses, rel

pytestmark = pytest.mark.gpu


def _copy_case(tmp_path, case="tiny"):
    d = str(tmp_path / case)
    shutil.copytree(golden_dir(case), d)
    return d


def _load(ctx, d, tag):
    return ctx.load_moltype(d + "/mol%s.pqr" % tag, d + "/im" + tag, d + "/exp" + tag, "mol%s.0" % tag)


def _err_ctx():
    import pbsam_b200 as pb
    P = poses("tiny")
    return pb.CSystem(poles=P["poles"], salt=P["salt"], idiel=P["idiel"])


def test_truncated_imat_is_an_io_error(tmp_path):
    import pbsam_b200 as pb
    d = _copy_case(tmp_path)
    fn = os.path.join(d, "imA", "imat.sp1.out.bin")
    data = open(fn, "rb").read()
    open(fn, "wb").write(data[: len(data) // 2])
    ctx = _err_ctx()
    try:
        with pytest.raises(pb.PbsamError) as e:
            _load(ctx, d, "A")
        assert e.value.code == -2 and b"imat.sp1.out.bin" in pb.lib().pbsam_last_error()
        # the context stays usable: an intact type still loads
        assert _load(ctx, golden_dir("tiny"), "B") == 0
    finally:
        ctx.close()


def test_missing_imat_and_short_header_are_io_errors(tmp_path):
    import pbsam_b200 as pb
    d = _copy_case(tmp_path)
    os.remove(os.path.join(d, "imA", "imat.sp0.out.bin"))
    fn = os.path.join(d, "imB", "imat.sp2.out.bin")
    open(fn, "wb").write(b"\x01\x00")
    ctx = _err_ctx()
    try:
        for tag in ("A", "B"):
            with pytest.raises(pb.PbsamError) as e:
                _load(ctx, d, tag)
            assert e.value.code == -2
    finally:
        ctx.close()


def test_malformed_expansion_file_is_an_io_error(tmp_path):
    import pbsam_b200 as pb
    d = _copy_case(tmp_path)
    fn = os.path.join(d, "expA", "molA.0.2.H.exp")
    lines = open(fn).read().split("\n")
    open(fn, "w").write("\n".join(lines[:4] + ["0.1 garbage 0.3"] + lines[5:]))
    fn2 = os.path.join(d, "expB", "molB.0.0.F.exp")
    open(fn2, "w").write("6\n")
    ctx = _err_ctx()
    try:
        for tag, name in (("A", b"molA.0.2.H.exp"), ("B", b"molB.0.0.F.exp")):
            with pytest.raises(pb.PbsamError) as e:
                _load(ctx, d, tag)
            assert e.value.code == -2 and name in pb.lib().pbsam_last_error()
    finally:
        ctx.close()


def test_non_finite_moltype_input_is_refused():
    import pbsam_b200 as pb
    from pbsam_b200 import synth
    cen, rad, pos, q = synth.read_pqr(os.path.join(golden_dir("tiny"), "molA.pqr"))
    ctx = _err_ctx()
    try:
        P2 = ctx.params.poles ** 2
        ns = len(rad)
        im = np.zeros((ns, P2 * P2))
        F = np.zeros((ns, P2))
        H = np.zeros((ns, P2))
        H[1, 3] = np.nan
        with pytest.raises(pb.PbsamError) as e:
            ctx.create_moltype(cen, rad, pos, q, im, F, H, 1.0 / rad)
        assert e.value.code == -1
        im[0, 7] = np.inf
        H[1, 3] = 0.0
        with pytest.raises(pb.PbsamError):
            ctx.create_moltype(cen, rad, pos, q, im, F, H, 1.0 / rad)
    finally:
        ctx.close()


def test_nan_pose_reports_sys_nan_and_spares_the_batch():
    import pbsam_b200 as pb
    ctx, types = make_ctx("tiny")
    try:
        fr = poses("tiny")["poses"][0]["frame"]
        pos, quat = frame_arrays([fr, fr, fr])
        pos[0, 1, 2] = np.nan
        quat[2, 0] = 0.0
        mol = ctx.molecules(types, n_systems=3)
        mol.set_poses(pos, quat)
        f, t, st = mol.compute_forces()
        assert st[0] == pb.PBSAM_SYS_NAN and st[2] == pb.PBSAM_SYS_NAN
        assert np.all(f[0] == 0) and np.all(t[2] == 0)
        ref = oracle.parse(os.path.join(golden_dir("tiny"), "ref_default", "pose0.txt"))[0]
        assert st[1] == pb.PBSAM_SYS_OK
        assert rel(f[1], ref["force"]) < 1e-8 and rel(t[1], ref["torque"]) < 1e-8
        # the next call with a good pose in the refused slot is back to normal
        pos[0, 1, 2] = pos[1, 1, 2]
        quat[2] = quat[1]
        mol.reset()
        mol.set_poses(pos, quat)
        f, t, st = mol.compute_forces()
        assert list(st) == [0, 0, 0]
        assert rel(f[0], ref["force"]) < 1e-8 and rel(f[2], ref["force"]) < 1e-8
        mol.close()
    finally:
        ctx.close()


def test_sweep_cap_reports_not_converged_with_forces():
    import pbsam_b200 as pb
    P = poses("cfg0")
    ctx = pb.CSystem(poles=P["poles"], salt=P["salt"], idiel=P["idiel"], max_polar_dev=0.0, solve_tol=1e-8,
                     solve_max_ct=100, max_pol_rounds=2)
    d = golden_dir("cfg0")
    try:
        types = [_load(ctx, d, "A"), _load(ctx, d, "B")]
        frames = [p["frame"] for p in P["poses"]]
        mol = ctx.molecules(types, n_systems=len(frames))
        pos, quat = frame_arrays(frames)
        mol.set_poses(pos, quat)
        f, t, st = mol.compute_forces()
        stats = mol.stats()
        polarized = stats[:, 2] > 0     # poses with a mutual polarization solve
        assert np.any(polarized)
        for k in range(len(frames)):
            if polarized[k]:
                assert st[k] == pb.PBSAM_SYS_NOT_CONVERGED, (k, st[k])
                assert stats[k, 0] == 2 and (stats[k, 4] & 1)
                assert np.all(np.isfinite(f[k])) and np.any(f[k] != 0)
            else:
                assert st[k] == pb.PBSAM_SYS_OK
        # the energy is still evaluated for a system whose sweeps stopped at the cap
        e = mol.compute_energy()
        assert np.all(np.isfinite(e)) and np.all(e[polarized] != 0)
        mol.close()
    finally:
        ctx.close()
