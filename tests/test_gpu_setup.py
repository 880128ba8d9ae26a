"""Molecule-type preparation on the GPU against the reference's own files.

The golden fixtures hold the reference's `pbsam mat` output (imat.sp<k>.out.bin,
250 000 quadrature points) and `pbsam spol` output (<name>.0.<k>.{F,H}.exp, 8
significant digits) for the same PQR files; pbsam_imat_build and pbsam_selfpol must
reproduce them.
"""
import os
import struct

import numpy as np
import pytest

from conftest import golden_dir

pytestmark = pytest.mark.gpu
TOL = 1e-8


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def read_imat(path):
    b = open(path, "rb").read()
    p = struct.unpack("i", b[:4])[0]
    return p, np.frombuffer(b[4:4 + 8 * p ** 4], dtype=np.float64).copy()


def read_exp(path):
    """.exp text (src/readutil.cpp:541-556): poles, scale, 1000, then degree rows."""
    t = open(path).read().split()
    p, scale = int(t[0]), float(t[1])
    vals = np.array([float(x) for x in t[3:3 + p * p]])
    return scale, vals


def molecule(case, tag):
    from pbsam_b200 import synth
    cen, rad, pos, q = synth.read_pqr(os.path.join(golden_dir(case), "mol%s.pqr" % tag))
    return [np.ascontiguousarray(a, dtype=np.float64) for a in (cen, rad, pos, q)]


@pytest.mark.parametrize("case,tag", [("cfg0", "A"), ("cfg0", "B"), ("tiny", "A")])
def test_imat_builder_vs_reference(case, tag):
    import json
    import pbsam_b200 as pb
    P = json.load(open(os.path.join(golden_dir(case), "poses.json")))
    cen, rad, _, _ = molecule(case, tag)
    ctx = pb.CSystem(poles=P["poles"], salt=P["salt"])
    try:
        got = ctx.build_imats(cen, rad, n_points=250000)
    finally:
        ctx.close()
    for k in range(len(rad)):
        p, ref = read_imat(os.path.join(golden_dir(case), "im" + tag, "imat.sp%d.out.bin" % k))
        assert p == P["poles"]
        assert rel(got[k], ref) < TOL, (k, rel(got[k], ref))


@pytest.mark.parametrize("case,tag", [("cfg0", "A"), ("tiny", "B")])
def test_selfpol_vs_reference(case, tag):
    """Self-polarization from the reference's IMats reproduces its .exp files (both
    are rounded to 8 significant digits, so one unit in the last digit may differ)."""
    import json
    import pbsam_b200 as pb
    P = json.load(open(os.path.join(golden_dir(case), "poses.json")))
    cen, rad, pos, q = molecule(case, tag)
    n, P2 = len(rad), P["poles"] ** 2
    imats = np.stack([read_imat(os.path.join(golden_dir(case), "im" + tag, "imat.sp%d.out.bin" % k))[1]
                      for k in range(n)])
    ctx = pb.CSystem(poles=P["poles"], salt=P["salt"], idiel=P["idiel"])
    try:
        t = ctx.create_moltype(cen, rad, pos, q, imats, np.zeros((n, P2)), np.zeros((n, P2)), 1.0 / rad)
        F, H, sc, sweeps = ctx.self_polarize(t)
    finally:
        ctx.close()
    assert 1 <= sweeps < 1700
    for k in range(n):
        scF, refF = read_exp(os.path.join(golden_dir(case), "exp" + tag, "mol%s.0.%d.F.exp" % (tag, k)))
        scH, refH = read_exp(os.path.join(golden_dir(case), "exp" + tag, "mol%s.0.%d.H.exp" % (tag, k)))
        assert abs(sc[k] - scH) <= 1e-8 * abs(scH)
        assert np.max(np.abs(F[k] - refF)) <= 2e-8 * np.max(np.abs(refF)), k
        assert np.max(np.abs(H[k] - refH)) <= 2e-8 * np.max(np.abs(refH)), k
