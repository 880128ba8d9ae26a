"""The multi-threaded CPU preparation (oracle/pbsam_prep.cpp) against the
reference's own `pbsam mat` and `pbsam spol` output files.

The benchmark's CPU arm makes its inputs with these two functions so that it never
loads the CUDA library; they must reproduce the reference's imat.sp<k>.out.bin
(1e-8 relative, the bar of the GPU builder) and its 8-digit .exp files (at most one
unit in the last digit apart).
"""
import json
import os

import numpy as np
import pytest

import oracle
from conftest import golden_dir
from test_gpu_setup import molecule, read_exp, read_imat, rel

TOL = 1e-8


@pytest.mark.parametrize("case,tag", [("tiny", "A"), ("tiny", "B"), ("cfg0", "A"), ("cfg0", "B")])
def test_prep_imats_vs_reference(case, tag):
    P = json.load(open(os.path.join(golden_dir(case), "poses.json")))
    cen, rad, _, _ = molecule(case, tag)
    got = oracle.prep_imats(P["poles"], cen, rad, n_points=250000)
    for k in range(len(rad)):
        p, ref = read_imat(os.path.join(golden_dir(case), "im" + tag, "imat.sp%d.out.bin" % k))
        assert p == P["poles"]
        assert rel(got[k], ref) < TOL, (k, rel(got[k], ref))


@pytest.mark.parametrize("case,tag", [("tiny", "A"), ("tiny", "B"), ("cfg0", "A"), ("cfg0", "B")])
def test_prep_selfpol_vs_reference(case, tag):
    P = json.load(open(os.path.join(golden_dir(case), "poses.json")))
    cen, rad, pos, q = molecule(case, tag)
    imats = np.stack([read_imat(os.path.join(golden_dir(case), "im" + tag, "imat.sp%d.out.bin" % k))[1]
                      for k in range(len(rad))])
    F, H, sc, sweeps = oracle.prep_selfpol(P["poles"], cen, rad, pos, q, imats, salt=P["salt"], idiel=P["idiel"])
    assert 1 <= sweeps < 1700
    for k in range(len(rad)):
        scF, refF = read_exp(os.path.join(golden_dir(case), "exp" + tag, "mol%s.0.%d.F.exp" % (tag, k)))
        scH, refH = read_exp(os.path.join(golden_dir(case), "exp" + tag, "mol%s.0.%d.H.exp" % (tag, k)))
        assert abs(sc[k] - scH) <= 1e-8 * abs(scH)
        assert np.max(np.abs(F[k] - refF)) <= 2e-8 * np.max(np.abs(refF)), k
        assert np.max(np.abs(H[k] - refH)) <= 2e-8 * np.max(np.abs(refH)), k


def test_prep_inputs_feed_the_oracle_like_the_reference_files(tmp_path):
    """Inputs made by the preparation, written in the reference's formats, give the
    same forces in the oracle as the reference's own files (p = 6 case)."""
    from pbsam_b200 import workload
    case = "tiny"
    d = golden_dir(case)
    P = json.load(open(os.path.join(d, "poses.json")))
    specs = []
    for tag in "AB":
        cen, rad, pos, q = molecule(case, tag)
        im = oracle.prep_imats(P["poles"], cen, rad)
        F, H, sc, _ = oracle.prep_selfpol(P["poles"], cen, rad, pos, q, im, salt=P["salt"], idiel=P["idiel"])
        specs.append((tag, cen, rad, pos, q, im, F, H, sc))
    out = str(tmp_path)
    files = []
    for tag, cen, rad, pos, q, im, F, H, sc in specs:
        os.makedirs(os.path.join(out, "im" + tag))
        os.makedirs(os.path.join(out, "exp" + tag))
        for k in range(len(rad)):
            workload.write_imat(os.path.join(out, "im" + tag, "imat.sp%d.out.bin" % k), im[k], P["poles"])
            workload.write_exp(os.path.join(out, "exp" + tag, "mol%s.0.%d.F.exp" % (tag, k)), F[k], P["poles"], sc[k])
            workload.write_exp(os.path.join(out, "exp" + tag, "mol%s.0.%d.H.exp" % (tag, k)), H[k], P["poles"], sc[k])
        files.append((os.path.join(d, "mol%s.pqr" % tag), os.path.join(out, "im" + tag),
                      os.path.join(out, "exp" + tag), "mol%s.0" % tag))
    fr = P["poses"][0]["frame"]
    a = oracle.run_spec(_spec(tmp_path, "a", files, fr, P), str(tmp_path / "a.out"))[0]
    b = oracle.run_spec(_spec(tmp_path, "b", oracle.golden_moltypes(d), fr, P), str(tmp_path / "b.out"))[0]
    assert rel(a["force"], b["force"]) < 1e-8 and rel(a["torque"], b["torque"]) < 1e-8


def _spec(tmp_path, name, files, fr, P):
    path = str(tmp_path / (name + ".txt"))
    oracle.write_spec(path, files, oracle.golden_frames(fr), salt=P["salt"], idiel=P["idiel"], poles=P["poles"])
    return path
