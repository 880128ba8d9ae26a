"""Potential at points (pbsam_system_potential) against the reference and the oracle.

CMolecule::computePotInSpace (src/moldynamics.cpp:470-506) is run by the reference's
own harness after computeForces on the same pose (oracle/ref_harness.cpp, potpoint
entries); the GPU evaluates the same state through the C ABI.  1e-8 relative, the bar
of the plain drop-in.  The lab-frame form is checked against the oracle and for
invariance under a rigid rotation of the system and the points together.
"""
import json
import os
import subprocess

import numpy as np
import pytest

import oracle
from conftest import golden_dir
from test_gpu_parity import make_ctx, rel

pytestmark = pytest.mark.gpu
PTS = np.array([[0.0, 0.0, 30.0], [5.0, -40.0, 12.0], [25.0, 10.0, -5.0], [-30.0, 2.0, 3.0], [12.0, 18.0, 22.0]])


def _frame(case, k):
    P = json.load(open(os.path.join(golden_dir(case), "poses.json")))
    fr = P["poses"][k]["frame"]
    return P, np.array([m["pos"] for m in fr], float), np.array([m["quat"] for m in fr], float)


def _reference_pot(case, P, pos, quat, tmp):
    exe = os.path.join(oracle.HERE, "_ref", "p%d_default" % P["poles"], "harness")
    if not os.path.exists(exe):
        pytest.skip("reference build missing (oracle/build_ref.py)")
    spec = os.path.join(tmp, "ref.txt")
    with open(spec, "w") as fh:
        fh.write("salt %r\nidiel %r\ndump 0\nenergy 0\n" % (P["salt"], P["idiel"]))
        for mt in oracle.golden_moltypes(golden_dir(case)):
            fh.write("moltype %s %s %s %s\n" % mt)
        fh.write("frame\n")
        for i in range(len(pos)):
            fh.write("mol %d %s %s\n" % (i, " ".join("%.17g" % v for v in pos[i]), " ".join("%.17g" % v for v in quat[i])))
        for pt in PTS:
            fh.write("potpoint %.17g %.17g %.17g\n" % tuple(pt))
    subprocess.run([exe, spec, spec + ".out"], check=True, env=dict(os.environ, OMP_NUM_THREADS="1"),
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    return oracle.parse(spec + ".out")[0]["pot"]


@pytest.mark.parametrize("case,pose", [("tiny", 0), ("cfg0", 3)])
def test_potential_vs_reference(case, pose, tmp_path):
    P, pos, quat = _frame(case, pose)
    ref = _reference_pot(case, P, pos, quat, str(tmp_path))
    ctx, types = make_ctx(case)
    try:
        mol = ctx.molecules(types, n_systems=2)
        mol.set_poses(np.array([pos, pos]), np.array([quat, quat]))
        f, t, st = mol.compute_forces()
        assert list(st) == [0, 0]
        pot = mol.potential(PTS)
        assert rel(pot[0], ref) < 1e-8 and rel(pot[1], ref) < 1e-8, (pot[0], ref)
        # per-system points: the second system gets the points in reverse order
        per = np.array([PTS, PTS[::-1]])
        pot2 = mol.potential(per)
        assert np.array_equal(pot2[0], pot[0]) and np.array_equal(pot2[1], pot[1][::-1])
        mol.close()
    finally:
        ctx.close()


def test_lab_potential_vs_oracle_and_rigid_motion(tmp_path):
    case = "cfg0"
    P, pos, quat = _frame(case, 3)
    ctx, types = make_ctx(case)
    try:
        mol = ctx.molecules(types, n_systems=2)
        # system 1: the whole system turned by g about the origin, the points with it
        g = np.array([0.8, 0.2, -0.4, 0.4])
        g /= np.linalg.norm(g)

        def rot(v):
            w, u = g[0], g[1:]
            return v + 2 * np.cross(u, np.cross(u, v) + w * v)

        def qmul(a, b):
            return np.concatenate([[a[0] * b[0] - a[1:] @ b[1:]], a[0] * b[1:] + b[0] * a[1:] + np.cross(a[1:], b[1:])])
        qn = quat / np.linalg.norm(quat, axis=1, keepdims=True)
        pos1 = np.array([rot(p) for p in pos])
        quat1 = np.array([qmul(g, q) for q in qn])
        mol.set_poses(np.array([pos, pos1]), np.array([qn, quat1]))
        mol.compute_forces()
        pts = np.array([PTS, np.array([rot(p) for p in PTS])])
        lab = mol.potential(pts, lab=True)
        spec, out = str(tmp_path / "s.txt"), str(tmp_path / "s.out")
        oracle.write_spec(spec, oracle.golden_moltypes(golden_dir(case)), [[(0, pos[0], qn[0]), (1, pos[1], qn[1])]],
                          salt=P["salt"], idiel=P["idiel"], poles=P["poles"], potpoints=PTS, potlab=1)
        o = oracle.run_spec(spec, out)[0]
        assert rel(lab[0], o["pot"]) < 1e-8, (lab[0], o["pot"])
        # a rigid rotation of everything leaves the lab-frame potential unchanged
        assert rel(lab[1], lab[0]) < 1e-8, rel(lab[1], lab[0])
        mol.close()
    finally:
        ctx.close()
