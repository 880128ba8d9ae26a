"""Mixed-precision mode (IMats stored in FP32, products accumulated in FP64) against
the FP64 path and the reference's fixtures.

Tolerance: forces and torques within 1e-6 relative of the FP64 results (max |a-b|
over max |b| per system), the bar for the mixed-precision form; energies within
1e-6 relative.  The FP64 path itself matches the reference within 1e-8, so the
same bound holds against the reference.
"""
import json
import os

import numpy as np
import pytest

import oracle
from conftest import golden_dir

pytestmark = pytest.mark.gpu
TOL = 1e-6


def rel(a, b):
    b = np.asarray(b)
    return float(np.max(np.abs(np.asarray(a) - b)) / max(np.max(np.abs(b)), 1e-300))


def run(case, fp32, tight=False):
    import pbsam_b200 as pb
    P = json.load(open(os.path.join(golden_dir(case), "poses.json")))
    tol = oracle.TIGHT_TOL if tight else oracle.DEFAULT_TOL
    ctx = pb.CSystem(poles=P["poles"], salt=P["salt"], idiel=P["idiel"], max_polar_dev=tol[0], solve_tol=tol[1],
                     solve_max_ct=tol[2], max_pol_rounds=tol[3], imat_fp32=int(fp32))
    d = golden_dir(case)
    types = [ctx.load_moltype(d + "/molA.pqr", d + "/imA", d + "/expA", "molA.0"),
             ctx.load_moltype(d + "/molB.pqr", d + "/imB", d + "/expB", "molB.0")]
    frames = [p["frame"] for p in P["poses"]]
    mol = ctx.molecules(types, n_systems=len(frames))
    mol.set_poses(np.array([[m["pos"] for m in fr] for fr in frames]),
                  np.array([[m["quat"] for m in fr] for fr in frames]))
    f, t, st = mol.compute_forces()
    e = mol.compute_energy()
    stats = mol.stats()
    mol.close()
    ctx.close()
    return f, t, st, e, stats


@pytest.mark.parametrize("case", ["tiny", "cfg0"])
@pytest.mark.parametrize("tight", [False, True])
def test_fp32_imat_close_to_fp64(case, tight):
    f64, t64, s64, e64, _ = run(case, False, tight)
    f32, t32, s32, e32, _ = run(case, True, tight)
    assert list(s32) == list(s64)
    errs = []
    for k in range(len(f64)):
        if not np.any(f64[k]):
            continue
        errs.append((rel(f32[k], f64[k]), rel(t32[k], t64[k]), abs(e32[k] - e64[k]) / abs(e64[k])))
    worst = np.max(np.array(errs), axis=0)
    assert worst[0] < TOL and worst[1] < TOL and worst[2] < TOL, "force/torque/energy rel err %s" % worst
