"""The oracle's adjoint of the converged polarization against central differences.

The exact form of the solve: every sphere's inner F/H fixed point solved directly
(the reference iterates it, src/expcenter.cpp:1079-1135, and on these spheres the
iteration matrix has spectral radius above one, so its result drifts with
SOLVE_MAX_CT), and every polarized sphere swept until nothing changes (the
reference's selective update, src/molecule.cpp:2057, can leave a sphere out of
date).  The lab-frame interaction energy of that converged state is a smooth
function of the poses; the oracle's backward pass (explicit, exactly transposed
operators) must give its gradient to 1e-6 relative of central differences with
h = 1e-3 A and 1e-4 rad.  The case also checks that the reference's capped
iteration does not define such a function: its energy moves with the cap.
"""
import json
import os

import numpy as np

import oracle
from conftest import golden_dir

EXACT = (0.0, 0.0, 100, 200)    # no early stop: sweep to the fixed point
H_POS, H_ROT = 1e-3, 1e-4


def _qmul(a, b):
    w1, v1, w2, v2 = a[0], np.asarray(a[1:]), b[0], np.asarray(b[1:])
    return np.concatenate([[w1 * w2 - v1 @ v2], w1 * v2 + w2 * v1 + np.cross(v1, v2)])


def _axis_quat(c, ang):
    v = np.zeros(3)
    v[c] = np.sin(ang / 2)
    return np.concatenate([[np.cos(ang / 2)], v])


def _run(tmp, case, P, frames, backward=0, exact=1, tol=EXACT):
    spec, out = os.path.join(tmp, "s.txt"), os.path.join(tmp, "s.out")
    oracle.write_spec(spec, oracle.golden_moltypes(golden_dir(case)), frames, salt=P["salt"], idiel=P["idiel"],
                      poles=P["poles"], tol=tol, energy=2, backward=backward, nograd=1, exact=exact)
    return oracle.run_spec(spec, out)


def test_oracle_backward_matches_central_differences(tmp_path):
    case = "tiny"
    P = json.load(open(os.path.join(golden_dir(case), "poses.json")))
    fr = P["poses"][0]["frame"]
    base = [(m["type"], np.array(m["pos"], float), np.array(m["quat"], float) / np.linalg.norm(m["quat"]))
            for m in fr]
    r = _run(str(tmp_path), case, P, [base], backward=1)[0]
    assert int(r["info"][r["info"].index("solves") + 1]) > 0, "the pose must polarize"
    frames = []
    for i in range(len(base)):
        for c in range(3):
            for s in (1, -1):
                f = [(t, p.copy(), q.copy()) for t, p, q in base]
                f[i][1][c] += s * H_POS
                frames.append(f)
            for s in (1, -1):
                f = [(t, p.copy(), q.copy()) for t, p, q in base]
                f[i] = (f[i][0], f[i][1], _qmul(_axis_quat(c, s * H_ROT), f[i][2]))
                frames.append(f)
    # every frame in a fresh solver state (one run each)
    E = np.array([_run(str(tmp_path), case, P, [f])[0]["energy_lab"] for f in frames]).reshape(len(base), 3, 4)
    fd_pos = (E[:, :, 0] - E[:, :, 1]) / (2 * H_POS)
    fd_rot = (E[:, :, 2] - E[:, :, 3]) / (2 * H_ROT)
    err_pos = np.max(np.abs(r["dpos"] - fd_pos)) / np.max(np.abs(fd_pos))
    err_rot = np.max(np.abs(r["drot"] - fd_rot)) / np.max(np.abs(fd_rot))
    assert err_pos < 1e-6 and err_rot < 1e-6, (err_pos, err_rot)
    # translation invariance of the lab-frame energy
    assert np.max(np.abs(r["dpos"].sum(axis=0))) < 1e-12 * np.max(np.abs(r["dpos"]))


def test_reference_iteration_depends_on_its_cap(tmp_path):
    """The reference's inner iteration run to a fixed count drifts: its energy at 300
    and 1000 inner iterations differs far more than the exact form's at 20 and 60
    outer sweeps."""
    case = "tiny"
    P = json.load(open(os.path.join(golden_dir(case), "poses.json")))
    fr = [(m["type"], m["pos"], m["quat"]) for m in P["poses"][0]["frame"]]
    e300 = _run(str(tmp_path), case, P, [fr], exact=0, tol=(0.0, 0.0, 300, 150))[0]["energy_lab"]
    e1000 = _run(str(tmp_path), case, P, [fr], exact=0, tol=(0.0, 0.0, 1000, 150))[0]["energy_lab"]
    x20 = _run(str(tmp_path), case, P, [fr], tol=(0.0, 0.0, 100, 20))[0]["energy_lab"]
    x60 = _run(str(tmp_path), case, P, [fr], tol=(0.0, 0.0, 100, 60))[0]["energy_lab"]
    assert abs(e1000 - e300) > 1e-5 * abs(e300)
    assert abs(x60 - x20) < 1e-7 * abs(x60)
