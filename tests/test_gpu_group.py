"""Groups of system handles (pbsam_group_*): systems of different molecule lists,
sphere counts and pole orders in one launch.

* Forces: handles of the p = 6 golden molecules in two molecule lists ([A, B] and
  [B, A, A]) and of the p = 10 ones, evaluated by their own calls and then, from the
  same starting state, by one group launch: every force, torque and status equal bit
  for bit (one CTA per system in both), in the creation order and after tune().
* Brownian dynamics: NAM handles of both molecule lists and a three-molecule MULTI
  handle stepped by their own graphs and, from the same start, by the group's graph:
  poses, statuses, steps and times equal bit for bit (the noise is per system).
"""
import json
import os

import numpy as np
import pytest

from conftest import golden_dir

pytestmark = pytest.mark.gpu


def _ctx(case):
    import pbsam_b200 as pb
    P = json.load(open(os.path.join(golden_dir(case), "poses.json")))
    ctx = pb.CSystem(poles=P["poles"], salt=P["salt"], idiel=P["idiel"], cluster_size=1)
    d = golden_dir(case)
    types = [ctx.load_moltype(d + "/mol%s.pqr" % t, d + "/im" + t, d + "/exp" + t, "mol%s.0" % t) for t in "AB"]
    return ctx, types, P


def _frames(P, idx):
    out = []
    for k in idx:
        fr = P["poses"][k]["frame"]
        out.append((np.array([m["pos"] for m in fr], float), np.array([m["quat"] for m in fr], float)))
    return out


def _handles(tiny, cfg0):
    (ct, tt, Pt), (cc, tc, Pc) = tiny, cfg0
    h1 = ct.molecules([tt[0], tt[1]], n_systems=3)
    fr = _frames(Pt, [0, 1, 2])
    h1.set_poses(np.array([f[0] for f in fr]), np.array([f[1] for f in fr]))
    # [B, A, A]: the two golden molecules and a third copy of A far out along x
    h2 = ct.molecules([tt[1], tt[0], tt[0]], n_systems=2)
    pos2, quat2 = [], []
    for p, q in _frames(Pt, [0, 1]):
        pos2.append([p[1], p[0], p[0] + np.array([60.0, 0.0, 0.0])])
        quat2.append([q[1], q[0], [1.0, 0.0, 0.0, 0.0]])
    h2.set_poses(np.array(pos2), np.array(quat2))
    h3 = cc.molecules([tc[0], tc[1]], n_systems=2)
    fr = _frames(Pc, [1, 3])
    h3.set_poses(np.array([f[0] for f in fr]), np.array([f[1] for f in fr]))
    return [h1, h2, h3]


def test_group_forces_equal_each_handles_own():
    import pbsam_b200 as pb
    tiny, cfg0 = _ctx("tiny"), _ctx("cfg0")
    hs = _handles(tiny, cfg0)
    try:
        own = [h.compute_forces() for h in hs]
        assert all(np.all(o[2] == 0) for o in own)
        g = pb.Group(hs)
        for tune in (False, True):
            for h in hs:
                h.reset()
            if tune:
                g.tune()
            got = g.compute_forces()
            for o, r in zip(own, got):
                for a, b in zip(o, r):
                    assert np.array_equal(a, b)
        g.close()
    finally:
        for h in hs:
            h.close()
        tiny[0].close()
        cfg0[0].close()


def test_group_bd_equals_each_handles_own():
    import pbsam_b200 as pb
    ct, tt, Pt = _ctx("tiny")
    dtr2, drot2 = (0.0, 0.03), (4.5e-5, 4e-5)
    dtr3, drot3 = (0.015, 0.015, 0.015), (4.5e-5, 4.5e-5, 4e-5)

    def make():
        a = ct.molecules([tt[0], tt[1]], n_systems=3)
        fr = _frames(Pt, [0, 1, 2])
        a.set_poses(np.array([f[0] for f in fr]), np.array([f[1] for f in fr]))
        a.bd_init(dtr2, drot2, mode=pb.PBSAM_BD_NAM, seed=5)
        b = ct.molecules([tt[1], tt[0]], n_systems=2)
        fr = _frames(Pt, [1, 0])
        b.set_poses(np.array([f[0][::-1] for f in fr]), np.array([f[1][::-1] for f in fr]))
        b.bd_init(dtr2, drot2, mode=pb.PBSAM_BD_NAM, seed=9)
        c = ct.molecules([tt[0], tt[0], tt[1]], n_systems=2)
        p0, q0 = _frames(Pt, [1])[0]
        pos = np.array([[p0[0], p0[0] - p0[1], p0[1]]] * 2)
        quat = np.array([[q0[0], [0.5, 0.5, -0.5, 0.5], q0[1]]] * 2)
        c.set_poses(pos, quat)
        c.bd_init(dtr3, drot3, mode=pb.PBSAM_BD_MULTI, seed=13)
        return [a, b, c]
    own = make()
    grp = make()
    try:
        for h in own:
            h.bd_run(6)
        ref = [h.bd_state() for h in own]
        g = pb.Group(grp)
        g.bd_run(3)
        g.tune()
        g.bd_run(3)
        got = [h.bd_state() for h in grp]
        for r, s in zip(ref, got):
            assert set(r) == set(s)
            for k in r:
                assert np.array_equal(r[k], s[k]), k
            assert np.all(s["steps"] == 6)
        g.close()
    finally:
        for h in own + grp:
            h.close()
        ct.close()
