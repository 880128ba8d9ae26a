"""The exact form and its backward pass on the GPU (through the C ABI).

Exact form (pbsam_params.exact = 1): each sphere's inner F/H fixed point solved
directly, every polarized sphere swept to the fixed point, forces and torques the
negative gradient of the lab-frame energy by the adjoint.  Checked:
  * the converged lab-frame energy against the oracle's exact form (1e-10 relative);
  * pbsam_system_backward against the oracle's backward pass, whose operators are
    explicit and exactly transposed (1e-8 relative);
  * the backward pass against central differences of the GPU's own lab-frame energy,
    h = 1e-3 A and 1e-4 rad (1e-6 relative), every perturbed pose one system of a
    batch;
  * compute_forces = -dU/dpos and -dU/domega, and dU/dquat along a tangent direction;
  * an 8-molecule case (40 spheres each, p = 10) against central differences;
  * the precomputed intra near-field operators against the plain transforms (numeric
    expansions of the surface charges, rotation + translation).
The reference's own forces (per-coordinate gradient solves) are printed beside the
adjoint's, not gated: they differentiate a different function (the reference's
energy ignores the orientation, and its sweeps stop short of the fixed point).
"""
import json
import os

import numpy as np
import pytest

import oracle
from conftest import golden_dir

pytestmark = pytest.mark.gpu
H_POS, H_ROT = 1e-3, 1e-4


def rel(a, b):
    b = np.asarray(b)
    return float(np.max(np.abs(np.asarray(a) - b)) / max(np.max(np.abs(b)), 1e-300))


def qmul(a, b):
    w1, v1, w2, v2 = a[0], np.asarray(a[1:]), b[0], np.asarray(b[1:])
    return np.concatenate([[w1 * w2 - v1 @ v2], w1 * v2 + w2 * v1 + np.cross(v1, v2)])


def axis_quat(c, ang):
    v = np.zeros(3)
    v[c] = np.sin(ang / 2)
    return np.concatenate([[np.cos(ang / 2)], v])


def fd_batch(pos, quat):
    """Base pose plus +-h along every position axis and +-angle about every lab axis,
    for every molecule: [1 + 12 n_mol] systems."""
    n = pos.shape[0]
    P, Q = [pos], [quat]
    for i in range(n):
        for c in range(3):
            for s in (1, -1):
                p = pos.copy()
                p[i, c] += s * H_POS
                P.append(p)
                Q.append(quat)
            for s in (1, -1):
                q = quat.copy()
                q[i] = qmul(axis_quat(c, s * H_ROT), quat[i])
                P.append(pos)
                Q.append(q)
    return np.array(P), np.array(Q)


def fd_grad(E, n):
    E = E[1:].reshape(n, 3, 4)
    return (E[:, :, 0] - E[:, :, 1]) / (2 * H_POS), (E[:, :, 2] - E[:, :, 3]) / (2 * H_ROT)


def exact_ctx(case, **kw):
    import pbsam_b200 as pb
    P = json.load(open(os.path.join(golden_dir(case), "poses.json")))
    ctx = pb.CSystem(poles=P["poles"], salt=P["salt"], idiel=P["idiel"], exact=1, max_pol_rounds=400, **kw)
    d = golden_dir(case)
    types = [ctx.load_moltype(d + "/mol%s.pqr" % t, d + "/im" + t, d + "/exp" + t, "mol%s.0" % t) for t in "AB"]
    return ctx, types, P


def frame_of(P, k):
    fr = P["poses"][k]["frame"]
    pos = np.array([m["pos"] for m in fr], float)
    quat = np.array([m["quat"] for m in fr], float)
    return pos, quat / np.linalg.norm(quat, axis=1, keepdims=True)


@pytest.mark.parametrize("case,pose", [("tiny", 0), ("cfg0", 3)])
def test_exact_backward_vs_oracle_and_central_differences(case, pose, tmp_path):
    import pbsam_b200 as pb
    ctx, types, P = exact_ctx(case)
    try:
        pos, quat = frame_of(P, pose)
        Pb, Qb = fd_batch(pos, quat)
        mol = ctx.molecules(types, n_systems=len(Pb))
        mol.set_poses(Pb, Qb)
        f, t, st = mol.compute_forces()
        assert np.all(st == 0), st
        stats = mol.stats()
        assert stats[0, 2] > 0, "the base pose must polarize"
        E = mol.compute_energy(lab=True)
        dp, dq, dr = mol.backward()
        # forces and torques are the negative gradient
        assert np.array_equal(f[0], -dp[0]) and np.array_equal(t[0], -dr[0])
        fdp, fdr = fd_grad(E, pos.shape[0])
        ep, er = rel(dp[0], fdp), rel(dr[0], fdr)
        assert ep < 1e-6 and er < 1e-6, (ep, er)
        # dU/dquat along a tangent direction dq = (1/2)(0, w) q is w . dU/dw
        w = np.array([0.3, -0.2, 0.5])
        for i in range(pos.shape[0]):
            tang = 0.5 * qmul(np.concatenate([[0.0], w]), quat[i])
            assert abs(dq[0, i] @ tang - w @ dr[0, i]) <= 1e-12 * max(1.0, np.abs(dr[0, i]).max())
            assert abs(dq[0, i] @ quat[i]) <= 1e-12 * max(1.0, np.abs(dq[0, i]).max())
        # the oracle's exact form and backward pass
        spec, out = str(tmp_path / "s.txt"), str(tmp_path / "s.out")
        frame = [(0, pos[0], quat[0]), (1, pos[1], quat[1])]
        oracle.write_spec(spec, oracle.golden_moltypes(golden_dir(case)), [frame], salt=P["salt"], idiel=P["idiel"],
                          poles=P["poles"], tol=(0.0, 0.0, 100, 400), energy=2, backward=1, nograd=1, exact=1)
        o = oracle.run_spec(spec, out)[0]
        assert abs(E[0] - o["energy_lab"]) <= 1e-10 * abs(o["energy_lab"])
        eo_p, eo_r = rel(dp[0], o["dpos"]), rel(dr[0], o["drot"])
        assert eo_p < 1e-8 and eo_r < 1e-8, (eo_p, eo_r)
        # the per-system seed scales the outputs
        sd = np.arange(1, len(Pb) + 1, dtype=float)
        dp2, _, _ = mol.backward(seed=sd)
        assert np.allclose(dp2[3], 4.0 * dp[3], rtol=1e-15, atol=0)
        print("%s pose %d: backward vs central differences %.2e (pos) %.2e (rot); vs oracle %.2e %.2e" % (
            case, pose, ep, er, eo_p, eo_r))
        mol.close()
    finally:
        ctx.close()


@pytest.mark.parametrize("case", ["tiny", "cfg0"])
def test_exact_operators_agree_with_plain_transforms(case):
    """The intra near-field operators and the exposed points' angles prepared once per
    type (exact_tables = 1) against the plain transforms and the per-call angles at
    every use (0): every pose of the case, forces and torques (the backward pass) and
    the lab-frame energy to 1e-11 relative."""
    res = []
    for tables in (1, 0):
        ctx, types, P = exact_ctx(case, exact_tables=tables)
        try:
            fr = [frame_of(P, k) for k in range(len(P["poses"]))]
            mol = ctx.molecules(types, n_systems=len(fr))
            mol.set_poses(np.array([f[0] for f in fr]), np.array([f[1] for f in fr]))
            f, t, st = mol.compute_forces()
            assert np.all(st == 0), st
            res.append((f, t, mol.compute_energy(lab=True), mol.stats()[:, 2].copy()))
            mol.close()
        finally:
            ctx.close()
    (f1, t1, e1, n1), (f0, t0, e0, n0) = res
    assert np.sum(n1) > 0
    ef, et, ee = rel(f1, f0), rel(t1, t0), rel(e1, e0)
    print("%s: operators vs plain transforms: force %.2e torque %.2e energy %.2e" % (case, ef, et, ee))
    assert ef < 1e-11 and et < 1e-11 and ee < 1e-11, (ef, et, ee)


def test_exact_reference_forces_reported():
    """The reference's forces (the plain drop-in: its per-coordinate gradient solves)
    beside the adjoint's, reported only."""
    from test_gpu_parity import make_ctx
    case = "cfg0"
    ctx, types, P = exact_ctx(case)
    pctx, ptypes = make_ctx(case)
    try:
        pos, quat = frame_of(P, 3)
        m1 = ctx.molecules(types, 1)
        m1.set_poses(pos[None], quat[None])
        f1, t1, _ = m1.compute_forces()
        m2 = pctx.molecules(ptypes, 1)
        m2.set_poses(pos[None], quat[None])
        f2, t2, _ = m2.compute_forces()
        print("adjoint force on B %s, reference %s; relative difference %.3f" % (f1[0, 1], f2[0, 1],
                                                                                 rel(f2[0], f1[0])))
        assert np.all(np.isfinite(f1)) and np.all(np.isfinite(t1))
        m1.close()
        m2.close()
    finally:
        ctx.close()
        pctx.close()


def test_exact_eight_molecules_central_differences():
    """Config-2 shape: 8 molecules of 40 spheres (r 3-6 A, 1200 charges in [-0.6, 0.6],
    net charge in {-3..3}), p = 10, packed so that neighbours polarize each other;
    the backward pass against central differences of the lab-frame energy."""
    import pbsam_b200 as pb
    from pbsam_b200 import synth, workload
    rng = np.random.default_rng(4242)
    mols = [synth.make_molecule(40, 3.0, 6.0, 1200, 0.6, float(rng.integers(-3, 4)), seed=5000 + k) for k in range(8)]
    prep = pb.CSystem(poles=10, salt=0.05)
    raw, tids, specs = [], [], []
    for m in mols:     # every type first: types are frozen once a system exists
        cen, rad, qp, q = workload._pqr_round(m)
        im = prep.build_imats(cen, rad, n_points=40000)
        raw.append((cen, rad, qp, q, im))
        tids.append(prep.create_moltype(cen, rad, qp, q, im, np.zeros((len(rad), 100)), np.zeros((len(rad), 100)),
                                        1.0 / rad))
    for t, r in zip(tids, raw):
        F, H, sc, _ = prep.self_polarize(t, max_rounds=6)
        specs.append(r + (F, H, sc))
    prep.close()
    ctx = pb.CSystem(poles=10, salt=0.05, exact=1, max_pol_rounds=400)
    try:
        types = [ctx.create_moltype(*sp) for sp in specs]
        quat = np.array([synth.random_quat(rng) for _ in range(8)])
        jitter = rng.uniform(-1.0, 1.0, (8, 3))
        corners = np.array([[x, y, z] for x in (0, 1) for y in (0, 1) for z in (0, 1)], float)
        # the tightest cube (0.5 A steps) whose molecules keep every gap above 1.5 A: the
        # molecules are elongated (extents 31-47 A), so several pairs sit inside the
        # 10 A polarization cutoff
        gaps = None
        for spacing in np.arange(10.0, 120.0, 0.5):
            pos = corners * spacing + jitter
            gaps = [synth.min_gap((mols[a].centres, mols[a].radii), pos[a], quat[a], (mols[b].centres, mols[b].radii),
                                  pos[b], quat[b]) for a in range(8) for b in range(a + 1, 8)]
            if min(gaps) > 1.5:
                break
        assert min(gaps) > 1.5 and sum(g < 10.0 for g in gaps) >= 2, gaps
        Pb, Qb = fd_batch(pos, quat)
        mol = ctx.molecules(types, n_systems=len(Pb))
        try:
            mol.set_poses(Pb, Qb)
            f, t, st = mol.compute_forces()
            assert np.all(st == 0), st
            assert mol.stats()[0, 2] > 0, "neighbours must polarize"
            E = mol.compute_energy(lab=True)
            dp, dq, dr = mol.backward()
            fdp, fdr = fd_grad(E, 8)
            ep, er = rel(dp[0], fdp), rel(dr[0], fdr)
            print("8 molecules: backward vs central differences %.2e (pos) %.2e (rot)" % (ep, er))
            assert ep < 1e-6 and er < 1e-6, (ep, er)
        finally:
            mol.close()
    finally:
        ctx.close()
