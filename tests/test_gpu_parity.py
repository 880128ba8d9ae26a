"""CUDA drop-in (through the C ABI) against the reference and the oracle.

Tolerance: energies, forces and torques within 1e-8 relative (the bar set for
the plain FP64 drop-in), measured as max |a-b| / max |b| over each system's
force (torque) components.
"""
import json
import os

import numpy as np
import pytest

import oracle
from conftest import golden_dir

pytestmark = pytest.mark.gpu
TOL = 1e-8


def rel(a, b):
    b = np.asarray(b)
    return float(np.max(np.abs(np.asarray(a) - b)) / max(np.max(np.abs(b)), 1e-300))


def poses(case):
    return json.load(open(os.path.join(golden_dir(case), "poses.json")))


def make_ctx(case, tight=False, cluster_size=0):
    import pbsam_b200 as pb
    P = poses(case)
    tol = oracle.TIGHT_TOL if tight else oracle.DEFAULT_TOL
    ctx = pb.CSystem(poles=P["poles"], salt=P["salt"], idiel=P["idiel"], max_polar_dev=tol[0],
                     solve_tol=tol[1], solve_max_ct=tol[2], max_pol_rounds=tol[3], cluster_size=cluster_size)
    d = golden_dir(case)
    ta = ctx.load_moltype(d + "/molA.pqr", d + "/imA", d + "/expA", "molA.0")
    tb = ctx.load_moltype(d + "/molB.pqr", d + "/imB", d + "/expB", "molB.0")
    return ctx, [ta, tb]


def frame_arrays(frames):
    pos = np.array([[m["pos"] for m in fr] for fr in frames])
    quat = np.array([[m["quat"] for m in fr] for fr in frames])
    return pos, quat


@pytest.fixture(scope="module")
def ctx_default():
    c = {case: make_ctx(case) for case in ("tiny", "cfg0")}
    yield c
    for ctx, _ in c.values():
        ctx.close()


@pytest.mark.parametrize("case", ["tiny", "cfg0"])
def test_poses_vs_reference(ctx_default, case):
    ctx, types = ctx_default[case]
    P = poses(case)
    frames = [p["frame"] for p in P["poses"]]
    mol = ctx.molecules(types, n_systems=len(frames))
    pos, quat = frame_arrays(frames)
    mol.set_poses(pos, quat)
    f, t, st = mol.compute_forces()
    e = mol.compute_energy()
    for k in range(len(frames)):
        ref = oracle.parse(os.path.join(golden_dir(case), "ref_default", "pose%d.txt" % k))[0]
        assert st[k] == 0
        assert rel(f[k], ref["force"]) < TOL
        assert rel(t[k], ref["torque"]) < TOL
        assert abs(e[k] - ref["energy"]) <= TOL * abs(ref["energy"])
    mol.close()


@pytest.mark.parametrize("case", ["tiny", "cfg0"])
def test_sequence_state_carried_between_calls(ctx_default, case):
    ctx, types = ctx_default[case]
    P = poses(case)
    mol = ctx.molecules(types, n_systems=1)
    ref = oracle.parse(os.path.join(golden_dir(case), "ref_default", "sequence.txt"))
    for k, fr in enumerate(P["sequence"]):
        pos, quat = frame_arrays([fr])
        mol.set_poses(pos, quat)
        f, t, st = mol.compute_forces()
        assert rel(f[0], ref[k]["force"]) < TOL and rel(t[0], ref[k]["torque"]) < TOL
    mol.close()


def test_tight_tolerances_vs_reference():
    ctx, types = make_ctx("cfg0", tight=True)
    P = poses("cfg0")
    ks = [1, 3, 4, 6]
    mol = ctx.molecules(types, n_systems=len(ks))
    pos, quat = frame_arrays([P["poses"][k]["frame"] for k in ks])
    mol.set_poses(pos, quat)
    f, t, st = mol.compute_forces()
    for j, k in enumerate(ks):
        ref = oracle.parse(os.path.join(golden_dir("cfg0"), "ref_tight", "pose%d.txt" % k))[0]
        assert rel(f[j], ref["force"]) < TOL and rel(t[j], ref["torque"]) < TOL
    mol.close()
    ctx.close()


def test_batch_invariance(ctx_default):
    """A system's result does not depend on the other systems of its batch."""
    ctx, types = ctx_default["cfg0"]
    P = poses("cfg0")
    frames = [P["poses"][k]["frame"] for k in (2, 2, 4, 2)]
    mol = ctx.molecules(types, n_systems=4)
    pos, quat = frame_arrays(frames)
    mol.set_poses(pos, quat)
    f, t, _ = mol.compute_forces()
    assert np.array_equal(f[0], f[1]) and np.array_equal(f[0], f[3])
    single = ctx.molecules(types, n_systems=1)
    p1, q1 = frame_arrays([frames[2]])
    single.set_poses(p1, q1)
    f1, _, _ = single.compute_forces()
    assert np.array_equal(f1[0], f[2])
    mol.close()
    single.close()


def seeded_frames(case, n, seed, gaps=(0.5, 12.0)):
    from pbsam_b200 import synth
    d = golden_dir(case)
    A = synth.read_pqr(d + "/molA.pqr")
    B = synth.read_pqr(d + "/molB.pqr")
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        qa, qb, ax = synth.random_quat(rng), synth.random_quat(rng), synth.random_axis(rng)
        g = rng.uniform(*gaps)
        dist = synth.place_at_gap((A[0], A[1]), qa, (B[0], B[1]), qb, ax, g)
        out.append([dict(type=0, pos=[0.0, 0.0, 0.0], quat=list(qa)),
                    dict(type=1, pos=list(dist * ax), quat=list(qb))])
    return out


def oracle_forces(tmp_path, case, frames):
    P = poses(case)
    res = []
    for k, fr in enumerate(frames):
        spec, out = str(tmp_path / ("s%d.txt" % k)), str(tmp_path / ("o%d.txt" % k))
        oracle.write_spec(spec, oracle.golden_moltypes(golden_dir(case)), oracle.golden_frames(fr),
                          salt=P["salt"], idiel=P["idiel"], poles=P["poles"])
        res.append(oracle.run_spec(spec, out)[0])
    return res


@pytest.mark.parametrize("case,seed", [("tiny", 101), ("cfg0", 202)])
def test_seeded_poses_vs_oracle(ctx_default, tmp_path, case, seed):
    ctx, types = ctx_default[case]
    frames = seeded_frames(case, 4, seed)
    mol = ctx.molecules(types, n_systems=len(frames))
    pos, quat = frame_arrays(frames)
    mol.set_poses(pos, quat)
    f, t, st = mol.compute_forces()
    e = mol.compute_energy()
    ref = oracle_forces(tmp_path, case, frames)
    for k in range(len(frames)):
        assert st[k] == 0 and ref[k]["ok"]
        assert rel(f[k], ref[k]["force"]) < TOL and rel(t[k], ref[k]["torque"]) < TOL
        assert abs(e[k] - ref[k]["energy"]) <= TOL * abs(ref[k]["energy"])
    mol.close()


def test_singular_rotations_vs_oracle(ctx_default, tmp_path):
    """Identity orientations (molecule rotation with sin(theta) = 0) and a pair axis
    along z (pair rotation with sin(theta) < 1e-12) take the reference's singular branches."""
    from pbsam_b200 import synth
    ctx, types = ctx_default["tiny"]
    d = golden_dir("tiny")
    A = synth.read_pqr(d + "/molA.pqr")
    B = synth.read_pqr(d + "/molB.pqr")
    ca = A[0] - A[0].mean(axis=0)
    cb = B[0] - B[0].mean(axis=0)
    ident = [1.0, 0.0, 0.0, 0.0]
    flip = [0.0, 1.0, 0.0, 0.0]       # rotation by pi about x
    # B placed so that sphere 0 of B sits straight above sphere 0 of A, raised in
    # 0.5 A steps from a 3 A gap until no two spheres are closer than 1 A
    zoff = A[1][0] + B[1][0] + 3.0
    while True:
        posb = list(ca[0] - cb[0] + np.array([0.0, 0.0, zoff]))
        if synth.min_gap((A[0], A[1]), np.zeros(3), ident, (B[0], B[1]), np.array(posb), ident) > 1.0:
            break
        zoff += 0.5
    frames = [[dict(type=0, pos=[0, 0, 0], quat=ident), dict(type=1, pos=posb, quat=ident)]]
    frames.append([dict(type=0, pos=[0, 0, 0], quat=flip),
                   dict(type=1, pos=list(40.0 * np.array([0.0, 0.0, 1.0])), quat=ident)])
    mol = ctx.molecules(types, n_systems=len(frames))
    pos, quat = frame_arrays(frames)
    mol.set_poses(pos, quat)
    f, t, st = mol.compute_forces()
    ref = oracle_forces(tmp_path, "tiny", frames)
    for k in range(len(frames)):
        assert st[k] == 0 and ref[k]["ok"]
        assert rel(f[k], ref[k]["force"]) < TOL and rel(t[k], ref[k]["torque"]) < TOL
    mol.close()


def test_overlap_and_single_molecule(ctx_default):
    import pbsam_b200 as pb
    ctx, types = ctx_default["tiny"]
    P = poses("tiny")
    fr = P["poses"][0]["frame"]
    mol = ctx.molecules(types, n_systems=1)
    pos = np.array([[[0, 0, 0], [0.5, 0, 0]]], dtype=float)
    quat = np.array([[fr[0]["quat"], fr[1]["quat"]]])
    mol.set_poses(pos, quat)
    f, t, st = mol.compute_forces()
    assert st[0] == pb.PBSAM_SYS_OVERLAP and np.all(f == 0)
    mol.close()
    one = ctx.molecules([types[0]], n_systems=2)
    one.set_poses(np.zeros((2, 1, 3)), np.array([[[1.0, 0, 0, 0]], [[0.0, 1.0, 0, 0]]]))
    f, t, st = one.compute_forces()
    assert np.all(st == 0) and np.all(f == 0) and np.all(t == 0)
    one.close()


def test_cluster_sizes_agree():
    """The CTAs working on a system (1, 2, 4, 8, 16, or adaptive regrouping between
    calls) change only the rounding.  Three calls in a row on the same poses (each
    system keeps its state between calls, as the reference's molecules do, so the
    later calls differ from a fresh one): the first matches the reference, and every
    size agrees with one CTA per system, call by call, to 1e-12."""
    P = poses("cfg0")
    frames = [p["frame"] for p in P["poses"]]
    pos, quat = frame_arrays(frames)
    refs = [oracle.parse(os.path.join(golden_dir("cfg0"), "ref_default", "pose%d.txt" % k))[0]
            for k in range(len(frames))]
    results = {}
    for size in (1, 2, 4, 8, 16, -1):
        ctx, types = make_ctx("cfg0", cluster_size=size)
        mol = ctx.molecules(types, n_systems=len(frames))
        for call in range(3):      # adaptive: the first call is uniform, the next ones regrouped
            mol.set_poses(pos, quat)
            f, t, st = mol.compute_forces()
            assert np.all(st == 0)
            if call == 0:
                for k in range(len(frames)):
                    assert rel(f[k], refs[k]["force"]) < TOL and rel(t[k], refs[k]["torque"]) < TOL, (size, k)
            results.setdefault(size, []).append((f, t))
            if size > 0:
                assert np.all(mol.stats()[:, 5] == size)
        mol.close()
        ctx.close()
    for size, runs in results.items():
        for call, (f, t) in enumerate(runs):
            f1, t1 = results[1][call]
            for k in range(len(frames)):
                assert rel(f[k], f1[k]) < 1e-12 and rel(t[k], t1[k]) < 1e-12, (size, call, k)
