"""Brownian dynamics through the C ABI (pbsam_system_bd_*) against the oracle.

The GPU steps (time step and force mask, the force kernel, the move kernel with
its rejection loops) and the oracle's restatement of CBDnam::run / makeMove and
CBDmulti::propagate / makeMove draw the same Philox noise, so each trajectory
is compared step by step: positions within 1e-9 A + 1e-9 relative, quaternion
components within 1e-9, statuses, step and force-evaluation counts exactly.
The forces inside a step agree to the 1e-8 relative bar of the force tests.
"""
import json
import os

import numpy as np
import pytest

import oracle
from conftest import golden_dir

pytestmark = pytest.mark.gpu
DTR = (0.0, 0.03)          # the reference's m_Dtr (src/BDnam.cpp:145), molecule 0 never translates
DROT = (4.5e-5, 4e-5)      # m_Dr1, m_Dr2


def tiny_ctx(cluster_size=0, **kw):
    import pbsam_b200 as pb
    P = json.load(open(os.path.join(golden_dir("tiny"), "poses.json")))
    ctx = pb.CSystem(poles=P["poles"], salt=P["salt"], idiel=P["idiel"], cluster_size=cluster_size, **kw)
    d = golden_dir("tiny")
    ta = ctx.load_moltype(d + "/molA.pqr", d + "/imA", d + "/expA", "molA.0")
    tb = ctx.load_moltype(d + "/molB.pqr", d + "/imB", d + "/expB", "molB.0")
    return ctx, [ta, tb], P


def oracle_traj(tmp_path, frame, mode, n, seed, system, dtr, drot, P, **kw):
    spec, out = os.path.join(tmp_path, "bd%d.txt" % system), os.path.join(tmp_path, "bd%d.out" % system)
    oracle.write_bd_spec(spec, oracle.golden_moltypes(golden_dir("tiny")), frame, mode, n, seed, system, dtr, drot,
                         salt=P["salt"], idiel=P["idiel"], poles=P["poles"], **kw)
    return oracle.run_bd_spec(spec, out)


def check_step(g, b, o):
    assert g["status"][b] == o["status"]
    assert g["steps"][b] == o["steps"]
    assert g["fevals"][b] == o["fevals"]
    assert abs(g["time"][b] - o["time"]) <= 1e-12 * abs(o["time"])
    np.testing.assert_allclose(g["pos"][b], o["pos"], rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(g["quat"][b], o["quat"], rtol=0, atol=1e-9)


def run_compare(tmp_path, mol_types, frame, mode, n, seed, dtr, drot, n_sys=2, use_graph=True, **kw):
    ctx, types, P = tiny_ctx()
    mol = ctx.molecules([types[t] for t in mol_types], n_systems=n_sys)
    pos = np.array([[m[1] for m in frame]] * n_sys)
    quat = np.array([[m[2] for m in frame]] * n_sys)
    mol.set_poses(pos, quat)
    mol.bd_init(dtr, drot, mode=mode, seed=seed, use_graph=use_graph, **kw)
    ref = [oracle_traj(str(tmp_path), frame, mode, n, seed, b, dtr, drot, P, **kw) for b in range(n_sys)]
    states = []
    for k in range(n):
        mol.bd_run(1)
        g = mol.bd_state()
        states.append(g)
        for b in range(n_sys):
            check_step(g, b, ref[b][k])
    mol.close()
    ctx.close()
    return states, ref


def gap5_frame():
    P = json.load(open(os.path.join(golden_dir("tiny"), "poses.json")))
    fr = P["poses"][1]["frame"]
    return [(m["type"], m["pos"], m["quat"]) for m in fr]


def test_nam_close_range_vs_oracle(tmp_path):
    states, ref = run_compare(tmp_path, [0, 1], gap5_frame(), 0, 8, 11, DTR, DROT)
    assert ref[0][-1]["fevals"] == 8          # every step evaluated forces (inside f_DIST)
    assert not np.allclose(states[-1]["pos"][0], states[-1]["pos"][1])


def test_nam_graph_and_stream_launches_agree(tmp_path):
    a, _ = run_compare(tmp_path, [0, 1], gap5_frame(), 0, 4, 5, DTR, DROT, use_graph=True)
    b, _ = run_compare(tmp_path, [0, 1], gap5_frame(), 0, 4, 5, DTR, DROT, use_graph=False)
    assert np.array_equal(a[-1]["pos"], b[-1]["pos"]) and np.array_equal(a[-1]["quat"], b[-1]["quat"])


def test_nam_crossing_force_distance_vs_oracle(tmp_path):
    # start just outside a small force distance: rotations are stored while far
    # and applied on the step that brings the pair back inside
    fr = gap5_frame()
    far = np.array(fr[1][1]) * 1.6
    frame = [fr[0], (fr[1][0], list(far), fr[1][2])]
    run_compare(tmp_path, [0, 1], frame, 0, 12, 3, (0.0, 2.0), (4.5e-3, 4e-3), force_dist=float(np.linalg.norm(far)) - 0.5)


def test_multi_three_molecules_vs_oracle(tmp_path):
    fr = gap5_frame()
    third = (0, list(-np.array(fr[1][1])), [0.5, 0.5, -0.5, 0.5])
    run_compare(tmp_path, [0, 1, 0], fr + [third], 1, 6, 9, (0.03, 0.03, 0.03), (4.5e-5, 4e-5, 4.5e-5))


def test_escape_and_stuck_vs_oracle(tmp_path):
    fr = gap5_frame()
    esc = [fr[0], (fr[1][0], [140.0, 0.0, 0.0], fr[1][2])]
    s, ref = run_compare(tmp_path, [0, 1], esc, 0, 60, 2, (0.0, 0.5), DROT, escape_dist=150.0)
    stuck = [fr[0], (fr[1][0], [0.3, 0.0, 0.0], fr[1][2])]
    s2, ref2 = run_compare(tmp_path, [0, 1], stuck, 0, 2, 2, (0.0, 1e-8), DROT, max_tries=1, force_dist=0.0)
    assert ref2[0][0]["status"] == 2 and s2[-1]["status"][0] == 2


def _ref_bd(tmp_path, frame, n, seed, P):
    """The reference's own CBDnam steps (oracle/ref_bd_harness.cpp) from srand48(seed)."""
    import subprocess
    exe = oracle.ref_bd_harness()
    if exe is None:
        pytest.skip("reference BD harness not built")
    spec = os.path.join(tmp_path, "r%d.txt" % seed)
    oracle.write_bd_spec(spec, oracle.golden_moltypes(golden_dir("tiny")), frame, 0, n, seed, 0, DTR, DROT,
                         salt=P["salt"], idiel=P["idiel"], poles=P["poles"])
    out = spec + ".out"
    subprocess.check_call([exe, spec, out], env=dict(os.environ, OMP_NUM_THREADS="1"),
                          stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    steps = []
    for ln in open(out):
        t = ln.split()
        if t[0] == "BDSTEP":
            steps.append(dict(status=int(t[2]), fevals=int(t[3]), time=float(t[4]), steps=int(t[1]), pos=[], quat=[]))
        elif t[0] == "POSE":
            v = [float(x) for x in t[2:]]
            steps[-1]["pos"].append(v[:3])
            steps[-1]["quat"].append(v[3:])
    return steps


@pytest.mark.parametrize("far", [False, True])
def test_reference_stream_vs_reference_bdnam(tmp_path, far):
    """With the reference's own noise stream (drand48, polar Box-Muller) system b
    repeats the reference's CBDnam run seeded with seed + b, step by step: at close
    range with forces every step, and across the force distance with stored
    rotations (CUDA's log and sqrt differ from the host's in the last bit)."""
    import pbsam_b200 as pb
    fr = gap5_frame()
    if far:
        axis = np.array(fr[1][1]) / np.linalg.norm(fr[1][1])
        fr = [fr[0], (fr[1][0], list(100.4 * axis), fr[1][2])]
    n, seed = (20, 777) if far else (8, 12345)
    ctx, types, P = tiny_ctx()
    mol = ctx.molecules(types, n_systems=2)
    mol.set_poses(np.array([[m[1] for m in fr]] * 2), np.array([[m[2] for m in fr]] * 2))
    mol.bd_init(DTR, DROT, mode=0, seed=seed, noise=pb.PBSAM_BD_NOISE_DRAND48)
    refs = [_ref_bd(str(tmp_path), fr, n, seed + b, P) for b in range(2)]
    for k in range(n):
        mol.bd_run(1)
        g = mol.bd_state()
        for b in range(2):
            check_step(g, b, dict(refs[b][k], pos=np.array(refs[b][k]["pos"]), quat=np.array(refs[b][k]["quat"])))
    mol.close()
    ctx.close()


@pytest.mark.parametrize("scale", [1.0, 9.0])
def test_reference_stream_vs_reference_bdm(tmp_path, scale):
    """Multi-molecule steps with the reference's noise stream against the reference's
    own CBDmulti (three molecules; close together, and all beyond the interaction
    cutoff, where the time step follows the smallest sphere gap)."""
    import subprocess
    import pbsam_b200 as pb
    exe = oracle.ref_bdm_harness()
    if exe is None:
        pytest.skip("reference BD harness not built")
    fr = gap5_frame()
    posb = np.array(fr[1][1]) * scale
    frame = [(0, [0.0, 0.0, 0.0], fr[0][2]), (0, list(-posb), [0.5, 0.5, -0.5, 0.5]), (1, list(posb), fr[1][2])]
    ctx, types, P = tiny_ctx()
    dtr, drot = (0.015, 0.015, 0.015), (4.5e-5, 4.5e-5, 4e-5)
    spec = os.path.join(str(tmp_path), "m.txt")
    oracle.write_bd_spec(spec, oracle.golden_moltypes(golden_dir("tiny")), frame, 1, 6, 4242, 0, dtr, drot,
                         salt=P["salt"], idiel=P["idiel"], poles=P["poles"], noise=(1, 1))
    out = spec + ".out"
    subprocess.check_call([exe, spec, out], env=dict(os.environ, OMP_NUM_THREADS="1"),
                          stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    ref = []
    for ln in open(out):
        t = ln.split()
        if t[0] == "BDSTEP":
            ref.append(dict(status=0, steps=int(t[1]), fevals=int(t[3]), time=float(t[4]), pos=[], quat=[]))
        elif t[0] == "POSE":
            v = [float(x) for x in t[2:]]
            ref[-1]["pos"].append(v[:3])
            ref[-1]["quat"].append(v[3:])
    mol = ctx.molecules([types[m[0]] for m in frame], n_systems=1)
    mol.set_poses(np.array([[m[1] for m in frame]]), np.array([[m[2] for m in frame]]))
    mol.bd_init(dtr, drot, mode=pb.PBSAM_BD_MULTI, seed=4242, noise=pb.PBSAM_BD_NOISE_DRAND48)
    for k in range(6):
        mol.bd_run(1)
        g = mol.bd_state()
        check_step(g, 0, dict(ref[k], pos=np.array(ref[k]["pos"]), quat=np.array(ref[k]["quat"])))
    mol.close()
    ctx.close()


def _contact_files(tmp_path, dist):
    """Every sphere pair of the two tiny molecules, one contact needed: a contactdef
    file for readMolContact (distance from the command line) and the same with a
    distance on every pair line (readMolContactWithDist)."""
    na = sum(1 for ln in open(os.path.join(golden_dir("tiny"), "molA.pqr")) if "CEN" in ln)
    nb = sum(1 for ln in open(os.path.join(golden_dir("tiny"), "molB.pqr")) if "CEN" in ln)
    pairs = [(i, j) for i in range(na) for j in range(nb)]
    f1, f2 = os.path.join(tmp_path, "contact.dat"), os.path.join(tmp_path, "contact_dist.dat")
    with open(f1, "w") as fh:
        fh.write("0 1\n1 1 %d\n" % len(pairs) + "".join("%d %d\n" % pr for pr in pairs))
    with open(f2, "w") as fh:
        fh.write("0 1\n1 1 %d\n" % len(pairs) + "".join("%d %d %r\n" % (pr + (dist,)) for pr in pairs))
    return f1, f2, pairs


def test_docking_vs_reference_bdnam(tmp_path):
    """NAM docking (CMolContact::readMolContact, CBDnam::IsDocked): the reference's own
    CBDnam with a contact file (every sphere pair, one contact within 5.5 A) docks at
    step 30 of this run; the CUDA path with the reference's noise stream repeats every
    step and docks at the same step.  The same definitions read with per-pair distances
    and given as arrays agree; without them the trajectory keeps running."""
    import subprocess
    import pbsam_b200 as pb
    exe = oracle.ref_bd_harness()
    if exe is None:
        pytest.skip("reference BD harness not built")
    dist, seed, n = 5.5, 12345, 34
    f1, f2, pairs = _contact_files(str(tmp_path), dist)
    fr = gap5_frame()
    ctx, types, P = tiny_ctx()
    spec = os.path.join(str(tmp_path), "dock.txt")
    oracle.write_bd_spec(spec, oracle.golden_moltypes(golden_dir("tiny")), fr, 0, n, seed, 0, DTR, DROT,
                         salt=P["salt"], idiel=P["idiel"], poles=P["poles"])
    with open(spec, "a") as fh:
        fh.write("contact %s %r\n" % (f1, dist))
    subprocess.check_call([exe, spec, spec + ".out"], env=dict(os.environ, OMP_NUM_THREADS="1"),
                          stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    ref = []
    for ln in open(spec + ".out"):
        t = ln.split()
        if t[0] == "BDSTEP":
            ref.append(dict(status=int(t[2]), fevals=int(t[3]), time=float(t[4]), steps=int(t[1]), pos=[], quat=[]))
        elif t[0] == "POSE":
            v = [float(x) for x in t[2:]]
            ref[-1]["pos"].append(v[:3])
            ref[-1]["quat"].append(v[3:])
    assert ref[-1]["status"] == pb.PBSAM_BD_DOCKED and 10 < len(ref) < n, (len(ref), ref[-1]["status"])
    mols = []
    try:
        for how in ("file", "file_dist", "arrays", "none"):
            m = ctx.molecules(types, n_systems=1)
            mols.append(m)
            m.set_poses(np.array([[x[1] for x in fr]]), np.array([[x[2] for x in fr]]))
            m.bd_init(DTR, DROT, mode=0, seed=seed, noise=pb.PBSAM_BD_NOISE_DRAND48)
            if how == "file":
                m.bd_set_contacts_file(f1, dist)
            elif how == "file_dist":
                m.bd_set_contacts_file(f2, 0.0)
            elif how == "arrays":
                m.bd_set_contacts([(1, 1, [(i, j, dist) for i, j in pairs])])
            for k in range(len(ref)):
                m.bd_run(1)
                g = m.bd_state()
                r = dict(ref[k], pos=np.array(ref[k]["pos"]), quat=np.array(ref[k]["quat"]))
                if how == "none" and k == len(ref) - 1:
                    r["status"] = pb.PBSAM_BD_RUNNING
                check_step(g, 0, r)
            m.bd_run(2)                     # a docked trajectory stays as it is
            g = m.bd_state()
            if how != "none":
                assert g["status"][0] == pb.PBSAM_BD_DOCKED and g["steps"][0] == len(ref)
        # a contact naming a sphere the molecule does not have is refused
        with pytest.raises(pb.PbsamError):
            mols[0].bd_set_contacts([(1, 1, [(99, 0, dist)])])
    finally:
        for m in mols:
            m.close()
        ctx.close()
