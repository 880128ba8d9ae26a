"""The oracle's Brownian-dynamics restatement (CBDnam / CBDmulti steps) on CPU.

* its Philox4x64-10 blocks equal numpy's independent implementation
  (numpy.random.Philox advances its counter before each block);
* free diffusion beyond the force distance: per-step displacements are
  N(0, 2 D dt) per component with the reference's time step 2 + (d - 5)/15 ps,
  and no force evaluation is made (src/BDnam.cpp:196-222, 409-417);
* escape beyond q_DIST ends the trajectory (src/BDnam.cpp:288);
* a trajectory whose every move is rejected is STUCK (src/BDnam.cpp:287);
* drawing the reference's own stream (drand48 from srand48(seed), polar
  Box-Muller, the vector's deviates drawn z first as gcc evaluates
  CPnt(normRand(), normRand(), normRand())), the oracle's steps equal the
  reference's own CBDnam::makeMove loop (oracle/ref_bd_harness.cpp, one OpenMP
  thread: the reference's threaded force path races) bit for bit, at close range
  and across the force distance with stored rotations; and the multi-molecule
  steps equal the reference's own CBDmulti (oracle/ref_bdm_harness.cpp) with three
  molecules, close together and all farther apart than the interaction cutoff.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle
from conftest import golden_dir


def test_philox_matches_numpy():
    for ctr, key in (([1, 0, 0, 0], [0, 0]), ([5, 7, 9, 11], [123, 456]), ([2**64 - 1, 3, 0, 1], [2**63, 17])):
        g = np.random.Philox(counter=np.array([(ctr[0] - 1) % 2**64] + ctr[1:], dtype=np.uint64),
                             key=np.array(key, dtype=np.uint64))
        assert [int(x) for x in g.random_raw(4)] == oracle.philox(ctr, key)


def _frame(p1, q1=(1, 0, 0, 0)):
    return [(0, [0.0, 0.0, 0.0], [1.0, 0.0, 0.0, 0.0]), (1, list(p1), list(q1))]


def _run(tmp_path, frame, n, mode=0, seed=7, system=0, dtr=(0.0, 0.03), drot=(4.5e-5, 4e-5), **kw):
    case = golden_dir("tiny")
    spec, out = os.path.join(tmp_path, "bd.txt"), os.path.join(tmp_path, "bd.out")
    oracle.write_bd_spec(spec, oracle.golden_moltypes(case), frame, mode, n, seed, system, dtr, drot,
                         salt=0.1, idiel=4.0, poles=6, **kw)
    return oracle.run_bd_spec(spec, out)


def test_free_diffusion_statistics(tmp_path):
    n = 3000
    steps = _run(str(tmp_path), _frame((300.0, 0.0, 0.0)), n, escape_dist=1e9)
    pos = np.array([s["pos"][1] for s in steps])
    assert all(s["fevals"] == 0 and s["status"] == 0 for s in steps)
    prev = np.vstack([[300.0, 0.0, 0.0], pos[:-1]])
    d = pos - prev
    t = np.array([s["time"] for s in steps])
    dt = np.diff(np.concatenate([[0.0], t]))
    assert np.all(dt > 2.0)
    z = d / np.sqrt(2 * 0.03 * dt)[:, None]
    assert abs(z.mean()) < 4 / np.sqrt(z.size)
    assert abs(z.var() - 1.0) < 0.06
    # the time step follows the gap before the move: 2 + (gap - 5)/15
    gap0 = 300.0 - (dt[0] - 2.0) * 15 - 5
    c2c = np.linalg.norm(prev, axis=1)
    np.testing.assert_allclose(dt, 2.0 + (c2c - gap0 - 5) / 15, rtol=1e-12)


def test_escape(tmp_path):
    steps = _run(str(tmp_path), _frame((140.0, 0.0, 0.0)), 400, escape_dist=150.0, dtr=(0.0, 0.5))
    st = [s["status"] for s in steps]
    assert 1 in st, "no escape"
    k = st.index(1)
    assert all(x == 1 for x in st[k:])
    assert np.linalg.norm(steps[k]["pos"][1]) > 150.0
    assert steps[-1]["steps"] == k + 1      # nothing moves after the escape


def test_stuck_when_every_move_collides(tmp_path):
    # molecule 1 placed on top of molecule 0: with one draw per move and a tiny
    # diffusion constant every candidate position still overlaps
    steps = _run(str(tmp_path), _frame((0.3, 0.0, 0.0)), 3, max_tries=1, dtr=(0.0, 1e-8), force_dist=0.0)
    assert steps[0]["status"] == 2 and steps[-1]["steps"] == 1


@pytest.mark.parametrize("mode", [0, 1])
def test_same_seed_same_trajectory_other_system_differs(tmp_path, mode):
    fr = _frame((60.0, 10.0, -5.0))
    a = _run(str(tmp_path), fr, 5, mode=mode, system=0, force_dist=0.0, dtr=(0.03, 0.03))
    b = _run(str(tmp_path), fr, 5, mode=mode, system=0, force_dist=0.0, dtr=(0.03, 0.03))
    c = _run(str(tmp_path), fr, 5, mode=mode, system=1, force_dist=0.0, dtr=(0.03, 0.03))
    assert np.array_equal(a[-1]["pos"], b[-1]["pos"]) and np.array_equal(a[-1]["quat"], b[-1]["quat"])
    assert not np.allclose(a[-1]["pos"], c[-1]["pos"])
    if mode == 0:
        assert np.array_equal(a[-1]["pos"][0], [0, 0, 0])   # NAM: molecule 0 never translates


def _ref_steps(path, n_mol=2):
    steps = []
    for ln in open(path):
        t = ln.split()
        if t[0] == "BDSTEP":
            steps.append(dict(status=int(t[2]), fevals=int(t[3]), time=float(t[4]), pos={}, quat={}))
        elif t[0] == "POSE":
            v = [float(x) for x in t[2:]]
            steps[-1]["pos"][int(t[1])] = v[:3]
            steps[-1]["quat"][int(t[1])] = v[3:]
    for st in steps:
        st["pos"] = np.array([st["pos"][i] for i in range(n_mol)])
        st["quat"] = np.array([st["quat"][i] for i in range(n_mol)])
    return steps


def _vs_reference(tmp_path, frame, n, seed):
    exe = oracle.ref_bd_harness()
    if exe is None:
        pytest.skip("reference BD harness not built (oracle/build_ref.py)")
    case = golden_dir("tiny")
    spec = os.path.join(tmp_path, "ref.txt")
    oracle.write_bd_spec(spec, oracle.golden_moltypes(case), frame, 0, n, seed, 0, (0.0, 0.03), (4.5e-5, 4e-5),
                         salt=0.1, idiel=4.0, poles=6, noise=(1, 1))
    out = os.path.join(tmp_path, "ref.out")
    r = subprocess.run([exe, spec, out], env=dict(os.environ, OMP_NUM_THREADS="1"), capture_output=True)
    mine = oracle.run_bd_spec(spec, os.path.join(tmp_path, "orc.out"))
    return r.returncode, (_ref_steps(out) if r.returncode == 0 else []), mine


def _gap5_frame():
    import json
    P = json.load(open(os.path.join(golden_dir("tiny"), "poses.json")))
    return [(m["type"], m["pos"], m["quat"]) for m in P["poses"][1]["frame"]]


def test_reference_stream_matches_reference_bdnam_close_range(tmp_path):
    rc, ref, mine = _vs_reference(str(tmp_path), _gap5_frame(), 8, 12345)
    assert rc == 0 and len(ref) == len(mine) == 8
    for a, b in zip(mine, ref):
        assert a["status"] == b["status"] and a["fevals"] == b["fevals"] and a["time"] == b["time"]
        assert np.array_equal(a["pos"], b["pos"]) and np.array_equal(a["quat"], b["quat"])
    assert ref[-1]["fevals"] == 8


def test_reference_stream_matches_reference_bdnam_across_force_distance(tmp_path):
    fr = _gap5_frame()
    axis = np.array(fr[1][1]) / np.linalg.norm(fr[1][1])
    frame = [fr[0], (fr[1][0], list(100.4 * axis), fr[1][2])]
    rc, ref, mine = _vs_reference(str(tmp_path), frame, 30, 777)
    assert rc == 0 and len(ref) == len(mine) == 30
    for a, b in zip(mine, ref):
        assert a["status"] == b["status"] and a["fevals"] == b["fevals"]
        assert np.array_equal(a["pos"], b["pos"]) and np.array_equal(a["quat"], b["quat"])
    assert 0 < ref[-1]["fevals"] < 30          # steps with and without forces, stored rotations applied


def test_overlap_ends_the_trajectory_on_both_sides(tmp_path):
    fr = _gap5_frame()
    rc, ref, mine = _vs_reference(str(tmp_path), [fr[0], (fr[1][0], [0.3, 0.0, 0.0], fr[1][2])], 3, 5)
    assert rc == 4 and mine[0]["status"] == 4     # bdnam exits; the oracle reports FAILED


def _multi_frame(scale):
    fr = _gap5_frame()
    posb = np.array(fr[1][1]) * scale
    return [(0, [0.0, 0.0, 0.0], fr[0][2]), (0, list(-posb), [0.5, 0.5, -0.5, 0.5]), (1, list(posb), fr[1][2])]


@pytest.mark.parametrize("scale", [1.0, 9.0])
def test_reference_stream_matches_reference_bdm(tmp_path, scale):
    exe = oracle.ref_bdm_harness()
    if exe is None:
        pytest.skip("reference BD harness not built (oracle/build_ref.py)")
    spec = os.path.join(str(tmp_path), "m.txt")
    # the reference's bdm constants (src/BDmulti.cpp:204-205): D 0.015 for both species,
    # Dr 4.5e-5 (species 0) and 4e-5 (species 1); species 0 copies first
    oracle.write_bd_spec(spec, oracle.golden_moltypes(golden_dir("tiny")), _multi_frame(scale), 1, 6, 4242, 0,
                         (0.015, 0.015, 0.015), (4.5e-5, 4.5e-5, 4e-5), salt=0.1, idiel=4.0, poles=6,
                         noise=(1, 1))
    out = os.path.join(str(tmp_path), "m.out")
    subprocess.check_call([exe, spec, out], env=dict(os.environ, OMP_NUM_THREADS="1"))
    ref = _ref_steps(out, 3)
    mine = oracle.run_bd_spec(spec, os.path.join(str(tmp_path), "mo.out"))
    assert len(ref) == len(mine) == 6
    for a, b in zip(mine, ref):
        assert a["fevals"] == b["fevals"] and a["time"] == b["time"]
        assert np.array_equal(a["pos"], b["pos"]) and np.array_equal(a["quat"], b["quat"])
    assert (ref[-1]["fevals"] == 6) if scale == 1.0 else (ref[-1]["fevals"] == 0)


def test_reference_stream_matches_reference_bdnam_p10(tmp_path):
    """The same at pole order 10 on the 8-sphere molecules (reference `default` build
    at N_POLES 10), 4 A gap, forces every step."""
    import json
    exe = oracle.ref_bd_harness(10, "default")
    if exe is None:
        pytest.skip("reference BD harness not built (oracle/build_ref.py)")
    d = golden_dir("cfg0")
    P = json.load(open(os.path.join(d, "poses.json")))
    frame = [(m["type"], m["pos"], m["quat"]) for m in P["poses"][2]["frame"]]
    spec = os.path.join(str(tmp_path), "c.txt")
    oracle.write_bd_spec(spec, oracle.golden_moltypes(d), frame, 0, 5, 99, 0, (0.0, 0.03), (4.5e-5, 4e-5),
                         salt=P["salt"], idiel=P["idiel"], poles=P["poles"], noise=(1, 1))
    out = os.path.join(str(tmp_path), "c.out")
    subprocess.check_call([exe, spec, out], env=dict(os.environ, OMP_NUM_THREADS="1"), stdout=subprocess.DEVNULL)
    ref = _ref_steps(out)
    mine = oracle.run_bd_spec(spec, os.path.join(str(tmp_path), "co.out"))
    assert len(ref) == len(mine) == 5 and ref[-1]["fevals"] == 5
    for a, b in zip(mine, ref):
        assert np.array_equal(a["pos"], b["pos"]) and np.array_equal(a["quat"], b["quat"])
