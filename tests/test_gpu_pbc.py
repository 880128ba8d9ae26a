"""The periodic box (pbsam_params.box_length) against the reference with its box on.

bdm runs the reference with CSystem::initConstants(kappa, sdiel, T, true, L)
(src/BDmulti_main.cpp:67).  CMolecule::setPos and translate wrap the molecule centres
into the box (src/molecule.h:325-327); the pair lists, the polarization
re-expansions, reexpandGrad, the collision tests and the BD distances take the
minimum image of each displacement (CSystem::pbcPos, src/system.cpp:46-55), while
prepareDTA (src/molecule.cpp:1515-1619) and the energy (src/molecule.cpp:1873) take
the plain difference of the wrapped centres.  The plain drop-in reproduces that; the
lab-frame energy takes the minimum image everywhere.  Against the reference's own
harnesses with a `box` entry:
  * forces, torques and energy of a pose whose molecules meet only across a face of
    the box (1e-8 relative); the lab-frame energy equal to that of the same pose
    unwrapped without a box;
  * multi-molecule BD steps with the reference's noise stream against CBDmulti,
    molecules straddling the box faces, one carried through a face (positions 1e-9 A).
"""
import json
import os
import subprocess

import numpy as np
import pytest

import oracle
from conftest import golden_dir
from test_gpu_bd import check_step, gap5_frame, tiny_ctx
from test_gpu_parity import rel

pytestmark = pytest.mark.gpu
L = 70.0


def _ref_forces(tmp, P, frame, box):
    exe = os.path.join(oracle.HERE, "_ref", "p%d_default" % P["poles"], "harness")
    if not os.path.exists(exe):
        pytest.skip("reference build missing (oracle/build_ref.py)")
    spec = os.path.join(tmp, "f.txt")
    with open(spec, "w") as fh:
        fh.write("salt %r\nidiel %r\ndump 0\nenergy 1\nbox %r\n" % (P["salt"], P["idiel"], box))
        for mt in oracle.golden_moltypes(golden_dir("tiny")):
            fh.write("moltype %s %s %s %s\n" % mt)
        fh.write("frame\n")
        for t, p, q in frame:
            fh.write("mol %d %s %s\n" % (t, " ".join("%.17g" % v for v in p), " ".join("%.17g" % v for v in q)))
    subprocess.run([exe, spec, spec + ".out"], check=True, env=dict(os.environ, OMP_NUM_THREADS="1"),
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    return oracle.parse(spec + ".out")[0]


def test_pbc_forces_across_the_box_face(tmp_path):
    import pbsam_b200 as pb
    P = json.load(open(os.path.join(golden_dir("tiny"), "poses.json")))
    fr = P["poses"][0]["frame"]
    pa, pb_ = np.array(fr[0]["pos"]), np.array(fr[1]["pos"])
    # A 2 A inside the -x face; B (5 A further in -x) lies beyond it and is wrapped to the
    # +x side: the two meet only across the face
    shift = np.array([-L / 2 + 2.0, 0.0, 0.0]) - pa
    a = pa + shift
    b = pb_ + shift
    assert b[0] < -L / 2
    frame = [(0, list(a), fr[0]["quat"]), (1, list(b), fr[1]["quat"])]
    ref = _ref_forces(str(tmp_path), P, frame, L)
    assert ref["ok"]
    ctx = pb.CSystem(poles=P["poles"], salt=P["salt"], idiel=P["idiel"], box_length=L)
    plain = pb.CSystem(poles=P["poles"], salt=P["salt"], idiel=P["idiel"])
    try:
        d = golden_dir("tiny")
        types = [ctx.load_moltype(d + "/mol%s.pqr" % t, d + "/im" + t, d + "/exp" + t, "mol%s.0" % t) for t in "AB"]
        ptypes = [plain.load_moltype(d + "/mol%s.pqr" % t, d + "/im" + t, d + "/exp" + t, "mol%s.0" % t) for t in "AB"]
        m = ctx.molecules(types, 1)
        m.set_poses(np.array([[a, b]]), np.array([[fr[0]["quat"], fr[1]["quat"]]]))
        f, t, st = m.compute_forces()
        e = m.compute_energy()
        assert st[0] == 0 and m.stats()[0, 2] > 0, "the pose must polarize across the face"
        assert rel(f[0], ref["force"]) < 1e-8 and rel(t[0], ref["torque"]) < 1e-8, (rel(f[0], ref["force"]),)
        # the energy takes the plain difference of the wrapped centres (B wrapped as
        # setPos does, 65 A from A) where the forces see the 17 A minimum image
        assert abs(e[0] - ref["energy"]) <= 1e-8 * abs(ref["energy"]), (e[0], ref["energy"])
        # the same geometry unwrapped, without a box: the polarization is the same, so
        # the lab-frame energy (minimum image) is too
        mp = plain.molecules(ptypes, 1)
        mp.set_poses(np.array([[pa, pb_]]), np.array([[fr[0]["quat"], fr[1]["quat"]]]))
        f2, t2, st2 = mp.compute_forces()
        assert st2[0] == 0
        el, el2 = m.compute_energy(lab=True), mp.compute_energy(lab=True)
        assert abs(el[0] - el2[0]) <= 1e-9 * abs(el2[0]), (el[0], el2[0])
        m.close()
        mp.close()
    finally:
        ctx.close()
        plain.close()


def test_pbc_bdm_vs_reference(tmp_path):
    """Three molecules straddling the faces of the box, the reference's noise stream:
    six CBDmulti steps, one of which carries a molecule through a face (moves wrap
    into the box)."""
    import pbsam_b200 as pb
    exe = oracle.ref_bdm_harness()
    if exe is None:
        pytest.skip("reference BD harness not built")
    fr = gap5_frame()
    posb = np.array(fr[1][1])
    a = np.array([-L / 2 + 0.02, 1.0, 0.0])
    # A on the -x face (it wraps to the +x side in the second step) with B beside it; C near
    # the +x face, nearest to A through the face.  CBDmulti holds the copies of species 0
    # first (src/BDmulti.cpp constructor), so C (species 0) comes before B.
    frame = [(0, list(a), fr[0][2]), (0, [L / 2 - 20.0, -3.0, 2.0], [0.5, 0.5, -0.5, 0.5]),
             (1, list(a + posb), fr[1][2])]
    ctx, types, P = tiny_ctx(box_length=L)
    dtr, drot = (0.015, 0.015, 0.015), (4.5e-5, 4.5e-5, 4e-5)
    spec = os.path.join(str(tmp_path), "m.txt")
    oracle.write_bd_spec(spec, oracle.golden_moltypes(golden_dir("tiny")), frame, 1, 6, 777, 0, dtr, drot,
                         salt=P["salt"], idiel=P["idiel"], poles=P["poles"], noise=(1, 1))
    with open(spec, "a") as fh:
        fh.write("box %r\n" % L)
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
    assert len(ref) == 6 and ref[-1]["fevals"] > 0
    assert ref[0]["pos"][0][0] < 0 < ref[-1]["pos"][0][0], "A must wrap through the -x face"
    mol = ctx.molecules([types[m[0]] for m in frame], n_systems=1)
    mol.set_poses(np.array([[m[1] for m in frame]]), np.array([[m[2] for m in frame]]))
    mol.bd_init(dtr, drot, mode=pb.PBSAM_BD_MULTI, seed=777, noise=pb.PBSAM_BD_NOISE_DRAND48)
    for k in range(6):
        mol.bd_run(1)
        g = mol.bd_state()
        check_step(g, 0, dict(ref[k], pos=np.array(ref[k]["pos"]), quat=np.array(ref[k]["quat"])))
    assert np.all(np.abs(g["pos"]) <= L / 2 + 1e-9)
    mol.close()
    ctx.close()


def _lattice64():
    """64 molecules (32 copies of each golden p = 6 molecule, species 0 first as
    CBDmulti holds them) on a 4 x 4 x 4 lattice of 24 A, jittered and randomly
    turned, in a periodic box of 96 A: minimum gap 4 A, 115 molecule pairs inside the
    polarization cutoff, many of them across a face."""
    from pbsam_b200 import synth
    rng = np.random.default_rng(64)
    quat = np.array([synth.random_quat(rng) for _ in range(64)])
    jit = rng.uniform(-1.5, 1.5, (64, 3))
    perm = rng.permutation(64)
    grid = np.array([[x, y, z] for x in range(4) for y in range(4) for z in range(4)], float)
    s, box = 24.0, 96.0
    pos = grid[perm] * s + jit - box / 2 + s / 2
    types = [0] * 32 + [1] * 32
    return types, pos, quat, box


def test_pbc_64_molecules_vs_reference(tmp_path):
    """A 64-molecule periodic system (the molecule count of the reference's periodic bdm
    example): forces, torques and energy of one evaluation against the reference's
    (1e-8 relative)."""
    import pbsam_b200 as pb
    P = json.load(open(os.path.join(golden_dir("tiny"), "poses.json")))
    types, pos, quat, box = _lattice64()
    ref = _ref_forces(str(tmp_path), P, list(zip(types, pos.tolist(), quat.tolist())), box)
    assert ref["ok"]
    ctx = pb.CSystem(poles=P["poles"], salt=P["salt"], idiel=P["idiel"], box_length=box)
    try:
        d = golden_dir("tiny")
        ts = [ctx.load_moltype(d + "/mol%s.pqr" % t, d + "/im" + t, d + "/exp" + t, "mol%s.0" % t) for t in "AB"]
        m = ctx.molecules([ts[t] for t in types], 1)
        m.set_poses(pos[None], quat[None])
        f, t, st = m.compute_forces()
        e = m.compute_energy()
        assert st[0] == 0 and m.stats()[0, 2] > 0
        ef, et = rel(f[0], ref["force"]), rel(t[0], ref["torque"])
        print("64 molecules: force %.2e torque %.2e energy %.2e" % (ef, et, abs(e[0] - ref["energy"]) / abs(ref["energy"])))
        assert ef < 1e-8 and et < 1e-8 and abs(e[0] - ref["energy"]) <= 1e-8 * abs(ref["energy"])
        m.close()
    finally:
        ctx.close()


def test_pbc_bdm_64_molecules_vs_reference(tmp_path):
    """Three CBDmulti steps of the 64-molecule periodic system with the reference's
    noise stream against the reference's own bdm (positions 1e-9 A)."""
    import pbsam_b200 as pb
    exe = oracle.ref_bdm_harness()
    if exe is None:
        pytest.skip("reference BD harness not built")
    types, pos, quat, box = _lattice64()
    frame = list(zip(types, pos.tolist(), quat.tolist()))
    ctx, ts, P = tiny_ctx(box_length=box)
    # CBDmulti's per-species coefficients (src/BDmulti.cpp:204-205)
    dtr, drot = tuple([0.015] * 64), tuple([4.5e-5] * 32 + [4e-5] * 32)
    spec = os.path.join(str(tmp_path), "m64.txt")
    oracle.write_bd_spec(spec, oracle.golden_moltypes(golden_dir("tiny")), frame, 1, 3, 2024, 0, dtr, drot,
                         salt=P["salt"], idiel=P["idiel"], poles=P["poles"], noise=(1, 1))
    with open(spec, "a") as fh:
        fh.write("box %r\n" % box)
    subprocess.check_call([exe, spec, spec + ".out"], env=dict(os.environ, OMP_NUM_THREADS="1"),
                          stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    ref = []
    for ln in open(spec + ".out"):
        t = ln.split()
        if t[0] == "BDSTEP":
            ref.append(dict(status=0, steps=int(t[1]), fevals=int(t[3]), time=float(t[4]), pos=[], quat=[]))
        elif t[0] == "POSE":
            v = [float(x) for x in t[2:]]
            ref[-1]["pos"].append(v[:3])
            ref[-1]["quat"].append(v[3:])
    assert len(ref) == 3 and ref[-1]["fevals"] > 0
    mol = ctx.molecules([ts[t] for t in types], n_systems=1)
    try:
        mol.set_poses(pos[None], quat[None])
        mol.bd_init(dtr, drot, mode=pb.PBSAM_BD_MULTI, seed=2024, noise=pb.PBSAM_BD_NOISE_DRAND48)
        for k in range(3):
            mol.bd_run(1)
            g = mol.bd_state()
            check_step(g, 0, dict(ref[k], pos=np.array(ref[k]["pos"]), quat=np.array(ref[k]["quat"])))
    finally:
        mol.close()
        ctx.close()
