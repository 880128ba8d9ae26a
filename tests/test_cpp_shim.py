"""The C++ host layer (pb-sam_b200/cpp/pbsam_b200.hpp: CSystem / CMolecule with the
reference's names) through the reference harness's own spec and output format.

CPU: the harness compiles against the header and the library, and without a GPU
the set-up fails with exit status 3 instead of crashing.  GPU: the golden poses
and the state-carrying sequence of the p = 6 case equal the reference's outputs
within 1e-8 relative (forces, torques, energies), as through the Python mirror.
"""
import json
import os
import subprocess

import numpy as np
import pytest

import oracle
from conftest import REPO, golden_dir

SRC = os.path.join(REPO, "tests", "cpp", "shim_harness.cpp")
LIBDIR = os.path.join(REPO, "pb-sam_b200", "lib")


def build(tmp):
    exe = os.path.join(tmp, "shim_harness")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-o", exe, SRC, "-I", os.path.join(REPO, "include"),
                           "-I", os.path.join(REPO, "pb-sam_b200", "cpp"), "-L", LIBDIR, "-lpbsam_b200",
                           "-Wl,-rpath," + LIBDIR])
    return exe


def spec_for(tmp, frames, P, name):
    path = os.path.join(tmp, name)
    oracle.write_spec(path, oracle.golden_moltypes(golden_dir("tiny")), frames, salt=P["salt"], idiel=P["idiel"],
                      poles=P["poles"])
    return path


def rel(a, b):
    b = np.asarray(b)
    return float(np.max(np.abs(np.asarray(a) - b)) / max(np.max(np.abs(b)), 1e-300))


def test_builds_and_fails_cleanly_without_gpu(tmp_path):
    import torch
    if not os.path.exists(os.path.join(LIBDIR, "libpbsam_b200.so")):
        pytest.skip("CUDA library not built")
    exe = build(str(tmp_path))
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    P = json.load(open(os.path.join(golden_dir("tiny"), "poses.json")))
    spec = spec_for(str(tmp_path), oracle.golden_frames(P["poses"][0]["frame"]), P, "s.txt")
    r = subprocess.run([exe, spec, os.path.join(str(tmp_path), "o.txt")], capture_output=True, text=True)
    assert r.returncode == 3 and "pbsam-b200" in r.stderr


@pytest.mark.gpu
def test_golden_poses_and_sequence(tmp_path):
    exe = build(str(tmp_path))
    d = golden_dir("tiny")
    P = json.load(open(os.path.join(d, "poses.json")))
    for k, pose in enumerate(P["poses"]):
        spec = spec_for(str(tmp_path), oracle.golden_frames(pose["frame"]), P, "p%d.txt" % k)
        out = os.path.join(str(tmp_path), "p%d.out" % k)
        subprocess.check_call([exe, spec, out])
        g = oracle.parse(out)[0]
        ref = oracle.parse(os.path.join(d, "ref_default", "pose%d.txt" % k))[0]
        assert g["ok"] and ref["ok"]
        assert rel(g["force"], ref["force"]) < 1e-8 and rel(g["torque"], ref["torque"]) < 1e-8
        assert abs(g["energy"] - ref["energy"]) <= 1e-8 * abs(ref["energy"])
    frames = [[(m["type"], m["pos"], m["quat"]) for m in fr] for fr in P["sequence"]]
    spec = spec_for(str(tmp_path), frames, P, "seq.txt")
    out = os.path.join(str(tmp_path), "seq.out")
    subprocess.check_call([exe, spec, out])
    got = oracle.parse(out)
    ref = oracle.parse(os.path.join(d, "ref_default", "sequence.txt"))
    assert len(got) == len(ref)
    for g, r in zip(got, ref):
        assert rel(g["force"], r["force"]) < 1e-8 and rel(g["torque"], r["torque"]) < 1e-8


EXPAN_SRC = os.path.join(REPO, "tests", "cpp", "shim_expan.cpp")


def build_expan(tmp):
    exe = os.path.join(tmp, "shim_expan")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-o", exe, EXPAN_SRC, "-I", os.path.join(REPO, "include"),
                           "-I", os.path.join(REPO, "pb-sam_b200", "cpp"), "-L", LIBDIR, "-lpbsam_b200",
                           "-Wl,-rpath," + LIBDIR])
    return exe


def test_expansion_classes_build(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libpbsam_b200.so")):
        pytest.skip("CUDA library not built")
    assert os.path.exists(build_expan(str(tmp_path)))


@pytest.mark.gpu
def test_expansion_classes_vs_oracle(tmp_path):
    """CExpan / CRotCoeff / CTransCoeff / CXFormA / CGradExpan of the C++ layer, driven
    one operation at a time (and a rotateBatch), against the oracle's restatement of
    the reference's classes: 1e-12 relative; inprod against its formula."""
    exe = build_expan(str(tmp_path))
    NP = 10
    rng = np.random.default_rng(21)
    deg = np.floor(np.sqrt(np.arange(NP * NP)))

    def coeffs():
        return rng.standard_normal(NP * NP) * 0.6 ** deg

    def fmt(v):
        return " ".join("%.17g" % x for x in v)
    ops, lines = [], []
    # kappa of 0.05 M salt at eps 78, 298.15 K (src/BDnam_main.cpp:53-55)
    lines.append("init %d %.17g 78 298.15" % (NP, 0.07374))
    for th, ph, xi, p, wx, fw in [(0.7, 0.3, -1.2, NP, 0, 1), (2.1, -2.5, 0.4, 7, 1, 0), (0.0, 0.0, 0.9, NP, 0, 1),
                                  (np.pi, 0.0, 0.0, NP, 1, 1)]:
        x = coeffs()
        ops.append(("rotate", (th, ph, xi), p, wx, fw, x))
        lines.append("rotate %.17g %.17g %.17g %d %d %d %s" % (th, ph, xi, p, wx, fw, fmt(x)))
    for rho, scr, si, so, p, dv in [(18.0, 1, 4.0, 5.0, NP, 0), (11.5, 0, 3.2, 4.4, 8, 0), (25.0, 1, 5.5, 3.1, NP, 1)]:
        x = coeffs()
        ops.append(("translate", (rho, si, so), p, scr, dv, x))
        lines.append("translate %.17g %s %.17g %.17g %d %d %s" % (rho, "KAPPA" if scr else "0", si, so, p, dv, fmt(x)))
    for P, rs, rt, p, scr, gr in [((3.0, -9.0, 12.0), 4.2, 5.1, NP, 1, 1), ((-7.0, 2.0, -1.0), 3.3, 3.9, 6, 0, 0),
                                  ((0.0, 0.0, 14.0), 5.0, 3.5, NP, 1, 0)]:
        x = coeffs()
        ops.append(("xform", P + (rs, rt), p, scr, gr, x))
        lines.append("xform %.17g %.17g %.17g %.17g %.17g %d %d %d %s" % (P + (rs, rt, p, scr, gr, fmt(x))))
    brot = rng.uniform(0.2, 2.9, (5, 3))
    bx = [coeffs() for _ in range(5)]
    lines.append("batch 5")
    for a, x in zip(brot, bx):
        lines.append("%.17g %.17g %.17g %s" % (a[0], a[1], a[2], fmt(x)))
    M, L = coeffs(), coeffs()
    lines.append("inprod 0.25 4.0 %s %s" % (fmt(M), fmt(L)))
    # the screened translations use the context's own kappa (read back after init)
    spec = os.path.join(str(tmp_path), "ops.txt")
    out = os.path.join(str(tmp_path), "ops.out")
    with open(spec, "w") as fh:
        fh.write(lines[0] + "\n")
    subprocess.check_call([exe, spec, out])
    kappa = float(open(out).read().split()[1])
    with open(spec, "w") as fh:
        fh.write("\n".join(ln.replace("KAPPA", "%.17g" % kappa) for ln in lines) + "\n")
    subprocess.check_call([exe, spec, out])
    res = [ln.split() for ln in open(out)]
    assert res[0][0] == "kappa"
    k = 1
    for op in ops:
        name, args, p, f1, f2, x = op
        got = np.array([float(v) for v in res[k][2:]])
        k += 1
        if name == "rotate":
            ref = oracle.expan_op(NP, kappa, 0, np.array([args]), p, f1, f2, x[None])[0]
        elif name == "translate":
            ref = oracle.expan_op(NP, kappa, 1, np.array([args]), p, f1, f2, x[None])[0]
        else:
            if f1 and f2:
                ref, g = oracle.expan_op(NP, kappa, 2, np.array([args]), p, f1, 0, x[None], grad=True)
                ref, g = ref[0], g[0]
                gg = np.array([float(v) for v in res[k][1:]]).reshape(3, NP * NP)
                k += 1
                assert rel(gg, g) < 1e-11, rel(gg, g)
            else:
                ref = oracle.expan_op(NP, kappa, 2, np.array([args]), p, f1, 0, x[None])[0]
        assert rel(got, ref) < 1e-12, (name, args, rel(got, ref))
    bref = oracle.expan_op(NP, kappa, 0, brot, NP, 0, 1, np.array(bx))
    for i in range(5):
        got = np.array([float(v) for v in res[k][2:]])
        k += 1
        assert rel(got, bref[i]) < 1e-12
    n = np.floor(np.sqrt(np.arange(NP * NP))).astype(int)
    w = np.where(np.arange(NP * NP) == n * n, 1.0, 2.0)
    want = float(np.sum(w * M * L * (1.0 / (0.25 * 4.0)) ** n))
    assert res[k][0] == "inprod" and abs(float(res[k][1]) - want) <= 1e-13 * abs(want)
