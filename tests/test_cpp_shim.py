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
