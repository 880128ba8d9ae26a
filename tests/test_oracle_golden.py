"""The CPU oracle (oracle/pbsam_oracle.cpp) against the reference's own outputs.

The golden files under tests/golden/<case>/ref_{default,tight}/ were written by
the reference PB-SAM (force harness oracle/ref_harness.cpp over the reference
classes, script tests/golden/make_golden.py).  The oracle must reproduce them to
1e-11 relative (they agree to ~1e-14; the slack covers libm differences).
"""
import json
import os

import numpy as np
import pytest

import oracle
from conftest import golden_dir

TOL = 1e-11


def rel(a, b):
    b = np.asarray(b)
    return float(np.max(np.abs(np.asarray(a) - b)) / max(np.max(np.abs(b)), 1e-300))


def run_case(tmp_path, case, mode, frames, poses_file):
    d = golden_dir(case)
    P = json.load(open(os.path.join(d, "poses.json")))
    tol = oracle.DEFAULT_TOL if mode == "default" else oracle.TIGHT_TOL
    spec = str(tmp_path / "spec.txt")
    out = str(tmp_path / "out.txt")
    oracle.write_spec(spec, oracle.golden_moltypes(d), frames, salt=P["salt"], idiel=P["idiel"],
                      poles=P["poles"], tol=tol)
    got = oracle.run_spec(spec, out)
    ref = oracle.parse(os.path.join(d, "ref_" + mode, poses_file))
    assert len(got) == len(ref)
    for g, r in zip(got, ref):
        assert g["ok"] == r["ok"]
        if not r["ok"]:
            continue
        assert rel(g["force"], r["force"]) < TOL
        assert rel(g["torque"], r["torque"]) < TOL
        assert abs(g["energy"] - r["energy"]) <= TOL * abs(r["energy"])


def _poses(case):
    return json.load(open(os.path.join(golden_dir(case), "poses.json")))


@pytest.mark.parametrize("mode", ["default", "tight"])
@pytest.mark.parametrize("k", range(3))
def test_tiny_poses(tmp_path, mode, k):
    P = _poses("tiny")
    run_case(tmp_path, "tiny", mode, oracle.golden_frames(P["poses"][k]["frame"]), "pose%d.txt" % k)


@pytest.mark.parametrize("mode", ["default", "tight"])
def test_tiny_sequence(tmp_path, mode):
    P = _poses("tiny")
    frames = [[(m["type"], m["pos"], m["quat"]) for m in fr] for fr in P["sequence"]]
    run_case(tmp_path, "tiny", mode, frames, "sequence.txt")


@pytest.mark.parametrize("k", range(7))
def test_cfg0_default(tmp_path, k):
    P = _poses("cfg0")
    run_case(tmp_path, "cfg0", "default", oracle.golden_frames(P["poses"][k]["frame"]), "pose%d.txt" % k)


@pytest.mark.parametrize("k", [3, 4, 5, 6])
def test_cfg0_tight(tmp_path, k):
    P = _poses("cfg0")
    run_case(tmp_path, "cfg0", "tight", oracle.golden_frames(P["poses"][k]["frame"]), "pose%d.txt" % k)


def test_cfg0_sequence(tmp_path):
    P = _poses("cfg0")
    frames = [[(m["type"], m["pos"], m["quat"]) for m in fr] for fr in P["sequence"]]
    run_case(tmp_path, "cfg0", "default", frames, "sequence.txt")


def test_overlap_reported(tmp_path):
    """Overlapping molecules: computeForces returns false (src/molecule.cpp:1090-1097)."""
    P = _poses("tiny")
    fr = P["poses"][0]["frame"]
    frames = [[(fr[0]["type"], fr[0]["pos"], fr[0]["quat"]), (fr[1]["type"], [0.5, 0.0, 0.0], fr[1]["quat"])]]
    d = golden_dir("tiny")
    spec, out = str(tmp_path / "s.txt"), str(tmp_path / "o.txt")
    oracle.write_spec(spec, oracle.golden_moltypes(d), frames, salt=P["salt"], poles=P["poles"])
    got = oracle.run_spec(spec, out)
    assert not got[0]["ok"]
