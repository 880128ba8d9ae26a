"""bench.py's reference BD timing on CPU: the reference's own bdnam steps
(oracle/ref_bd_harness.cpp) run from given poses, one process per pose, and
report the wall time per step after the first."""
import json
import os
import sys

import numpy as np
import pytest

import oracle
from conftest import REPO, golden_dir

sys.path.insert(0, REPO)


def test_reference_bd_step_seconds(tmp_path):
    import bench
    if oracle.ref_bd_harness(6, "default") is None:
        pytest.skip("reference BD harness not built")
    P = json.load(open(os.path.join(golden_dir("tiny"), "poses.json")))
    fr = P["poses"][1]["frame"]
    pos = np.array([[m["pos"] for m in fr]] * 2)
    quat = np.array([[m["quat"] for m in fr]] * 2)
    cfg = dict(poles=6, salt=P["salt"], idiel=P["idiel"])
    t = bench.reference_bd_step_seconds(cfg, oracle.golden_moltypes(golden_dir("tiny")), pos, quat, 60,
                                        str(tmp_path), steps=3, variant="default")
    assert t is not None and len(t) == 2 and all(x > 0 for x in t)
