"""bdm restart configurations (pbsam_config_read / pbsam_config_write), host only: the
format CMolecule::saveConfig writes (src/molecule.cpp:255-269, the stream's default
six significant digits) read back as readConfigWithMolType reads it
(src/readutil.cpp:835-886); full-precision round trips; truncated or malformed files
refused with PBSAM_E_IO, too many molecules with PBSAM_E_BADARG."""
import os

import numpy as np
import pytest

from conftest import REPO

LIB = os.path.join(REPO, "pb-sam_b200", "lib", "libpbsam_b200.so")
pytestmark = pytest.mark.skipif(not os.path.exists(LIB), reason="library not built")


def saveconfig_text(pos, quat, mt):
    """The reference's saveConfig lines: operator<< on doubles at the default precision."""
    lines = []
    for p, q, t in zip(pos, quat, mt):
        vals = list(p) + list(q)
        lines.append(" ".join("%.6g" % v for v in vals) + " %d" % t)
    return "\n".join(lines) + "\n"


def test_reads_the_reference_format(tmp_path):
    import pbsam_b200 as pb
    rng = np.random.default_rng(5)
    pos = rng.uniform(-150, 150, (7, 3))
    quat = rng.standard_normal((7, 4))
    quat /= np.linalg.norm(quat, axis=1, keepdims=True)
    mt = np.array([0, 0, 0, 0, 1, 1, 1])
    path = str(tmp_path / "restart_run.config")
    with open(path, "w") as fh:
        fh.write(saveconfig_text(pos, quat, mt))
    p2, q2, t2 = pb.config_read(path)
    want = np.array([[float("%.6g" % v) for v in list(a) + list(b)] for a, b in zip(pos, quat)])
    assert np.array_equal(np.hstack([p2, q2]), want) and np.array_equal(t2, mt)


def test_full_precision_round_trip_and_errors(tmp_path):
    import pbsam_b200 as pb
    rng = np.random.default_rng(6)
    pos = rng.uniform(-150, 150, (5, 3))
    quat = rng.standard_normal((5, 4))
    mt = np.array([0, 1, 0, 1, 1], dtype=np.int32)
    path = str(tmp_path / "c.config")
    pb.config_write(path, pos, quat, mt)
    p2, q2, t2 = pb.config_read(path)
    assert np.array_equal(p2, pos) and np.array_equal(q2, quat) and np.array_equal(t2, mt)
    # a file that ends inside a molecule
    txt = open(path).read().split()
    with open(path, "w") as fh:
        fh.write(" ".join(txt[:-3]) + "\n")
    with pytest.raises(pb.PbsamError) as e:
        pb.config_read(path)
    assert e.value.code == -2 and "ends inside" in str(e.value)   # PBSAM_E_IO
    # a field that is not a number
    with open(path, "w") as fh:
        fh.write("1 2 3 1 0 0 0 0\n4 5 x 1 0 0 0 1\n")
    with pytest.raises(pb.PbsamError):
        pb.config_read(path)
    # more molecules than the caller's arrays
    import ctypes
    pb.config_write(path, pos, quat, mt)
    n = ctypes.c_int()
    buf = np.zeros(3 * 2)
    rc = pb.lib().pbsam_config_read(path.encode(), 2, ctypes.byref(n), buf.ctypes.data_as(pb._DP), None, None)
    assert rc != 0 and n.value == 5
