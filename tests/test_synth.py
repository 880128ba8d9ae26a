"""Synthetic inputs: packing rules, charge placement, PQR round trip, poses."""
import numpy as np

from pbsam_b200 import synth


def test_packing_rules():
    m = synth.make_molecule(12, 3, 6, 200, 0.6, 2.0, seed=3)
    d = np.linalg.norm(m.centres[:, None] - m.centres[None], axis=2)
    ov = m.radii[:, None] + m.radii[None] - d
    np.fill_diagonal(ov, -1)
    assert np.all(ov <= 1.5 + 1e-9)
    touching = ov > 0
    assert np.all(ov[touching] >= 0.5 - 1e-9)
    assert np.all(touching.sum(axis=1) >= 1)          # every sphere touches the cluster
    assert np.all((m.radii >= 3) & (m.radii <= 6))


def test_charges_inside_and_net():
    m = synth.make_molecule(8, 3, 6, 300, 0.6, -2.0, seed=4)
    assert abs(m.q.sum() + 2.0) < 1e-9
    inside = np.linalg.norm(m.qpos[:, None] - m.centres[None], axis=2) <= m.radii[None] - 0.3 + 1e-9
    assert np.all(inside.any(axis=1))


def test_pqr_round_trip(tmp_path):
    m = synth.make_molecule(5, 3, 6, 40, 0.6, 1.0, seed=5)
    p = tmp_path / "m.pqr"
    synth.write_pqr(m, str(p))
    cen, rad, pos, q = synth.read_pqr(str(p))
    assert np.allclose(cen, m.centres, atol=1e-6)
    assert np.allclose(rad, m.radii, atol=1e-4)
    assert np.allclose(pos, m.qpos, atol=1e-6) and np.allclose(q, m.q, atol=1e-5)
    for ln in open(p):
        assert len(ln.rstrip("\n")) < 98 and ln[18:21] in ("CEN", "ATM")


def test_quaternion_rotation():
    rng = np.random.default_rng(0)
    q = synth.random_quat(rng)
    assert abs(np.linalg.norm(q) - 1) < 1e-12
    v = rng.normal(size=3)
    r = synth.quat_rotate(q, v)
    assert abs(np.linalg.norm(r) - np.linalg.norm(v)) < 1e-12


def test_place_at_gap():
    rng = np.random.default_rng(1)
    A = synth.make_molecule(6, 3, 5, 30, 0.5, 1.0, seed=6)
    B = synth.make_molecule(6, 3, 5, 30, 0.5, -1.0, seed=7)
    a = (A.centres, A.radii)
    b = (B.centres, B.radii)
    qa, qb, ax = synth.random_quat(rng), synth.random_quat(rng), synth.random_axis(rng)
    d = synth.place_at_gap(a, qa, b, qb, ax, 4.0)
    g = synth.min_gap(a, np.zeros(3), qa, b, d * ax, qb)
    assert abs(g - 4.0) < 1e-4
