"""Seeded synthetic coarse-grained molecules in the reference's PQR layout.

A molecule is a cluster of dielectric spheres grown by attaching each new
sphere to a random existing one at centre distance r1 + r2 - ov with
ov ~ U(ov_lo, ov_hi); a candidate is rejected when it overlaps any other
sphere by more than ``ov_hi`` or by a positive amount below ``ov_lo``.
Point charges are placed uniformly in the union of the spheres, at least
``inset`` inside the surface of the sphere they were drawn in, with
q ~ U(-q_amp, q_amp) shifted so that the net charge is exactly ``net``.

PQR lines follow what the reference reader expects (src/readutil.cpp:285-355):
``ATOM`` records, the tag ``CEN`` at byte 18 marks a sphere, and
``x y z charge radius`` are read whitespace-separated from byte 31; lines stay
below the reader's 99-byte buffer.
"""
import math
import numpy as np


class Molecule:
    def __init__(self, centres, radii, qpos, q):
        self.centres = np.asarray(centres, dtype=np.float64)
        self.radii = np.asarray(radii, dtype=np.float64)
        self.qpos = np.asarray(qpos, dtype=np.float64)
        self.q = np.asarray(q, dtype=np.float64)

    @property
    def n_spheres(self):
        return len(self.radii)

    def extent(self):
        """Radius of the smallest origin-centred ball (origin = mean sphere
        centre) that holds every sphere."""
        c = self.centres.mean(axis=0)
        return float(np.max(np.linalg.norm(self.centres - c, axis=1) + self.radii))


def make_molecule(n_sph, r_lo, r_hi, n_q, q_amp, net, seed,
                  ov_lo=0.5, ov_hi=1.5, inset=0.3):
    rng = np.random.default_rng(seed)
    cens = [np.zeros(3)]
    rads = [rng.uniform(r_lo, r_hi)]
    tries = 0
    while len(cens) < n_sph:
        tries += 1
        if tries > 200000:
            raise RuntimeError("sphere packing did not converge")
        r = rng.uniform(r_lo, r_hi)
        j = int(rng.integers(len(cens)))
        ov = rng.uniform(ov_lo, ov_hi)
        v = rng.normal(size=3)
        v /= np.linalg.norm(v)
        c = cens[j] + (rads[j] + r - ov) * v
        ok = True
        for k in range(len(cens)):
            if k == j:
                continue
            o = rads[k] + r - np.linalg.norm(c - cens[k])
            if o > ov_hi or (0.0 < o < ov_lo):
                ok = False
                break
        if ok:
            cens.append(c)
            rads.append(r)
    cens = np.array(cens)
    rads = np.array(rads)
    cens -= cens.mean(axis=0)
    vol = rads ** 3
    pos = []
    while len(pos) < n_q:
        k = int(rng.choice(len(rads), p=vol / vol.sum()))
        rr = rads[k] - inset
        while True:
            u = rng.uniform(-1.0, 1.0, size=3)
            if u @ u <= 1.0:
                break
        p = cens[k] + rr * u
        # thin to uniform density over the union: keep with prob 1/multiplicity
        mult = int(np.sum(np.linalg.norm(cens - p, axis=1) < rads - inset))
        if rng.uniform() * max(mult, 1) <= 1.0:
            pos.append(p)
    q = rng.uniform(-q_amp, q_amp, size=n_q)
    q += (net - q.sum()) / n_q
    return Molecule(cens, rads, np.array(pos), q)


def write_pqr(mol, path):
    lines = []
    serial = 1
    for i in range(len(mol.q)):
        x, y, z = mol.qpos[i]
        lines.append("ATOM  %5d  C    ATM %5d    %11.6f %11.6f %11.6f %9.5f %8.4f"
                     % (serial % 100000, 1, x, y, z, mol.q[i], 1.5))
        serial += 1
    for k in range(mol.n_spheres):
        x, y, z = mol.centres[k]
        lines.append("ATOM  %5d  O    CEN %5d    %11.6f %11.6f %11.6f %9.5f %8.4f"
                     % (serial % 100000, 2, x, y, z, 0.0, mol.radii[k]))
        serial += 1
    for ln in lines:
        assert ln[18:21] in ("CEN", "ATM") and len(ln) < 98 and ln[30] == " "
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def read_pqr(path):
    """Parse a PQR the way the reference does: returns (centres, radii, qpos, q)."""
    cens, rads, pos, q = [], [], [], []
    with open(path) as fh:
        for ln in fh:
            if not ln.startswith("ATOM"):
                continue
            vals = ln[31:].split()
            x, y, z, c, r = (float(v) for v in vals[:5])
            if ln[18:21] == "CEN":
                cens.append((x, y, z))
                rads.append(r)
            else:
                pos.append((x, y, z))
                q.append(c)
    return (np.array(cens), np.array(rads), np.array(pos).reshape(-1, 3), np.array(q))


def random_quat(rng):
    """Uniform random unit quaternion (w, x, y, z), the law of the reference's
    CQuat::chooseRandom (src/util.h:488-499) drawn from a numpy Generator."""
    s = rng.uniform()
    sig1 = math.sqrt(1.0 - s)
    sig2 = math.sqrt(s)
    t1 = 2.0 * math.pi * rng.uniform()
    t2 = 2.0 * math.pi * rng.uniform()
    q = np.array([math.cos(t2) * sig2, math.sin(t1) * sig1, math.cos(t1) * sig1, math.sin(t2) * sig2])
    return q / np.linalg.norm(q)


def random_axis(rng):
    v = rng.normal(size=3)
    return v / np.linalg.norm(v)


def salt_to_kappa(salt, sdiel=78.0, temperature=298.15):
    """Inverse Debye length in 1/Angstrom (src/BDnam_main.cpp:53-55)."""
    avo, echg, eps0, kb, ang, lit = 6.0221415e23, 1.60217646e-19, 8.854187817e-12, 1.3806503e-23, 1e-10, 1e-3
    return ang * math.sqrt((2 * salt * avo / lit * echg * echg) / (sdiel * eps0 * kb * temperature))


def quat_rotate(q, r):
    """Rotate vector(s) r by the unit quaternion q = (w, x, y, z) the way the
    reference does (CQuat * CPnt, src/util.h:463-468)."""
    w = q[0]
    v = np.asarray(q[1:], dtype=np.float64)
    r = np.asarray(r, dtype=np.float64)
    qr = np.cross(v, r)
    return r + 2.0 * (w * qr + np.cross(v, qr))


def min_gap(mol_a, pos_a, q_a, mol_b, pos_b, q_b):
    """Smallest surface-to-surface gap between the spheres of two placed
    molecules (each rotated about its mean sphere centre)."""
    ca = mol_a[0] - mol_a[0].mean(axis=0)
    cb = mol_b[0] - mol_b[0].mean(axis=0)
    pa = np.array([quat_rotate(q_a, c) for c in ca]) + pos_a
    pb = np.array([quat_rotate(q_b, c) for c in cb]) + pos_b
    d = np.linalg.norm(pa[:, None, :] - pb[None, :, :], axis=2)
    return float(np.min(d - mol_a[1][:, None] - mol_b[1][None, :]))


def place_at_gap(mol_a, q_a, mol_b, q_b, axis, gap, tol=1e-6):
    """Distance along ``axis`` at which molecule b (orientation q_b) sits with
    the given minimum sphere gap from molecule a at the origin (bisection)."""
    lo, hi = 0.0, 400.0
    axis = np.asarray(axis, dtype=np.float64)
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if min_gap(mol_a, np.zeros(3), q_a, mol_b, mid * axis, q_b) < gap:
            lo = mid
        else:
            hi = mid
        if hi - lo < tol:
            break
    return hi
