"""Synthetic workloads with the shapes of the benchmark configurations.

Configuration "pose sweep, p = 30": two molecules of 60 dielectric spheres
(radii U(3,8) A, overlaps 0.5-1.5 A), 2000 charges U(-0.8,0.8) shifted to net
+4 / -4, eps_in 4, eps_out 78, 0.05 M, 298.15 K, pole order 30, inter-molecular
polarization cutoff 10 A; molecule B placed at centre distances 30, 32, ..., 80 A
from molecule A along a random axis with random orientations (26 poses).  A
distance at which two spheres would overlap is raised to the first distance
with a 1 A minimum surface gap (the reference cannot evaluate overlapping
poses), so every pose is a valid force evaluation.

Inputs are prepared on the GPU like the reference's `pbsam mat` and `pbsam spol`
(250 000 quadrature points per sphere) and written in the reference's file
formats when a directory is given, so the reference binaries can read them.
"""
import os
import struct

import numpy as np

from . import synth

SWEEP_P30 = dict(n_sph=60, r=(3.0, 8.0), n_q=2000, q_amp=0.8, nets=(4.0, -4.0), poles=30, salt=0.05,
                 idiel=4.0, dists=[30.0 + 2 * k for k in range(26)], min_gap=1.0, seeds=(2101, 2102),
                 pose_seed=2103)
SWEEP_P10 = dict(n_sph=8, r=(3.0, 6.0), n_q=300, q_amp=0.6, nets=(2.0, -2.0), poles=10, salt=0.05,
                 idiel=4.0, dists=[20.0 + 2 * k for k in range(11)], min_gap=1.0, seeds=(1, 2), pose_seed=7)
# Brownian dynamics of two-molecule encounters at p = 10 (bdnam): one pair of
# 35-sphere molecules (the mean of 10-60), charges as in the p = 10 case scaled to
# the sphere count, trajectories started at a 50 A centre distance with random
# orientations, escape at 150 A, time step 0.02 ps at contact rising linearly to 2 ps
# at a 30 A gap, Stokes-Einstein diffusion constants at 298.15 K (water, 0.89 mPa s)
# for a sphere of the molecule's extent.
BD_P10 = dict(n_sph=35, r=(3.0, 6.0), n_q=1200, q_amp=0.6, nets=(2.0, -2.0), poles=10, salt=0.05, idiel=4.0,
              seeds=(3101, 3102), pose_seed=3103, start=50.0, escape=150.0, dt_min=0.02, dt_max=2.0,
              dt_gap=30.0, viscosity=0.89e-3, temperature=298.15, min_gap=1.0)


# Brownian dynamics of molecules with uneven sphere counts (10..60 spheres per
# molecule, 300 charges U(-0.6, 0.6) per molecule): n_types "A" molecules (net +2) and
# n_types "B" molecules (net -2), every A-B pair a handle of per_pair trajectories.
BD_UNEVEN = dict(n_types=8, sizes=(10, 60), r=(3.0, 6.0), n_q=300, q_amp=0.6, nets=(2.0, -2.0), poles=10, salt=0.05,
                 idiel=4.0, seed=4100, pose_seed=4200, start=50.0, escape=150.0, dt_min=0.02, dt_max=2.0,
                 dt_gap=30.0, viscosity=0.89e-3, temperature=298.15, min_gap=1.0, per_pair=16)


# Many-body Brownian dynamics at p = 10 (bdm): 64 molecules of 30 spheres (radii
# U(3,6) A, 900 charges U(-0.6, 0.6)), 32 copies of molecule A (net +2) followed by
# 32 of molecule B (net -2), as CBDmulti holds its species, at random places and
# orientations in a periodic cube of 300 A with at least min_gap between any two
# molecules' spheres (minimum image); the reference bdm's own diffusion constants
# (D 0.015 A^2/ps, Dr 4.5e-5 and 4e-5 rad^2/ps, src/BDmulti.cpp:204-205) and time
# steps (pbsam_bd_params_default for the multi-molecule mode).
BD_MANY = dict(n_sph=30, r=(3.0, 6.0), n_q=900, q_amp=0.6, nets=(2.0, -2.0), poles=10, salt=0.05, idiel=4.0,
               seeds=(5101, 5102), pose_seed=5103, n_copies=32, box=300.0, min_gap=2.0,
               dtr=0.015, drot=(4.5e-5, 4e-5))


def many_start(cfg, mols, rank=0):
    """Species list, [n_mol, 3] positions and [n_mol, 4] quaternions of the many-body
    start: molecules placed one at a time at uniform random places (rejected while
    closer than min_gap to one already placed, minimum image)."""
    rng = np.random.default_rng(cfg["pose_seed"] + 7919 * rank)
    L = cfg["box"]
    shapes = [(m.centres, m.radii) for m in mols]
    ext = [m.extent() for m in mols]
    kinds = [0] * cfg["n_copies"] + [1] * cfg["n_copies"]
    pos, quat = [], []
    for k in kinds:
        for _ in range(10000):
            p = rng.uniform(-L / 2, L / 2, 3)
            q = synth.random_quat(rng)
            ok = True
            for j, (pj, qj) in enumerate(zip(pos, quat)):
                d = p - pj
                d -= L * np.round(d / L)
                if np.linalg.norm(d) > ext[k] + ext[kinds[j]] + cfg["min_gap"]:
                    continue
                if synth.min_gap(shapes[kinds[j]], np.zeros(3), qj, shapes[k], d, q) < cfg["min_gap"]:
                    ok = False
                    break
            if ok:
                break
        else:
            raise RuntimeError("no free place for molecule %d" % len(pos))
        pos.append(p)
        quat.append(q)
    return kinds, np.array(pos), np.array(quat)


def uneven_molecules(cfg):
    """(A molecules, B molecules) with sphere counts drawn uniformly from cfg['sizes']."""
    rng = np.random.default_rng(cfg["seed"])
    lo, hi = cfg["sizes"]
    out = []
    for side, net in enumerate(cfg["nets"]):
        out.append([synth.make_molecule(int(rng.integers(lo, hi + 1)), cfg["r"][0], cfg["r"][1], cfg["n_q"],
                                        cfg["q_amp"], net, seed=cfg["seed"] + 100 * (side + 1) + k)
                    for k in range(cfg["n_types"])])
    return out[0], out[1]


def stokes_einstein(radius_A, viscosity=0.89e-3, temperature=298.15):
    """(translational A^2/ps, rotational rad^2/ps) diffusion constants of a sphere."""
    kT = 1.3806503e-23 * temperature
    a = radius_A * 1e-10
    dt = kT / (6 * np.pi * viscosity * a) * 1e20 / 1e12
    dr = kT / (8 * np.pi * viscosity * a ** 3) / 1e12
    return dt, dr


def bd_start(cfg, mols, n_traj, rank=0):
    """Start poses of n_traj two-molecule trajectories: molecule A at the origin,
    molecule B at the start centre distance along a random axis (raised to the
    minimum gap where spheres would overlap), random orientations."""
    rng = np.random.default_rng(cfg["pose_seed"] + 7919 * rank)
    a = (mols[0].centres, mols[0].radii)
    b = (mols[1].centres, mols[1].radii)
    pos, quat = [], []
    for _ in range(n_traj):
        qa, qb, ax = synth.random_quat(rng), synth.random_quat(rng), synth.random_axis(rng)
        d = cfg["start"]
        if synth.min_gap(a, np.zeros(3), qa, b, d * ax, qb) < cfg["min_gap"]:
            d = synth.place_at_gap(a, qa, b, qb, ax, cfg["min_gap"])
        pos.append([[0.0, 0.0, 0.0], list(d * ax)])
        quat.append([list(qa), list(qb)])
    return np.array(pos), np.array(quat)


def molecules(cfg):
    return [synth.make_molecule(cfg["n_sph"], cfg["r"][0], cfg["r"][1], cfg["n_q"], cfg["q_amp"], net, seed=s)
            for net, s in zip(cfg["nets"], cfg["seeds"])]


def poses(cfg, mols, rank=0):
    """[n_pose, 2, 3] positions and [n_pose, 2, 4] quaternions (molecule A at the origin)."""
    rng = np.random.default_rng(cfg["pose_seed"] + 7919 * rank)
    a = (mols[0].centres, mols[0].radii)
    b = (mols[1].centres, mols[1].radii)
    pos, quat, dist = [], [], []
    for d in cfg["dists"]:
        qa, qb, ax = synth.random_quat(rng), synth.random_quat(rng), synth.random_axis(rng)
        dd = d
        if synth.min_gap(a, np.zeros(3), qa, b, d * ax, qb) < cfg["min_gap"]:
            dd = synth.place_at_gap(a, qa, b, qb, ax, cfg["min_gap"])
        pos.append([[0.0, 0.0, 0.0], list(dd * ax)])
        quat.append([list(qa), list(qb)])
        dist.append(dd)
    return np.array(pos), np.array(quat), np.array(dist)


def _pqr_round(mol):
    """Coordinates and charges as they read back from the PQR text (what the reference sees)."""
    import tempfile
    with tempfile.NamedTemporaryFile("w", suffix=".pqr", delete=False) as fh:
        path = fh.name
    synth.write_pqr(mol, path)
    out = synth.read_pqr(path)
    os.remove(path)
    return out


def write_imat(path, imat, poles):
    with open(path, "wb") as fh:
        fh.write(struct.pack("i", poles))
        fh.write(np.ascontiguousarray(imat, dtype=np.float64).tobytes())


def _fmt8(x):
    return "0" if abs(x) < 1e-15 else "%.8g" % x


def write_exp(path, coeffs, poles, scale):
    """Expansion text file as src/readutil.cpp:541-556 writes it."""
    with open(path, "w") as fh:
        fh.write("%d\n%s\n1000\n" % (poles, _fmt8(scale)))
        for n in range(poles):
            fh.write(" ".join(_fmt8(v) for v in coeffs[n * n:(n + 1) * (n + 1)]) + " \n")
        fh.write("\n")


def write_inputs(cfg, specs, outdir):
    """Write prepared inputs in the reference's formats (PQR, imat.sp<k>.out.bin,
    <name>.<k>.{F,H}.exp); returns per molecule (pqr, imat dir, exp dir, exp name)."""
    mols = molecules(cfg)
    files = []
    for k, (m, sp) in enumerate(zip(mols, specs)):
        tag = "AB"[k]
        os.makedirs(os.path.join(outdir, "im" + tag), exist_ok=True)
        os.makedirs(os.path.join(outdir, "exp" + tag), exist_ok=True)
        synth.write_pqr(m, os.path.join(outdir, "mol%s.pqr" % tag))
        for i in range(len(sp["radii"])):
            write_imat(os.path.join(outdir, "im" + tag, "imat.sp%d.out.bin" % i), sp["imats"][i], cfg["poles"])
            write_exp(os.path.join(outdir, "exp" + tag, "mol%s.0.%d.F.exp" % (tag, i)), sp["fself"][i],
                      cfg["poles"], sp["hself_scale"][i])
            write_exp(os.path.join(outdir, "exp" + tag, "mol%s.0.%d.H.exp" % (tag, i)), sp["hself"][i],
                      cfg["poles"], sp["hself_scale"][i])
        files.append((os.path.join(outdir, "mol%s.pqr" % tag), os.path.join(outdir, "im" + tag),
                      os.path.join(outdir, "exp" + tag), "mol%s.0" % tag))
    return files


def prepare(cfg, device=0, outdir=None, selfpol_rounds=1700, mols=None):
    """Build IMats and self-polarized expansions on the GPU (of the config's molecules,
    or of mols); returns (moltype specs for CSystem.create_moltype, prep timings, file
    specs or None)."""
    import time
    import pbsam_b200 as pb
    mols = molecules(cfg) if mols is None else mols
    specs, tm = [], {}
    prep = pb.CSystem(poles=cfg["poles"], salt=cfg["salt"], idiel=cfg["idiel"], device=device)
    types = []
    for k, m in enumerate(mols):
        cen, rad, pos, q = _pqr_round(m)
        t0 = time.time()
        im = prep.build_imats(cen, rad)
        tm["imat_s_%d" % k] = round(time.time() - t0, 2)
        ns = len(rad)
        P2 = cfg["poles"] ** 2
        types.append(prep.create_moltype(cen, rad, pos, q, im, np.zeros((ns, P2)), np.zeros((ns, P2)), 1.0 / rad))
        specs.append(dict(centres=cen, radii=rad, chg_pos=pos, chg=q, imats=im))
    for k, t in enumerate(types):
        t0 = time.time()
        F, H, sc, rounds = prep.self_polarize(t, max_rounds=selfpol_rounds)
        tm["selfpol_s_%d" % k] = round(time.time() - t0, 2)
        tm["selfpol_sweeps_%d" % k] = rounds
        specs[k].update(fself=F, hself=H, hself_scale=sc)
    prep.close()
    files = write_inputs(cfg, specs, outdir) if outdir else None
    return specs, tm, files


def open_context(cfg, specs, device=0, **kw):
    import pbsam_b200 as pb
    ctx = pb.CSystem(poles=cfg["poles"], salt=cfg["salt"], idiel=cfg["idiel"], device=device, **kw)
    types = [ctx.create_moltype(sp["centres"], sp["radii"], sp["chg_pos"], sp["chg"], sp["imats"], sp["fself"],
                                sp["hself"], sp["hself_scale"]) for sp in specs]
    return ctx, types
