"""Parity at pole order 30, the order of the benchmarked pose sweep.

The inputs are prepared on the GPU (IMats with 250 000 quadrature points, 5
self-polarization sweeps), written in the reference's own formats (PQR,
imat.sp<k>.out.bin, <name>.<k>.{F,H}.exp) and read back by both sides: the CUDA
path through pbsam_moltype_load, and the reference compiled at N_POLES = 30 with
its own tolerances and -O2 (oracle/_ref/p30_default, built by oracle/build_ref.py)
through its force harness (CBDnam's molecule set-up, computeForces,
computeTotalIntEnergy).  Forces, torques and energy must agree within 1e-8
relative, the bar of the plain FP64 drop-in.

The reference's own result is not reproducible to 1e-8 on every pose at this order:
its inner F/H iteration has spectral radius above one on some spheres, so its capped
iterates amplify rounding, and the reference built with -O2 and with its Makefile's
-O3 -ffast-math disagrees with itself (2e-4 relative force on one pose of the small
workload here).  Each checked pose is therefore run through both builds; the bar is
1e-8 relative where the two builds agree to 1e-9 and ten times their own spread
elsewhere.  At least one polarized pose must be held to the reference's own
reproducibility: the GPU as close to the -O2 build as the -ffast-math build is, or
within 1e-8, whichever is looser.

Two workloads:
  * two 8-sphere molecules (300 charges each) at centre distances where the
    spheres of the two molecules polarize each other;
  * the benchmark's own two 60-sphere molecules (2000 charges), on poses of the
    26-pose sweep whose solve takes at most a few thousand inner iterations (the
    reference needs about 3 ms per inner iteration on one core).
"""
import os
import subprocess
import tempfile
import time

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
TOL = 1e-8
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(REPO, "oracle", "_ref", "p30_default", "harness")
HARNESS_FAST = os.path.join(REPO, "oracle", "_ref", "p30_fast", "harness")

SMALL_P30 = dict(n_sph=8, r=(3.0, 6.0), n_q=300, q_amp=0.6, nets=(2.0, -2.0), poles=30, salt=0.05, idiel=4.0,
                 dists=[18.0 + 1.5 * k for k in range(8)], min_gap=1.0, seeds=(1, 2), pose_seed=7)


def rel(a, b):
    b = np.asarray(b)
    return float(np.max(np.abs(np.asarray(a) - b)) / max(np.max(np.abs(b)), 1e-300))


def _spec(path, cfg, files, pos, quat):
    with open(path, "w") as fh:
        fh.write("salt %r\nidiel %r\ndump 0\nenergy 1\n" % (cfg["salt"], cfg["idiel"]))
        for fl in files:
            fh.write("moltype %s %s %s %s\n" % fl)
        fh.write("frame\n")
        for m in range(len(pos)):
            fh.write("mol %d %s %s\n" % (m, " ".join("%.17g" % v for v in pos[m]),
                                         " ".join("%.17g" % v for v in quat[m])))


def _run_reference(cfg, files, pos, quat, idx, workdir, limit_s=900):
    """Both reference builds on poses idx, one single-threaded process per pose and
    build; returns {pose: (default result, fast result)}."""
    procs = []
    for j in idx:
        spec = os.path.join(workdir, "p30_pose%d.txt" % j)
        _spec(spec, cfg, files, pos[j], quat[j])
        env = dict(os.environ, OMP_NUM_THREADS="1")
        for tag, exe in (("default", HARNESS), ("fast", HARNESS_FAST)):
            procs.append((j, tag, spec, subprocess.Popen([exe, spec, spec + "." + tag], env=env,
                                                         stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)))
    t0 = time.time()
    out = {}
    for j, tag, spec, p in procs:
        p.wait(timeout=max(1.0, limit_s - (time.time() - t0)))
        assert p.returncode == 0, "reference harness (%s) failed on pose %d" % (tag, j)
        fr = oracle.parse(spec + "." + tag)
        assert fr and fr[0]["ok"]
        out.setdefault(j, {})[tag] = fr[0]
    return {j: (v["default"], v["fast"]) for j, v in out.items()}


def _gpu_case(cfg, workdir, pick):
    """Prepare inputs on the GPU, write them, load them back through the C ABI and
    evaluate every pose; pick(stats) chooses the poses the reference checks."""
    import pbsam_b200 as pb
    from pbsam_b200 import workload
    specs, _, files = workload.prepare(cfg, outdir=workdir, selfpol_rounds=5)
    ctx = pb.CSystem(poles=cfg["poles"], salt=cfg["salt"], idiel=cfg["idiel"])
    try:
        types = [ctx.load_moltype(*fl) for fl in files]
        mols = workload.molecules(cfg)
        pos, quat, _ = workload.poses(cfg, mols)
        sysb = ctx.molecules(types, n_systems=len(pos))
        sysb.set_poses(pos, quat)
        f, t, st = sysb.compute_forces()
        e = sysb.compute_energy()
        stats = sysb.stats()
        sysb.close()
    finally:
        ctx.close()
    assert np.all(st == 0)
    idx = pick(stats)
    ref = _run_reference(cfg, files, pos, quat, idx, workdir)
    held = []
    for j in idx:
        r, rf = ref[j]
        spread = max(rel(rf["force"], r["force"]), rel(rf["torque"], r["torque"]),
                     abs(rf["energy"] - r["energy"]) / max(abs(r["energy"]), 1e-300))
        bar = TOL if spread <= 1e-9 else 10 * spread
        ef, et = rel(f[j], r["force"]), rel(t[j], r["torque"])
        ee = abs(e[j] - r["energy"]) / max(abs(r["energy"]), 1e-300)
        print("p=30 pose %d (inner its %d): GPU vs reference force %.2e torque %.2e energy %.2e; the reference's "
              "-O2 vs -ffast-math builds %.2e; bar %.1e" % (j, int(stats[j, 1]), ef, et, ee, spread, bar))
        assert ef < bar and et < bar and ee < bar, (j, ef, et, ee, spread)
        if max(ef, et, ee) <= max(TOL, spread) and stats[j, 1] > 0:
            held.append(j)
    return held


def _cheap_polarized(stats, max_its, n):
    """Up to n poses with a mutual solve of at most max_its inner iterations, plus the
    pose with the fewest iterations (only self-polarized interactions if none)."""
    its = stats[:, 1]
    pol = [int(j) for j in np.argsort(its, kind="stable") if 0 < its[j] <= max_its]
    pick = pol[-n:] if len(pol) > n else pol
    low = int(np.argmin(its))
    return sorted(set(pick + [low]))


@pytest.mark.skipif(not (os.path.exists(HARNESS) and os.path.exists(HARNESS_FAST)),
                    reason="reference p=30 builds missing (oracle/build_ref.py)")
def test_p30_small_molecules_vs_reference():
    with tempfile.TemporaryDirectory() as td:
        held = _gpu_case(SMALL_P30, td, lambda st: _cheap_polarized(st, 4000, 4))
    assert held, "no polarized pose held to the reference's own reproducibility"


@pytest.mark.skipif(not (os.path.exists(HARNESS) and os.path.exists(HARNESS_FAST)),
                    reason="reference p=30 builds missing (oracle/build_ref.py)")
def test_p30_benchmark_sweep_poses_vs_reference():
    from pbsam_b200 import workload
    with tempfile.TemporaryDirectory() as td:
        held = _gpu_case(dict(workload.SWEEP_P30), td, lambda st: _cheap_polarized(st, 3000, 3))
    assert held, "no polarized pose held to the reference's own reproducibility"
