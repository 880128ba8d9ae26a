#!/usr/bin/env python3
"""Benchmark: polarization solves + forces per second, pose sweep at pole order 30.

Workload (one step = one pass of the hot path over one batch): two synthetic
molecules of 60 spheres (radii 3-8 A), 2000 charges, p = 30, molecule B at the 26
centre distances 30, 32, ..., 80 A (raised to a 1 A minimum gap where spheres
would overlap), random orientations; every pose is an independent system and one
step evaluates CMolecule::computeForces for all 26 of them (mutual polarization,
gradient solves, forces and torques).  Inputs (IMats, self-polarized F/H) are
prepared on the GPU before timing, exactly like the reference's `pbsam mat` and
`pbsam spol`.  The IMats (120 x 6.5 MB) exceed L2, so no flush is needed.

Multi-GPU: one process per GPU (torchrun), each rank solves its own batch of 26
poses (weak scaling, no data-path collective); rank 0 prints the max-over-ranks
device time.  --impl reference times the reference's own CPU implementation
(oracle/_ref, compiled from the reference sources) on the same workload.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "pb-sam_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))

METRIC = "pol. solves/s (computeForces calls per second), pose sweep p=30"
UNIT = "solves/s"


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks during the timed region."""

    def __init__(self, gpu):
        self.gpu = gpu
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for ln in open(self.path):
                f = [x.strip() for x in ln.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = float(f[2])
                except ValueError:
                    continue
                for n, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        except OSError:
            pass
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def algorithmic_bytes(stats, poles):
    """IMat bytes the solve must stream: two applications per inner F/H iteration
    (8 p^4 bytes each; the three gradient components share one read)."""
    return float(np.sum(stats[:, 1])) * 2 * 8 * poles ** 4


def run_ours(args):
    import torch
    import torch.distributed as dist
    from pbsam_b200 import replicas, workload
    rank, world, local = replicas.rank_env()
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    cfg = dict(workload.SWEEP_P30)
    t0 = time.time()
    specs, prep_t, _ = workload.prepare(cfg, device=local, selfpol_rounds=args.selfpol_rounds)
    ctx, types = workload.open_context(cfg, specs, device=local)
    mols = workload.molecules(cfg)
    pos, quat, dist_ = workload.poses(cfg, mols, rank=rank)
    B = len(dist_)
    sysb = ctx.molecules(types, n_systems=B)
    prep_s = time.time() - t0
    # device-resident inputs for the kernel-only rate
    dpos = torch.tensor(pos, dtype=torch.float64, device="cuda")
    dquat = torch.tensor(quat, dtype=torch.float64, device="cuda")
    dF = torch.zeros((B, 2, 3), dtype=torch.float64, device="cuda")
    dT = torch.zeros_like(dF)
    dS = torch.zeros(B, dtype=torch.int32, device="cuda")

    def step_device():
        sysb.set_poses_device(dpos.data_ptr(), dquat.data_ptr())
        sysb.compute_forces_device(dF.data_ptr(), dT.data_ptr(), dS.data_ptr())

    for _ in range(args.warmup):
        step_device()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    kernel_ms = []
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        e0.record()
        for _ in range(args.steps):
            step_device()
        e1.record()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if world > 1:
        dist.barrier()
    ms_max = replicas.max_over_ranks(ms, dist if world > 1 else None)
    status = dS.cpu().numpy()
    stats = sysb.stats()
    phases = sysb.phase_ms()
    # e2e: through the C ABI with host buffers (H2D poses, D2H forces/torques/status) each step
    hp, hq = np.ascontiguousarray(pos), np.ascontiguousarray(quat)
    torch.cuda.synchronize()
    t1 = time.time()
    for _ in range(args.steps):
        sysb.set_poses(hp, hq)
        f, t, st = sysb.compute_forces()
    torch.cuda.synchronize()
    e2e_s = time.time() - t1
    e2e_max = replicas.max_over_ranks(e2e_s, dist if world > 1 else None)
    # one launch timed alone for the roofline
    sysb.set_poses_device(dpos.data_ptr(), dquat.data_ptr())
    sysb.compute_forces_device(dF.data_ptr(), dT.data_ptr(), dS.data_ptr())
    torch.cuda.synchronize()
    one_ms = sysb.last_kernel_ms()
    launch_stats = sysb.stats()
    peak, peak_kind = measured_peaks()
    nbytes = algorithmic_bytes(launch_stats, cfg["poles"])
    achieved = nbytes / (one_ms * 1e-3) / 1e9
    out = None
    if rank == 0:
        units = B * world * args.steps
        out = {
            "metric": METRIC, "value": units / (ms_max * 1e-3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator; IMats and self-polarized expansions built on the GPU)",
            "config": {"workload": "pose sweep p=30: 2 molecules x 60 spheres (r 3-8 A), 2000 charges, "
                                   "26 centre distances 30-80 A, 0.05 M, eps 4/78",
                       "poles": cfg["poles"], "systems_per_gpu": B, "spheres_per_system": 120,
                       "parallelism": "replicas: %d ranks x %d independent systems" % (world, B),
                       "l2": "inputs larger than L2 (120 IMats x 6.5 MB), no flush"},
            "e2e": {"value": units / e2e_max, "unit": UNIT,
                    "h2d_bytes_per_step": int(hp.nbytes + hq.nbytes),
                    "d2h_bytes_per_step": int(2 * f.nbytes + st.nbytes)},
            "gpu_launches": args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind,
                         "kernel": "pbsam_forces_kernel", "launch_ms": one_ms,
                         "algorithmic_bytes_per_launch": nbytes},
            "clocks": clk.summary(),
            "status_ok": int(np.sum(status == 0)),
            "inner_iterations_per_step": int(np.sum(stats[:, 1])),
            "phase_ms_max_system": [round(float(x), 1) for x in phases[np.argmax(phases[:, 6])][:7]],
            "prep_s": round(prep_s, 1), "prep": prep_t,
        }
        if args.cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(cfg, specs, pos, quat, args)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    sysb.close()
    ctx.close()
    return out


def _ref_harness(poles):
    return os.path.join(REPO, "oracle", "_ref", "p%d_fast" % poles, "harness")


def _write_inputs(cfg, specs, outdir):
    from pbsam_b200 import workload
    mols = workload.molecules(cfg)
    files = []
    for k, (m, sp) in enumerate(zip(mols, specs)):
        tag = "AB"[k]
        for sub in ("im" + tag, "exp" + tag):
            os.makedirs(os.path.join(outdir, sub), exist_ok=True)
        workload.synth.write_pqr(m, os.path.join(outdir, "mol%s.pqr" % tag))
        for i in range(len(sp["radii"])):
            workload.write_imat(os.path.join(outdir, "im" + tag, "imat.sp%d.out.bin" % i), sp["imats"][i], cfg["poles"])
            workload.write_exp(os.path.join(outdir, "exp" + tag, "mol%s.0.%d.F.exp" % (tag, i)), sp["fself"][i],
                               cfg["poles"], sp["hself_scale"][i])
            workload.write_exp(os.path.join(outdir, "exp" + tag, "mol%s.0.%d.H.exp" % (tag, i)), sp["hself"][i],
                               cfg["poles"], sp["hself_scale"][i])
        files.append((os.path.join(outdir, "mol%s.pqr" % tag), os.path.join(outdir, "im" + tag),
                      os.path.join(outdir, "exp" + tag), "mol%s.0" % tag))
    return files


def _run_poses(files, cfg, pos, quat, idx, budget_s, ncores, outdir):
    """Run the reference harness on poses idx (one fresh process per pose, ncores at a
    time) until budget_s; returns (completed poses, elapsed s)."""
    import oracle
    procs, done, t0, k = [], 0, time.time(), 0
    while True:
        while len(procs) < ncores and k < len(idx) and time.time() - t0 < budget_s:
            j = idx[k]
            spec = os.path.join(outdir, "spec%d.txt" % k)
            with open(spec, "w") as fh:
                fh.write("salt %r\nidiel %r\ndump 0\nenergy 0\n" % (cfg["salt"], cfg["idiel"]))
                for f in files:
                    fh.write("moltype %s %s %s %s\n" % f)
                fh.write("frame\n")
                for m in range(2):
                    fh.write("mol %d %s %s\n" % (m, " ".join("%.17g" % v for v in pos[j][m]),
                                                 " ".join("%.17g" % v for v in quat[j][m])))
            env = dict(os.environ, OMP_NUM_THREADS="1")
            procs.append(subprocess.Popen([_ref_harness(cfg["poles"]), spec, spec + ".out"], env=env,
                                          stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL))
            k += 1
        if not procs:
            break
        time.sleep(0.2)
        still = []
        for p in procs:
            if p.poll() is None:
                if time.time() - t0 > budget_s * 4:
                    p.kill()
                    p.wait()
                else:
                    still.append(p)
            elif p.returncode == 0:
                done += 1
        procs = still
        if k >= len(idx) and not procs:
            break
    _ = oracle
    return done, time.time() - t0


def cpu_baseline(cfg, specs, pos, quat, args):
    """The reference (compiled from its sources with its Makefile flags and a plain cblas
    stand-in for MKL) on a bounded sample of the same poses, one single-threaded process
    per pose (its OpenMP path races) on all host cores."""
    if not os.path.exists(_ref_harness(cfg["poles"])):
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": "reference binary not built"}
    ncores = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as td:
        files = _write_inputs(cfg, specs, td)
        order = list(range(len(pos)))[::-1]          # sweep from the far end (cheapest poses first)
        done, el = _run_poses(files, cfg, pos, quat, order, args.cpu_budget, ncores, td)
    return {"value": done / el if el > 0 else None, "unit": UNIT, "cores": min(ncores, len(pos)), "kind": "reference",
            "sample": "%d poses completed in %.0f s (budget %d s), far end of the sweep first, 1 thread per pose"
                      % (done, el, args.cpu_budget)}


def run_reference(args):
    from pbsam_b200 import replicas, workload
    rank, world, local = replicas.rank_env()
    if rank != 0:
        return None
    cfg = dict(workload.SWEEP_P30)
    if not os.path.exists(_ref_harness(cfg["poles"])):
        return {"impl": "reference", "unavailable": "reference binary oracle/_ref/p30_fast/harness not built"}
    specs, _, _ = workload.prepare(cfg, device=local, selfpol_rounds=args.selfpol_rounds)
    mols = workload.molecules(cfg)
    pos, quat, _ = workload.poses(cfg, mols)
    ncores = os.cpu_count() or 1
    vals = []
    with tempfile.TemporaryDirectory() as td:
        files = _write_inputs(cfg, specs, td)
        order = list(range(len(pos)))[::-1]
        for s in range(args.warmup + args.steps):
            done, el = _run_poses(files, cfg, pos, quat, order, args.cpu_budget, ncores, td)
            if s >= args.warmup:
                vals.append(done / el)
    v = float(np.mean(vals))
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": {"workload": "pose sweep p=30 (same poses)"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": min(ncores, len(pos)), "kind": "reference",
                             "sample": "poses from the far end of the sweep, %d s per step" % args.cpu_budget},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--selfpol-rounds", type=int, default=1700)
    ap.add_argument("--cpu-baseline", type=int, default=1)
    ap.add_argument("--cpu-budget", type=int, default=30)
    args = ap.parse_args()
    out = run_reference(args) if args.impl == "reference" else run_ours(args)
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
