#!/usr/bin/env python3
"""Benchmark: polarization solves + forces per second, pose sweep at pole order 30.

Workload (one step = one pass of the hot path over one batch): two synthetic
molecules of 60 spheres (radii 3-8 A), 2000 charges, p = 30, molecule B at the 26
centre distances 30, 32, ..., 80 A (raised to a 1 A minimum gap where spheres
would overlap), random orientations; every pose is an independent system and one
step evaluates CMolecule::computeForces for all 26 of them (mutual polarization,
gradient solves, forces and torques).  Inputs (IMats, self-polarized F/H) are
prepared on the GPU before timing, like the reference's `pbsam mat` and
`pbsam spol` (5 self-polarization sweeps).  The IMats (120 x 6.5 MB) exceed L2,
so no flush is needed.

The same line carries a Brownian-dynamics leg ("bd", --bd 1): 1024 independent
two-molecule bdnam trajectories at p = 10 (35 + 35 spheres), each step a force
evaluation where the pair is inside the force distance plus the Ermak-McCammon
move, one CUDA graph per step of the whole batch; BD steps/s with its own e2e,
clocks and the reference's computeForces timed on the host cores.  Further legs:
"bd_exact" (the same trajectories, exact form with adjoint forces, checked against
central differences), "bd_uneven" (1024 trajectories of molecules of 10-60 spheres in
64 handles, one group launch per step against the handles' own launches) and
"bd_many" (bdm dynamics of 148 systems of 64 molecules x 30 spheres in a periodic
300 A cube, with the reference's own bdm timed on the host cores).

Multi-GPU: one process per GPU (torchrun), each rank solves its own batch of 26
poses and its own 1024 trajectories (weak scaling, no data-path collective); rank 0
prints the max-over-ranks device time.  --impl reference times the reference's own
CPU implementation (oracle/_ref, compiled from the reference sources) on the same
poses.
"""
import argparse
import datetime
import json
import os
import subprocess
import sys
import tempfile
import time
from collections import Counter

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "pb-sam_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))

METRIC = "pol. solves/s (computeForces calls per second), pose sweep p=30"
UNIT = "solves/s"
WORKLOAD = ("pose sweep p=30: 2 molecules x 60 spheres (r 3-8 A), 2000 charges (net +4/-4), "
            "26 centre distances 30-80 A, eps 4/78, 0.05 M, 298.15 K")


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi SM clocks and throttle reasons of one GPU during the timed region."""
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu_id), "--query-gpu=" + q,
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
                for n, v in zip(self.NAMES, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        except OSError:
            pass
        os.remove(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def gpu_id_for_smi(local):
    import torch
    try:
        u = str(torch.cuda.get_device_properties(local).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return str(local)


def measured_traffic_per_inner_iteration():
    """DRAM bytes (read + write) per inner F/H iteration of the force kernel, from
    the ncu capture summarised in profiles/ (a small case of the same kernel;
    traffic grows with the inner iterations, which dominate it)."""
    p = os.path.join(REPO, "profiles", "pbsam_forces_kernel_p30_traffic.txt")
    if os.path.exists(p):
        for ln in open(p):
            t = ln.split()
            if len(t) == 2 and t[0] == "dram_bytes_per_inner_iteration":
                return float(t[1])
    return None


def algorithmic_bytes(stats, poles):
    """IMat bytes the solve must stream: every inner F/H iteration applies the
    p^2 x p^2 FP64 IMat twice (8 p^4 bytes each; D = 3 gradient solves share one
    read of the matrix across their three operands)."""
    return float(np.sum(stats[:, 1])) * 2 * 8 * float(poles) ** 4


def run_ours(args):
    import torch
    import torch.distributed as dist
    import pbsam_b200 as pb
    from pbsam_b200 import replicas, workload
    rank, world, local = replicas.rank_env()
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))
    torch.cuda.set_device(local)
    cfg = dict(workload.SWEEP_P30)
    t0 = time.time()
    specs, prep_t, _ = workload.prepare(cfg, device=local, selfpol_rounds=args.selfpol_rounds)
    ctx, types = workload.open_context(cfg, specs, device=local, cluster_size=args.cluster_size)
    mols = workload.molecules(cfg)
    pos, quat, _ = workload.poses(cfg, mols, rank=rank)
    if args.poses:
        sel = [int(x) for x in args.poses.split(",")]
        pos, quat = pos[sel], quat[sel]
    B = len(pos)
    sysb = ctx.molecules(types, n_systems=B)
    stream = torch.cuda.current_stream()
    sysb.set_stream(stream.cuda_stream)
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
    with ClockSampler(gpu_id_for_smi(local)) as clk, torch.cuda.nvtx.range("sweep"):   # NVTX: ncu --nvtx-include
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            step_device()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    clocks = clk.summary()
    if world > 1:
        dist.barrier()
    ms_max = replicas.max_over_ranks(ms, dist if world > 1 else None)
    status = dS.cpu().numpy()
    stats = sysb.stats()
    phases = sysb.phase_ms()
    # e2e: the public API with host buffers; H2D of the poses and D2H of forces,
    # torques and status inside the timed region, every step
    hp, hq = np.ascontiguousarray(pos), np.ascontiguousarray(quat)
    ee0, ee1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ee0.record(stream)
    for _ in range(args.steps):
        sysb.set_poses(hp, hq)
        f, t, st = sysb.compute_forces()
    ee1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = ee0.elapsed_time(ee1)
    e2e_max = replicas.max_over_ranks(e2e_ms, dist if world > 1 else None)
    # roofline of the (only) kernel of a step: its algorithmic IMat bytes over its
    # average duration inside the timed region
    peak, peak_kind = measured_peaks()
    launch_ms = ms / args.steps
    nbytes = algorithmic_bytes(stats, cfg["poles"])
    achieved = nbytes / (launch_ms * 1e-3) / 1e9
    # the IMat rows are re-read from L2 (DRAM sees ~1% of these bytes) and the arithmetic
    # is FP64 on CUDA cores: both rates measured on this device
    fp64_peak, l2_peak = pb.device_peaks(local)
    nflops = float(np.sum(stats[:, 1])) * 2 * 2 * float(cfg["poles"]) ** 4
    traffic = args.traffic_per_launch
    per_it = measured_traffic_per_inner_iteration()
    if traffic is None and per_it is not None:
        traffic = per_it * float(np.sum(stats[:, 1]))
    out = None
    if rank == 0:
        units = B * world * args.steps
        out = {
            "metric": METRIC, "value": units / (ms_max * 1e-3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator; IMats and self-polarized expansions built on the GPU)",
            "config": {"workload": WORKLOAD, "poses": args.poses or "all", "poles": cfg["poles"],
                       "systems_per_gpu": B,
                       "spheres_per_system": 2 * cfg["n_sph"],
                       "parallelism": "replicas: %d rank(s) x %d independent systems; CTAs per system %s" % (
                           world, B, dict(sorted(Counter(int(x) for x in stats[:, 5]).items()))),
                       "l2": "no flush: inputs larger than L2 (120 IMats x 6.5 MB = 778 MB)"},
            "e2e": {"value": units / (e2e_max * 1e-3), "unit": UNIT,
                    "h2d_bytes_per_step": int(hp.nbytes + hq.nbytes),
                    "d2h_bytes_per_step": int(f.nbytes + t.nbytes + st.nbytes)},
            # one force-kernel launch per crew size in use (adaptive crews: up to 4) per step
            "gpu_launches": args.steps * len(set(int(x) for x in stats[:, 5])),
            "roofline": {"bound": "l2", "achieved": achieved, "peak": l2_peak, "unit": "GB/s",
                         "frac": achieved / l2_peak, "traffic": traffic,
                         "peak_kind": "measured in place (L2 read bandwidth over every SM, pbsam_device_peaks)",
                         "kernel": "pbsam_forces_kernel", "launch_ms": launch_ms,
                         "algorithmic_bytes_per_launch": nbytes,
                         "hbm": {"achieved_if_from_dram": achieved, "peak": peak, "peak_kind": peak_kind,
                                 "frac": achieved / peak,
                                 "dram_traffic_fraction": (traffic / nbytes) if traffic else None},
                         "fp64": {"achieved_tflops": nflops / (launch_ms * 1e-3) / 1e12,
                                  "peak_tflops": fp64_peak, "frac": nflops / (launch_ms * 1e-3) / 1e12 / fp64_peak,
                                  "algorithmic_flops_per_launch": nflops}},
            "clocks": clocks,
            "systems_ok": int(np.sum(status == 0)),
            "inner_iterations_per_step": int(np.sum(stats[:, 1])),
            "slowest_system_phase_ms": dict(zip(
                ["solve", "surface", "numeric", "intra", "LS", "DTA", "grad_reexp", "total", "grad_surface",
                 "setup", "grad_book", "forces", "grad_reexp_inter", "grad_reexp_analytic", "grad_reexp_numeric",
                 "solve_matvec"],
                [round(float(x), 1) for x in phases[int(np.argmax(phases[:, 7]))]])),
            "prep_s": round(prep_s, 1), "prep": prep_t,
        }
        if args.cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(cfg, specs, pos, quat, args)
    sysb.close()
    ctx.close()
    if args.bd:
        specs_bd = None
        try:
            bd, specs_bd = run_bd(args, local, rank, world, dist)
        except Exception as e:   # the headline line stands without the BD leg
            bd = {"error": "%s: %s" % (type(e).__name__, e), "gpu_launches": 0}
        if out is not None:
            out["bd"] = bd
            out["gpu_launches"] += bd["gpu_launches"]
        if args.bd_exact:
            try:
                bdx, _ = run_bd(args, local, rank, world, dist, exact=True, specs=specs_bd)
                if "value" in bd and "value" in bdx:
                    bdx["vs_plain_bd"] = bdx["value"] / bd["value"]
            except Exception as e:
                bdx = {"error": "%s: %s" % (type(e).__name__, e), "gpu_launches": 0}
            if out is not None:
                out["bd_exact"] = bdx
                out["gpu_launches"] += bdx["gpu_launches"]
        if args.bd_uneven:
            try:
                bdu = run_bd_uneven(args, local, rank, world, dist)
            except Exception as e:
                bdu = {"error": "%s: %s" % (type(e).__name__, e), "gpu_launches": 0}
            if out is not None:
                out["bd_uneven"] = bdu
                out["gpu_launches"] += bdu["gpu_launches"]
        if args.bd_many:
            try:
                bdm = run_bd_many(args, local, rank, world, dist)
            except Exception as e:
                bdm = {"error": "%s: %s" % (type(e).__name__, e), "gpu_launches": 0}
            if out is not None:
                out["bd_many"] = bdm
                out["gpu_launches"] += bdm["gpu_launches"]
            if args.bd_many_exact:
                try:
                    bdmx = run_bd_many(args, local, rank, world, dist, exact=True)
                    if "value" in bdm and "value" in bdmx:
                        bdmx["vs_plain_bd"] = bdmx["value"] / bdm["value"]
                except Exception as e:
                    bdmx = {"error": "%s: %s" % (type(e).__name__, e), "gpu_launches": 0}
                if out is not None:
                    out["bd_many_exact"] = bdmx
                    out["gpu_launches"] += bdmx["gpu_launches"]
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return out


# ---------------------------------------------------------------- Brownian dynamics leg
BD_METRIC = "BD steps/s (two-molecule bdnam trajectories, p=10)"
BD_WORKLOAD = ("bdnam p=10: %d trajectories of 2 molecules x 35 spheres (r 3-6 A, 1200 charges, net +2/-2), start "
               "50 A, escape 150 A, dt 0.02 ps at contact rising to 2 ps at a 30 A gap, Stokes-Einstein D, Philox "
               "noise; a step = force evaluation (where c2c < 100 A) + Ermak-McCammon move, one CUDA graph")


def fd_force_check(ctx, types, poses, quats, h=1e-3, hr=1e-4):
    """Relative error of the exact form's adjoint forces and torques against central
    differences of its lab-frame energy (h A, hr rad) on several poses, every perturbed
    pose a system of one batch.  The energy has steps where a sphere pair crosses the
    polarization cutoff or a truncation order changes; a pose whose central differences
    at h and h/4 disagree by more than 1e-4 has one within reach and is left out (and
    counted)."""
    n = poses[0].shape[0]

    def qmul(a, b):
        w1, v1, w2, v2 = a[0], a[1:], b[0], b[1:]
        return np.concatenate([[w1 * w2 - v1 @ v2], w1 * v2 + w2 * v1 + np.cross(v1, v2)])

    P, Q = [], []
    for pos, quat in zip(poses, quats):
        P.append(pos)
        Q.append(quat)
        for hh, hhr in ((h, hr), (h / 4, hr / 4)):
            for i in range(n):
                for c in range(3):
                    for sg in (1, -1):
                        p = pos.copy()
                        p[i, c] += sg * hh
                        P.append(p)
                        Q.append(quat)
                    for sg in (1, -1):
                        ax = np.zeros(3)
                        ax[c] = np.sin(sg * hhr / 2)
                        q = quat.copy()
                        q[i] = qmul(np.concatenate([[np.cos(sg * hhr / 2)], ax]), quat[i])
                        P.append(pos)
                        Q.append(q)
    m = ctx.molecules(types, n_systems=len(P))
    m.set_poses(np.array(P), np.array(Q))
    f, t, st = m.compute_forces()
    E = m.compute_energy(lab=True)
    m.close()
    per = 1 + 2 * 12 * n

    def rel(a, b):
        return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
    errs_f, errs_t, rough = [], [], 0
    for k in range(len(poses)):
        b = k * per
        E1 = E[b + 1:b + 1 + 12 * n].reshape(n, 3, 4)
        E4 = E[b + 1 + 12 * n:b + per].reshape(n, 3, 4)
        fd = [(-(Ex[:, :, 0] - Ex[:, :, 1]) / (2 * hh), -(Ex[:, :, 2] - Ex[:, :, 3]) / (2 * hhr))
              for Ex, hh, hhr in ((E1, h, hr), (E4, h / 4, hr / 4))]
        if st[b] != 0 or rel(fd[0][0], fd[1][0]) > 1e-4 or rel(fd[0][1], fd[1][1]) > 1e-4:
            rough += 1
            continue
        errs_f.append(rel(f[b], fd[0][0]))
        errs_t.append(rel(t[b], fd[0][1]))
    return {"force_rel_err": max(errs_f) if errs_f else None, "torque_rel_err": max(errs_t) if errs_t else None,
            "h_A": h, "h_rad": hr, "poses": len(poses), "poses_checked": len(errs_f),
            "poses_with_a_step_within_h": rough}


def vs_converged(cfg, specs, local, ctx, types, state, sel):
    """Forces and torques of the exact form at the leg's exact_tol / exact_relax against
    the default (exact_tol 1e-14, plain Gauss-Seidel) on the same poses, both evaluated
    from the self-polarized state: the largest per-system relative difference."""
    from pbsam_b200 import workload
    ref_ctx, ref_types = workload.open_context(cfg, specs, device=local, exact=1)
    res = []
    for c, t in ((ref_ctx, ref_types), (ctx, types)):
        m = c.molecules(t, n_systems=len(sel))
        m.set_poses(state["pos"][sel], state["quat"][sel])
        f, tq, st = m.compute_forces()
        res.append((f, tq, st, float(m.stats()[:, 0].mean())))
        m.close()
    ref_ctx.close()
    (f0, t0, st0, sw0), (f1, t1, st1, sw1) = res

    def worst(a, b):
        return float(max(np.max(np.abs(a[k] - b[k])) / max(np.max(np.abs(b[k])), 1e-300) for k in range(len(b))))
    return {"force_rel_err": worst(f1, f0), "torque_rel_err": worst(t1, t0), "systems": len(sel),
            "statuses_ok": int(np.sum(st1 == 0)), "mean_sweeps": sw1, "mean_sweeps_converged": sw0}


def run_bd(args, local, rank, world, dist, exact=False, specs=None):
    """BD steps per second of a batch of independent two-molecule trajectories:
    every step (a CUDA graph: time step and force mask, force kernel, move kernel)
    of every trajectory counts as one unit.  exact: the exact form (direct inner
    solves, sweeps to the fixed point, forces by the adjoint of the lab-frame energy)."""
    import torch
    from pbsam_b200 import replicas, workload
    cfg = dict(workload.BD_P10)
    prep_t = {}
    if specs is None:
        specs, prep_t, _ = workload.prepare(cfg, device=local, selfpol_rounds=args.selfpol_rounds_p10)
    t_ctx = time.time()
    xkw = {"exact": 1, "exact_tol": args.exact_tol, "exact_relax": args.exact_relax} if exact else {}
    ctx, types = workload.open_context(cfg, specs, device=local, **xkw)
    mols = workload.molecules(cfg)
    B = args.bd_traj
    pos, quat = workload.bd_start(cfg, mols, B, rank=rank)
    ext = max(m.extent() for m in mols)
    dtr, drot = workload.stokes_einstein(ext, cfg["viscosity"], cfg["temperature"])
    sysb = ctx.molecules(types, n_systems=B)
    prep_t["context_s"] = round(time.time() - t_ctx, 2)
    stream = torch.cuda.current_stream()
    sysb.set_stream(stream.cuda_stream)
    sysb.set_poses(pos, quat)
    sysb.bd_init([0.0, dtr], [drot, drot], mode=0, seed=1234 + rank, escape_dist=cfg["escape"],
                 dt_min=cfg["dt_min"], dt_max=cfg["dt_max"], dt_ref=0.0,
                 dt_div=cfg["dt_gap"] / (cfg["dt_max"] - cfg["dt_min"]))
    sysb.bd_run(args.warmup)
    torch.cuda.synchronize()
    s0 = sysb.bd_state()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(gpu_id_for_smi(local)) as clk, torch.cuda.nvtx.range("bd_exact" if exact else "bd"):
        torch.cuda.synchronize()
        e0.record(stream)
        sysb.bd_run(args.bd_steps)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    clocks = clk.summary()
    s1 = sysb.bd_state()
    st_timed = sysb.stats()          # counters of the last timed step
    ms_max = replicas.max_over_ranks(ms, dist if world > 1 else None)
    units = int(np.sum(s1["steps"] - s0["steps"]))
    fe = int(np.sum(s1["fevals"] - s0["fevals"]))
    units_all = replicas.sum_over_ranks(units, dist if world > 1 else None)
    # e2e: one step at a time through the public API with the poses, statuses and
    # counters read back to the host after every step
    ee0, ee1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n_e2e = max(1, args.bd_steps // 2)
    torch.cuda.synchronize()
    ee0.record(stream)
    for _ in range(n_e2e):
        sysb.bd_run(1)
        st = sysb.bd_state()
    ee1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = replicas.max_over_ranks(ee0.elapsed_time(ee1), dist if world > 1 else None)
    e2e_units = replicas.sum_over_ranks(int(np.sum(st["steps"] - s1["steps"])), dist if world > 1 else None)
    d2h = sum(int(v.nbytes) for v in st.values())
    out = {"metric": BD_METRIC, "value": units_all / (ms_max * 1e-3), "unit": "BD steps/s",
           "ms_per_step": ms_max / args.bd_steps, "steps": args.bd_steps, "warmup": args.warmup, "dtype": "f64",
           "config": {"workload": BD_WORKLOAD % B, "trajectories_per_gpu": B, "dtr_A2_per_ps": dtr,
                      "drot_rad2_per_ps": drot},
           "force_evaluations_fraction": fe / max(units, 1),
           "status_counts": {pb_status: int(np.sum(s1["status"] == k)) for k, pb_status in
                             ((0, "running"), (1, "escaped"), (2, "stuck"), (4, "failed"))},
           "e2e": {"value": e2e_units / (e2e_ms * 1e-3), "unit": "BD steps/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": d2h, "note": "one step per call, state read back to the host each step"},
           "gpu_launches": 3 * args.bd_steps, "clocks": clocks, "prep": prep_t}
    if not exact:
        # roofline of the force kernel (99.99 % of a step): the IMat bytes of the last
        # timed step's inner iterations (16 p^4 bytes each, re-read from L2) over the
        # average step time, and its FP64 rate; the solve is only part of a BD
        # evaluation (mean_phase_ms), the rest being latency-bound re-expansions
        import pbsam_b200 as pb
        fp64_peak, l2_peak = pb.device_peaks(local)
        P = cfg["poles"]
        its = float(np.sum(st_timed[:, 1]))
        step_ms = ms / args.bd_steps
        nbytes, nflops = its * 16.0 * P ** 4, its * 4.0 * P ** 4
        out_roof = {"bound": "l2", "achieved": nbytes / (step_ms * 1e-3) / 1e9, "peak": l2_peak, "unit": "GB/s",
                    "frac": nbytes / (step_ms * 1e-3) / 1e9 / l2_peak, "traffic": None,
                    "peak_kind": "measured in place (L2 read bandwidth over every SM, pbsam_device_peaks)",
                    "kernel": "pbsam_forces_kernel", "launch_ms": step_ms, "algorithmic_bytes_per_launch": nbytes,
                    "units": "inner F/H iterations of the last timed step (%d) stand for every step" % int(its),
                    "fp64": {"achieved_tflops": nflops / (step_ms * 1e-3) / 1e12, "peak_tflops": fp64_peak,
                             "frac": nflops / (step_ms * 1e-3) / 1e12 / fp64_peak}}
    ph = sysb.phase_ms()
    names = ["solve", "surface", "numeric", "intra", "LS", "DTA", "grad_or_backward", "total"]
    out["mean_phase_ms"] = {k: round(float(v), 2) for k, v in zip(names, ph[:, :8].mean(axis=0))}
    if not exact:
        out["roofline"] = out_roof
    if exact:
        out["mean_phase_ms"].update({k: round(float(v), 2) for k, v in zip(
            ["backward_energy", "backward_sweeps", "backward_first_round"], ph[:, 12:15].mean(axis=0))})
    st_last = sysb.stats()
    out["mean_sweeps"] = float(st_last[:, 0].mean())
    out["mean_inner_solves"] = float(st_last[:, 2].mean())
    if exact:
        out["metric"] = BD_METRIC + ", exact form with adjoint forces"
        out["config"]["form"] = ("exact: direct inner solves, sweeps to the fixed point, forces and torques the "
                                 "negative gradient of the lab-frame energy by the adjoint (lab frame)")
        out["config"]["exact_tol"] = args.exact_tol
        out["config"]["exact_relax"] = args.exact_relax
        run = [b for b in range(B) if s1["status"][b] == 0]
        if rank == 0 and run:
            out["accuracy"] = fd_force_check(ctx, types, s1["pos"][run[:8]], s1["quat"][run[:8]])
            if args.exact_tol != 1e-14 or args.exact_relax != 1.0:
                out["accuracy"]["vs_converged"] = vs_converged(cfg, specs, local, ctx, types, s1, run[:32])
    if rank == 0 and args.cpu_baseline and not exact:
        out["cpu_baseline"] = bd_cpu_baseline(cfg, specs, sysb, s1, fe / max(units, 1), args)
    sysb.close()
    ctx.close()
    return out, specs


def run_bd_uneven(args, local, rank, world, dist):
    """BD steps/s of 1024 two-molecule trajectories whose molecules have uneven sphere
    counts (8 A and 8 B molecules of 10-60 spheres, every A-B pair a handle of 16
    trajectories), exact form with adjoint forces: every step of every handle in one
    group launch (one CUDA graph per step, longest systems first), against the same
    handles stepped by their own graphs on their own streams."""
    import torch
    import pbsam_b200 as pb
    from pbsam_b200 import replicas, workload
    cfg = dict(workload.BD_UNEVEN)
    A, B = workload.uneven_molecules(cfg)
    t0 = time.time()
    specs, prep_t, _ = workload.prepare(cfg, device=local, selfpol_rounds=args.selfpol_rounds_p10, mols=A + B)
    prep_t = {"molecules_s": round(time.time() - t0, 1)}
    t0 = time.time()
    ctx, types = workload.open_context(cfg, specs, device=local, exact=1, exact_tol=args.exact_tol)
    prep_t["context_s"] = round(time.time() - t0, 1)
    n = cfg["n_types"]
    stream = torch.cuda.current_stream()

    def handles(streams):
        hs = []
        for i in range(n):
            for j in range(n):
                h = ctx.molecules([types[i], types[n + j]], n_systems=cfg["per_pair"])
                h.set_stream(streams[len(hs)].cuda_stream)
                pcfg = dict(cfg, pose_seed=cfg["pose_seed"] + 64 * i + j)
                pos, quat = workload.bd_start(pcfg, [A[i], B[j]], cfg["per_pair"], rank=rank)
                h.set_poses(pos, quat)
                ext = max(A[i].extent(), B[j].extent())
                dtr, drot = workload.stokes_einstein(ext, cfg["viscosity"], cfg["temperature"])
                h.bd_init([0.0, dtr], [drot, drot], mode=0, seed=97 + 64 * i + j + 4096 * rank,
                          escape_dist=cfg["escape"], dt_min=cfg["dt_min"], dt_max=cfg["dt_max"], dt_ref=0.0,
                          dt_div=cfg["dt_gap"] / (cfg["dt_max"] - cfg["dt_min"]))
                hs.append(h)
        return hs

    def steps_of(hs):
        return int(sum(int(np.sum(h.bd_state()["steps"])) for h in hs))

    out = {}
    timings = {}
    finals = {}
    for mode in ("group", "own"):
        # "own": every handle on a stream of its own, so that their graphs run side by side
        streams = [stream] * (n * n) if mode == "group" else [torch.cuda.Stream() for _ in range(n * n)]
        hs = handles(streams)
        g = pb.Group(hs) if mode == "group" else None
        run = (lambda k: g.bd_run(k)) if mode == "group" else (lambda k: [h.bd_run(k) for h in hs])
        run(args.warmup)
        if g is not None:
            g.tune()
        torch.cuda.synchronize()
        s0 = steps_of(hs)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(gpu_id_for_smi(local)) as clk, torch.cuda.nvtx.range("bd_uneven_" + mode):
            torch.cuda.synchronize()
            e0.record(stream)
            for st in set(streams):
                st.wait_event(e0)
            run(args.bd_steps)
            for st in set(streams):
                stream.wait_stream(st)
            e1.record(stream)
            torch.cuda.synchronize()
        ms = replicas.max_over_ranks(e0.elapsed_time(e1), dist if world > 1 else None)
        units = replicas.sum_over_ranks(steps_of(hs) - s0, dist if world > 1 else None)
        timings[mode] = (units / (ms * 1e-3), ms, clk.summary())
        finals[mode] = [h.bd_state() for h in hs]
        if g is not None:
            g.close()
        for h in hs:
            h.close()
    same = all(np.array_equal(a[k], b[k]) for a, b in zip(finals["group"], finals["own"]) for k in a)
    sizes = [len(m.radii) for m in A + B]
    out = {"metric": "BD steps/s (two-molecule bdnam trajectories, molecules of 10-60 spheres, p=10), exact form "
                     "with adjoint forces, one group launch per step",
           "value": timings["group"][0], "unit": "BD steps/s", "ms_per_step": timings["group"][1] / args.bd_steps,
           "steps": args.bd_steps, "warmup": args.warmup, "dtype": "f64",
           "config": {"workload": "%d trajectories: %d x %d molecule pairs x %d, sphere counts %s (A) and %s (B), "
                                  "300 charges in [-0.6, 0.6] with net +2/-2, start 50 A, escape 150 A; exact_tol %g" % (
                                      n * n * cfg["per_pair"], n, n, cfg["per_pair"], sizes[:n], sizes[n:],
                                      args.exact_tol),
                      "handles": n * n},
           "own_launches": {"value": timings["own"][0], "ms_per_step": timings["own"][1] / args.bd_steps,
                            "note": "each handle's own step graph, every handle on a stream of its own"},
           "vs_own_launches": timings["group"][0] / timings["own"][0],
           "same_trajectories": bool(same),
           "gpu_launches": 3 * args.bd_steps, "clocks": timings["group"][2], "prep": prep_t}
    ctx.close()
    return out


BD_MANY_METRIC = "BD steps/s (bdm: 64 molecules x 30 spheres in a periodic 300 A cube, p=10)"


def run_bd_many(args, local, rank, world, dist, exact=False):
    """BD steps per second of independent many-body systems: 64 molecules of 30
    spheres (32 of each species) in a periodic 300 A cube, the reference bdm's
    multi-molecule dynamics (forces of every molecule whenever two are inside the
    interaction cutoff, then every molecule moved in turn), plain FP64 drop-in or
    (exact) the exact form with adjoint forces.  Every system starts from the same
    configuration with its own noise stream; every step of every system counts as one
    unit."""
    import torch
    from pbsam_b200 import replicas, workload
    cfg = dict(workload.BD_MANY)
    t0 = time.time()
    specs, prep_t, _ = workload.prepare(cfg, device=local, selfpol_rounds=args.selfpol_rounds_p10)
    xkw = {"exact": 1, "exact_tol": args.exact_tol} if exact else {}
    ctx, types = workload.open_context(cfg, specs, device=local, box_length=cfg["box"], **xkw)
    mols = workload.molecules(cfg)
    kinds, pos, quat = workload.many_start(cfg, mols, rank=rank)
    B = args.bd_many_systems
    sysb = ctx.molecules([types[k] for k in kinds], n_systems=B)
    prep_t["total_s"] = round(time.time() - t0, 1)
    stream = torch.cuda.current_stream()
    sysb.set_stream(stream.cuda_stream)
    sysb.set_poses(np.repeat(pos[None], B, 0), np.repeat(quat[None], B, 0))
    n = len(kinds)
    dtr = [cfg["dtr"]] * n
    drot = [cfg["drot"][k] for k in kinds]
    sysb.bd_init(dtr, drot, mode=1, seed=2718 + rank)
    sysb.bd_run(args.warmup)
    torch.cuda.synchronize()
    s0 = sysb.bd_state()
    if world > 1:
        dist.barrier()
    steps = args.bd_many_steps
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(gpu_id_for_smi(local)) as clk, torch.cuda.nvtx.range("bd_many"):
        torch.cuda.synchronize()
        e0.record(stream)
        sysb.bd_run(steps)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    clocks = clk.summary()
    s1 = sysb.bd_state()
    ms_max = replicas.max_over_ranks(ms, dist if world > 1 else None)
    units = int(np.sum(s1["steps"] - s0["steps"]))
    fe = int(np.sum(s1["fevals"] - s0["fevals"]))
    units_all = replicas.sum_over_ranks(units, dist if world > 1 else None)
    st_last = sysb.stats()
    ph = sysb.phase_ms()
    # e2e: one step per call through the public API, the state read back every step
    ee0, ee1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n_e2e = max(1, steps // 2)
    torch.cuda.synchronize()
    ee0.record(stream)
    for _ in range(n_e2e):
        sysb.bd_run(1)
        st = sysb.bd_state()
    ee1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = replicas.max_over_ranks(ee0.elapsed_time(ee1), dist if world > 1 else None)
    e2e_units = replicas.sum_over_ranks(int(np.sum(st["steps"] - s1["steps"])), dist if world > 1 else None)
    d2h = sum(int(v.nbytes) for v in st.values())
    L = cfg["box"]
    d = pos[:, None] - pos[None]
    d -= L * np.round(d / L)
    r = np.linalg.norm(d, axis=2) + np.eye(n) * 1e9
    names = ["solve", "surface", "numeric", "intra", "LS", "DTA", "grad_or_backward", "total"]
    out = {"metric": BD_MANY_METRIC, "value": units_all / (ms_max * 1e-3), "unit": "BD steps/s",
           "ms_per_step": ms_max / steps, "steps": steps, "warmup": args.warmup, "dtype": "f64",
           "config": {"workload": "bdm p=10: %d systems of 64 molecules x 30 spheres (r 3-6 A, 900 charges in "
                                  "[-0.6, 0.6], net +2 x 32 / -2 x 32) in a periodic 300 A cube, random start with "
                                  "a 2 A minimum gap (%d molecule pairs within 100 A), D 0.015 A^2/ps, Dr 4.5e-5 / "
                                  "4e-5 rad^2/ps, bdm time steps, Philox noise per system; plain FP64 form" % (
                                      B, int(np.sum(r < 100) // 2)),
                      "systems_per_gpu": B, "spheres_per_system": int(sum(len(mols[k].radii) for k in kinds))},
           "force_evaluations_fraction": fe / max(units, 1),
           "status_counts": {name: int(np.sum(s1["status"] == k)) for k, name in
                             ((0, "running"), (2, "stuck"), (4, "failed"))},
           "e2e": {"value": e2e_units / (e2e_ms * 1e-3), "unit": "BD steps/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": d2h, "note": "one step per call, state read back to the host each step"},
           "gpu_launches": 3 * steps, "clocks": clocks, "prep": prep_t,
           "mean_phase_ms": {k: round(float(v), 2) for k, v in zip(names, ph[:, :8].mean(axis=0))},
           "mean_sweeps": float(st_last[:, 0].mean()), "mean_inner_solves": float(st_last[:, 2].mean())}
    if exact:
        out["metric"] = BD_MANY_METRIC + ", exact form with adjoint forces"
        out["config"]["workload"] = out["config"]["workload"].replace("plain FP64 form", "exact form, exact_tol %g" %
                                                                      args.exact_tol)
        out["mean_phase_ms"].update({k: round(float(v), 2) for k, v in zip(
            ["backward_energy", "backward_sweeps", "backward_first_round"], ph[:, 12:15].mean(axis=0))})
    if rank == 0 and args.cpu_baseline and not exact:
        out["cpu_baseline"] = bd_many_cpu_baseline(cfg, kinds, pos, quat, args)
    sysb.close()
    ctx.close()
    return out


def bd_many_cpu_baseline(cfg, kinds, pos, quat, args, steps=3):
    """The reference's own bdm (CBDmulti: computeMinSepDist, computeForces below the
    interaction cutoff, makeMove; oracle/ref_bdm_harness.cpp, `fast` build) on the same
    start, one single-threaded process per host core, each with its own drand48 seed,
    all concurrently: steps/s = processes x (steps - 1) / the longest time of the steps
    after the first (the first builds the solver state).  Inputs from the host-side
    preparation (oracle/pbsam_prep.cpp)."""
    import tempfile
    exe = os.path.join(REPO, "oracle", "_ref", "p%d_fast" % cfg["poles"], "bdm_harness")
    if not os.path.exists(exe):
        return {"value": None, "note": "reference bdm harness not built"}
    ncores = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as wd:
        files, _ = reference_inputs_cpu(cfg, args.selfpol_rounds_p10, wd)
        procs = []
        for c in range(ncores):
            spec = os.path.join(wd, "bdm%d.txt" % c)
            with open(spec, "w") as fh:
                fh.write("salt %r\nidiel %r\n" % (cfg["salt"], cfg["idiel"]))
                for fl in files:
                    fh.write("moltype %s %s %s %s\n" % fl)
                fh.write("frame\n")
                for k, p, q in zip(kinds, pos, quat):
                    fh.write("mol %d %s %s\n" % (k, " ".join("%.17g" % v for v in p),
                                                 " ".join("%.17g" % v for v in q)))
                fh.write("bd 1 %d %d 0\nbox %r\n" % (steps, 31 + c, cfg["box"]))
            procs.append((spec, subprocess.Popen([exe, spec, spec + ".out"], env=dict(os.environ, OMP_NUM_THREADS="1"),
                                                 stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)))
        t0 = time.time()
        per = []
        for spec, p in procs:
            try:
                p.wait(timeout=max(1.0, 4 * args.cpu_limit - (time.time() - t0)))
            except subprocess.TimeoutExpired:
                p.kill()
                p.wait()
                continue
            if p.returncode != 0 or not os.path.exists(spec + ".out"):
                continue
            for ln in open(spec + ".out"):
                t = ln.split()
                if t and t[0] == "TIME" and int(t[2]) > 0:
                    per.append((float(t[1]), int(t[2])))
    if not per:
        return {"value": None, "note": "no reference process finished"}
    T = max(x[0] for x in per)
    return {"value": len(per) * per[0][1] / T, "unit": "BD steps/s", "cores": ncores, "kind": "reference",
            "sample": "%d single-threaded processes of the reference's bdm (CBDmulti, p=%d `fast` build), each %d "
                      "steps from the same start with its own seed, run concurrently; steps after the first timed "
                      "(slowest process %.2f s for %d steps)" % (len(per), cfg["poles"], steps, T, per[0][1])}


def reference_bd_step_seconds(cfg, files, pos, quat, limit_s, workdir, steps=3, variant="fast", seed=1):
    """The reference's own bdnam step (CBDnam: computeForces while the pair is inside
    f_DIST, then makeMove; oracle/ref_bd_harness.cpp) from each given pose, one
    single-threaded process per pose, run concurrently; returns the wall seconds per
    step of the steps after the first (the first builds the solver state that a
    running trajectory carries), one value per pose that finished."""
    exe = os.path.join(REPO, "oracle", "_ref", "p%d_%s" % (cfg["poles"], variant), "bd_harness")
    if not os.path.exists(exe):
        return None
    procs = []
    for j in range(len(pos)):
        spec = os.path.join(workdir, "bdref%d.txt" % j)
        _pose_spec(spec, cfg, files, pos[j], quat[j])
        with open(spec, "a") as fh:
            fh.write("bd 0 %d %d 0\n" % (steps, seed + j))
        env = dict(os.environ, OMP_NUM_THREADS="1")
        procs.append((spec, subprocess.Popen([exe, spec, spec + ".out"], env=env, stdout=subprocess.DEVNULL,
                                             stderr=subprocess.DEVNULL)))
    t0 = time.time()
    out = []
    for spec, p in procs:
        try:
            p.wait(timeout=max(1.0, limit_s - (time.time() - t0)))
        except subprocess.TimeoutExpired:
            p.kill()
            p.wait()
            continue
        if p.returncode != 0:
            continue
        for ln in open(spec + ".out"):
            t = ln.split()
            if t and t[0] == "TIME" and int(t[2]) > 0:
                out.append(float(t[1]) / int(t[2]))
    return out


def bd_cpu_baseline(cfg, specs, sysb, state, force_frac, args):
    """The reference's computeForces (p = 10 build) on consecutive poses of sampled
    trajectories: for each, the harness evaluates the pose before the last step
    (untimed, it sets up the carried solver state as in a BD run) and then the pose
    after it (timed), one single-threaded process per trajectory on all host cores.
    BD steps/s = cores / (mean force time x fraction of steps with forces); the
    move itself (a few hundred distance tests) is not counted."""
    from pbsam_b200 import workload
    if not os.path.exists(_ref_harness(cfg["poles"])):
        return {"value": None, "unit": "BD steps/s", "cores": 0, "kind": "reference",
                "sample": "reference binary not built"}
    ncores = os.cpu_count() or 1
    run = [b for b in range(len(state["status"])) if state["status"][b] == 0]
    sel = run[:: max(1, len(run) // ncores)][:ncores]
    with tempfile.TemporaryDirectory() as td:
        files = workload.write_inputs(cfg, specs, td)
        per_step = reference_bd_step_seconds(cfg, files, state["pos"][sel], state["quat"][sel], args.cpu_limit, td)
    if per_step:
        t = float(np.mean(per_step))
        return {"value": ncores / t, "unit": "BD steps/s", "cores": ncores, "kind": "reference",
                "sample": "the reference's own bdnam steps (CBDnam: computeForces + makeMove, `fast` build) from "
                          "the poses of %d trajectories at the end of the timed run, 1 thread per process, all "
                          "concurrently; steps 2-3 of each timed (mean %.3f s per step)" % (len(per_step), t)}
    sysb.bd_run(1)
    after = sysb.bd_state()
    times = []
    with tempfile.TemporaryDirectory() as td:
        files = workload.write_inputs(cfg, specs, td)
        procs = []
        for j in sel:
            spec = os.path.join(td, "bd%d.txt" % j)
            with open(spec, "w") as fh:
                fh.write("salt %r\nidiel %r\ndump 0\nenergy 0\n" % (cfg["salt"], cfg["idiel"]))
                for fl in files:
                    fh.write("moltype %s %s %s %s\n" % fl)
                for s in (state, after):
                    fh.write("frame\n")
                    for m in range(2):
                        fh.write("mol %d %s %s\n" % (m, " ".join("%.17g" % v for v in s["pos"][j, m]),
                                                     " ".join("%.17g" % v for v in s["quat"][j, m])))
            env = dict(os.environ, OMP_NUM_THREADS="1")
            procs.append((spec, subprocess.Popen([_ref_harness(cfg["poles"]), spec, spec + ".out"], env=env,
                                                 stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)))
        import oracle
        t0 = time.time()
        for spec, p in procs:
            try:
                p.wait(timeout=max(1.0, args.cpu_limit - (time.time() - t0)))
            except subprocess.TimeoutExpired:
                p.kill()
                p.wait()
                continue
            if p.returncode == 0:
                fr = oracle.parse(spec + ".out")
                if len(fr) == 2 and fr[1]["ok"]:
                    times.append(float(fr[1]["info"][0]))
    if not times:
        return {"value": None, "unit": "BD steps/s", "cores": ncores, "kind": "reference",
                "sample": "no trajectory finished"}
    t = float(np.mean(times))
    return {"value": ncores / (t * max(force_frac, 1e-9)), "unit": "BD steps/s", "cores": ncores,
            "kind": "reference",
            "sample": "%d trajectories, the force call of one step each (mean %.3f s, 1 thread per process), scaled "
                      "by the fraction of steps with forces (%.3f)" % (len(times), t, force_frac)}


# ---------------------------------------------------------------- reference CPU leg
def _ref_harness(poles):
    return os.path.join(REPO, "oracle", "_ref", "p%d_fast" % poles, "harness")


def _pose_spec(path, cfg, files, pos, quat):
    with open(path, "w") as fh:
        fh.write("salt %r\nidiel %r\ndump 0\nenergy 0\n" % (cfg["salt"], cfg["idiel"]))
        for fl in files:
            fh.write("moltype %s %s %s %s\n" % fl)
        fh.write("frame\n")
        for m in range(len(pos)):
            fh.write("mol %d %s %s\n" % (m, " ".join("%.17g" % v for v in pos[m]),
                                         " ".join("%.17g" % v for v in quat[m])))


def reference_inputs_cpu(cfg, selfpol_rounds, outdir):
    """The sweep's inputs made on the host cores, without the CUDA library: IMats
    (250 000 quadrature points) and self-polarized F/H from the multi-threaded oracle
    preparation (oracle/pbsam_prep.cpp, pinned to the reference's own `pbsam mat` /
    `pbsam spol` files), written in the reference's formats.  Returns the file specs
    and the seconds each part took."""
    import oracle
    from pbsam_b200 import workload
    mols = workload.molecules(cfg)
    specs, tm = [], {}
    for k, m in enumerate(mols):
        cen, rad, pos, q = workload._pqr_round(m)
        t0 = time.time()
        im = oracle.prep_imats(cfg["poles"], cen, rad)
        tm["imat_s_%d" % k] = round(time.time() - t0, 1)
        t0 = time.time()
        F, H, sc, rounds = oracle.prep_selfpol(cfg["poles"], cen, rad, pos, q, im, salt=cfg["salt"],
                                               idiel=cfg["idiel"], max_rounds=selfpol_rounds)
        tm["selfpol_s_%d" % k] = round(time.time() - t0, 1)
        tm["selfpol_sweeps_%d" % k] = rounds
        specs.append(dict(centres=cen, radii=rad, chg_pos=pos, chg=q, imats=im, fself=F, hself=H, hself_scale=sc))
    return workload.write_inputs(cfg, specs, outdir), tm


def reference_throughput(cfg, files, pos, quat, steps, warmup, workdir, variant="fast", limit_s=3000, seed=17):
    """The reference's own computeForces on the sweep's poses, on every host core.

    One single-threaded process of the reference harness (oracle/_ref/p<P>_<variant>,
    the reference compiled from its sources; its OpenMP path races, so one thread per
    process) per core.  Each process builds the molecules once and then evaluates its
    own list of poses in order: `warmup` evaluations of the farthest pose (untimed),
    then `steps` poses, process c taking pose order[(s * C + c) mod n] at step s, where
    order is a seeded permutation of the n sweep poses (every pose recurs equally
    often over the steps).  The harness times each computeForces call; a process's
    busy time is the sum over its timed poses, and the rate is C * steps / (the
    largest busy time): the poses solved per second by all cores together, measured
    without a model."""
    import oracle
    exe = os.path.join(REPO, "oracle", "_ref", "p%d_%s" % (cfg["poles"], variant), "harness")
    if not os.path.exists(exe):
        return None
    ncores = os.cpu_count() or 1
    n = len(pos)
    order = np.random.default_rng(seed).permutation(n)
    far = int(np.argmax(np.linalg.norm(pos[:, 1] - pos[:, 0], axis=1)))
    procs = []
    for c in range(ncores):
        spec = os.path.join(workdir, "ref_core%d.txt" % c)
        seq = [far] * warmup + [int(order[(s * ncores + c) % n]) for s in range(steps)]
        with open(spec, "w") as fh:
            fh.write("salt %r\nidiel %r\ndump 0\nenergy 0\n" % (cfg["salt"], cfg["idiel"]))
            for fl in files:
                fh.write("moltype %s %s %s %s\n" % fl)
            for j in seq:
                fh.write("frame\n")
                for m in range(pos.shape[1]):
                    fh.write("mol %d %s %s\n" % (m, " ".join("%.17g" % v for v in pos[j, m]),
                                                 " ".join("%.17g" % v for v in quat[j, m])))
        env = dict(os.environ, OMP_NUM_THREADS="1")
        procs.append((c, seq, spec, subprocess.Popen([exe, spec, spec + ".out"], env=env, stdout=subprocess.DEVNULL,
                                                     stderr=subprocess.DEVNULL)))
    t0 = time.time()
    busy, solved, failed = [], 0, 0
    for c, seq, spec, p in procs:
        try:
            p.wait(timeout=max(1.0, limit_s - (time.time() - t0)))
        except subprocess.TimeoutExpired:
            p.kill()
            p.wait()
        fr = oracle.parse(spec + ".out") if os.path.exists(spec + ".out") else []
        timed = fr[warmup:]
        if p.returncode != 0 or len(timed) != steps or not all(f["ok"] for f in timed):
            failed += 1
            continue
        busy.append(sum(float(f["info"][0]) for f in timed))
        solved += steps
    wall = time.time() - t0
    if failed or not busy:
        return {"value": None, "failed_processes": failed}
    T = max(busy)
    return {"value": ncores * steps / T, "ms_per_step": 1e3 * T / steps, "cores": ncores, "solved": solved,
            "busy_s_max": round(T, 2), "busy_s_mean": round(float(np.mean(busy)), 2), "wall_s": round(wall, 1),
            "sample": "%d single-threaded processes of the reference harness (p=%d `%s` build), each evaluating "
                      "%d poses of the %d-pose sweep (a seeded permutation taken round-robin over the cores: "
                      "%d solves, every pose about %.1f times) after %d untimed evaluation(s) of the farthest "
                      "pose; rate = cores x poses per process / the largest summed computeForces time" % (
                          ncores, cfg["poles"], variant, steps, n, solved, solved / n, warmup)}


def cpu_baseline(cfg, specs, pos, quat, args):
    """The reference's computeForces on one pose per host core (the bounded sample of
    the timed region), on the inputs the GPU prepared."""
    from pbsam_b200 import workload
    with tempfile.TemporaryDirectory() as td:
        files = workload.write_inputs(cfg, specs, td)
        r = reference_throughput(cfg, files, pos, quat, 1, 0, td)
    if r is None:
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": "reference binary not built"}
    if r["value"] is None:
        return {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                "sample": "a reference process failed"}
    return {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": "reference", "sample": r["sample"],
            "busy_s_max": r["busy_s_max"]}


def run_reference(args):
    """The reference arm: the reference's own CPU implementation of the path, with
    inputs made on the host cores and no CUDA library loaded."""
    from pbsam_b200 import replicas, workload
    rank, world, local = replicas.rank_env()
    if rank != 0:
        return None
    cfg = dict(workload.SWEEP_P30)
    exe = os.path.join(REPO, "oracle", "_ref", "p%d_fast" % cfg["poles"], "harness")
    if not os.path.exists(exe):
        return {"impl": "reference", "unavailable": "reference binary oracle/_ref/p30_fast/harness not built"}
    mols = workload.molecules(cfg)
    pos, quat, _ = workload.poses(cfg, mols)
    with tempfile.TemporaryDirectory() as td:
        t0 = time.time()
        files, prep = reference_inputs_cpu(cfg, args.selfpol_rounds, td)
        prep_s = time.time() - t0
        r = reference_throughput(cfg, files, pos, quat, args.steps, args.warmup, td)
    if r is None or r["value"] is None:
        return {"impl": "reference", "unavailable": "a reference process failed or did not finish"}
    v = r["value"]
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator; IMats and self-polarized "
                                                       "expansions made on the host cores)",
            "config": {"workload": WORKLOAD, "poles": cfg["poles"],
                       "step": "one pose per host core (the sweep's poses round-robin over the cores)"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": r["cores"], "kind": "reference",
                             "sample": r["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "busy_s_max": r["busy_s_max"], "busy_s_mean": r["busy_s_mean"], "timed_wall_s": r["wall_s"],
            "prep_s": round(prep_s, 1), "prep": prep}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    # the reference's spol runs up to 1700 sweeps; on this synthetic geometry at p = 30
    # the sweeps stop contracting after a few rounds, so the inputs are taken after 5
    ap.add_argument("--selfpol-rounds", type=int, default=5)
    ap.add_argument("--cpu-baseline", type=int, default=1)
    ap.add_argument("--cpu-limit", type=int, default=60, help="seconds before a sample pose is abandoned")
    ap.add_argument("--cluster-size", type=int, default=-1,
                    help="CTAs per system (0: automatic, -1: adaptive from the previous step's costs)")
    ap.add_argument("--bd", type=int, default=1, help="also time the Brownian-dynamics workload")
    ap.add_argument("--bd-traj", type=int, default=1024, help="BD trajectories per GPU")
    ap.add_argument("--bd-exact", type=int, default=1,
                    help="also time the BD workload in the exact form with adjoint forces")
    ap.add_argument("--bd-steps", type=int, default=20, help="timed BD steps")
    ap.add_argument("--bd-uneven", type=int, default=1,
                    help="also time BD of molecules with uneven sphere counts (groups of handles)")
    ap.add_argument("--bd-many", type=int, default=1,
                    help="also time many-body bdm dynamics (64 molecules x 30 spheres, periodic 300 A cube)")
    ap.add_argument("--bd-many-systems", type=int, default=148, help="many-body systems per GPU")
    ap.add_argument("--bd-many-steps", type=int, default=6, help="timed many-body BD steps")
    ap.add_argument("--bd-many-exact", type=int, default=0,
                    help="also time the many-body leg in the exact form (about a minute per step at 148 systems)")
    ap.add_argument("--exact-tol", type=float, default=1e-10,
                    help="exact BD leg: pbsam_params.exact_tol (the leg reports the force error against 1e-14)")
    ap.add_argument("--exact-relax", type=float, default=1.0, help="exact BD leg: pbsam_params.exact_relax")
    ap.add_argument("--selfpol-rounds-p10", type=int, default=200)
    ap.add_argument("--poses", default="", help="comma-separated subset of the sweep's poses (small cases)")
    ap.add_argument("--traffic-per-launch", type=float, default=None,
                    help="DRAM bytes per launch measured by ncu (scaled from a small capture)")
    args = ap.parse_args()
    out = run_reference(args) if args.impl == "reference" else run_ours(args)
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
