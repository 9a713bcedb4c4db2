#!/usr/bin/env python
"""Throughput of the B200 DFSPH step on the 1M-particle tilt workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference]

A bench step is one 1/120 s frame of the tilt_1m workload (1,048,576
particles, 128x64x128 lattice in a 1.28 x 0.64 x 1.28 m box, 4,096 tracers,
seeded tilt), advanced the way Renderer::frame does it (render.rs:3021-3229):
substeps_for picks the substeps, each substep runs the tolerance solve (1 %
divergence, 0.1 % density, at most 100 iterations), then reduce_stats and one
tracer pass. The metric counts executed substeps: particle-steps/s.

value: K frames launched back to back on the sim's stream, timed with CUDA
events; the state lives in HBM (working set ~0.5 GB, past the 126 MB L2, so
no flush is needed). e2e: the same frames through the C ABI with a stats
read back to host memory after every frame, wall-clocked. roofline: the
dominant kernel, timed kernel by kernel with CUDA events on the sim's
stream, against the peak (MEASURED_PEAKS.json, else the 6.65 TB/s fallback)
and against a device-to-device copy measured in the same run. cpu_baseline: the CPU oracle on this host's cores over a bounded
sample (one substep of the same state). N > 1: one independent replica per
GPU (a single box does not shard), max over ranks.

batched: the batched-boxes workload (256 boxes, ~5.7M particles) as one
batch per GPU; with N > 1 the boxes are LPT-sharded across the ranks
(strong scaling, no collective in the step), device time max over ranks.
At N = 1 the same boxes are also stepped by the plain step, one Sim per box,
over the batch's first timed substeps (one box at a time, and all boxes on
their own streams at once), for the batch-over-plain ratio.

adjoint: the adjoint workload (65,536 particles, 120 frames): one forward
and one backward of the differentiable model, timed on the device, next to
the production step on the same configuration.

grid: the grid build alone on 16,777,216 positions in 2^24 cells, in three
distributions, timed on the device, against its algorithmic bytes.
"""
import argparse
import ctypes as C
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "fluid-simulation-app_b200")
WORKLOAD = "tilt_1m"
METRIC = "particle-steps/s at 0.1% density error: plain vs batched vs adjoint, 1×B200"
UNIT = "particle-steps/s"
# The batched and adjoint legs run four substeps per 1/120 s frame
# (substeps_for's floor at 5 mm spacing, render.rs:63-65); the plain step
# runs the reference's whole policy, capped at SUBSTEP_CAP.
SUBSTEPS_PER_FRAME = 4
SUBSTEP_CAP = 16

# Algorithmic bytes per particle of each substep kernel: the particle's own
# records it must read and write once (neighbour reads are cache hits in
# cell order and not counted). keys+count 20, reorder 116, density 44,
# divergence kappa 28 / apply 36, forces 84 / 92, density kappa 36 / apply
# 36, integrate 120.
ALGO_BYTES = {"grid": 20.0, "gather": 116.0, "density_div": 44.0, "div_kappa": 28.0,
              "div_apply": 36.0, "forces_eval": 84.0, "forces_den_apply": 92.0,
              "den_kappa": 36.0, "den_apply": 36.0, "integrate": 120.0}
# DRAM bytes (read + write) per particle per launch: a constant taken from
# one ncu capture of each kernel on this workload at its full 1,048,576
# particles, on the state after the benchmark's 25 frames
# (dram__bytes_read.sum + dram__bytes_write.sum), not measured by this
# script; a kernel change calls for a new capture.
NCU_TRAFFIC_PER_PARTICLE = {"density_div": (106.80e6 + 318.62e6) / 1048576,
                            "forces_eval": (410.57e6 + 38.01e6) / 1048576,
                            "den_kappa": (406.19e6 + 15.34e6) / 1048576}


# What holds each leading kernel back, from the same ncu capture: none of
# them is DRAM-bound, so their fraction of the HBM roofline stays low.
NCU_LIMITER = {
    "density_div": "SM issue and L1 (ncu: 65 % SM throughput, 68 % issue active, 65 % L1 "
                   "wavefronts, 43 % warps active; ~194 candidate tests and ~33 hits a particle)",
    "forces_eval": "SM issue (ncu: 72 % SM throughput, 76 % issue active; ten IEEE divisions "
                   "and a square root per pair)",
    "den_kappa": "L1 data pipe (ncu: 80 % L1 wavefronts; neighbour records gathered through L1)",
}


def workload_config(w, n):
    """The workload both arms run, as the JSON line's `config`."""
    return {"workload": WORKLOAD, "particles": n, "lattice": "x".join(str(v) for v in w["lattice"]),
            "box_m": "x".join(str(v) for v in w["box_hi"]), "spacing_m": w["spacing"], "h_ratio": 1.2,
            "tracers": w["tracers"], "frame_dt_s": float(np.float32(1.0 / 120.0)),
            "step": "one 1/120 s frame: the policy's DFSPH substeps, reduce_stats, one tracer "
                    "pass; the metric counts substeps",
            "substeps_per_frame": "substeps_for on the one-frame-stale v_max (render.rs:3090-3094), cap 16",
            "solve": "tolerance div 1% / den 0.1%, cap 100, FP64 residuals",
            "tilt": "seed 1, three sinusoids per axis, <= 35 degrees, 0.2-2 Hz",
            "l2": "working set > 126 MB L2; no flush"}


def load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def copy_gbs(device):
    """STREAM-style copy on this GPU, measured beside the kernels it judges:
    bytes read + written per second (GB/s) over ten 2 GiB device-to-device
    copies, after three untimed ones, CUDA events on the current stream."""
    import torch

    src = torch.ones(1 << 29, dtype=torch.float32, device=device)
    dst = torch.empty_like(src)
    for _ in range(3):
        dst.copy_(src)
    torch.cuda.synchronize(device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    reps = 10
    e0.record()
    for _ in range(reps):
        dst.copy_(src)
    e1.record()
    e1.synchronize()
    gbs = 2.0 * src.numel() * src.element_size() * reps / (e0.elapsed_time(e1) / 1e3) / 1e9
    del src, dst
    torch.cuda.empty_cache()
    return gbs


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons while timing."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms",
                 "100", "-i", str(self.device)], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cuda_arm(args):
    import torch

    world, rank, local = dist_init()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    fcu = load("fluidcu", os.path.join(PKG, "fluidcu.py"))
    wl = load("workloads", os.path.join(PKG, "workloads.py"))
    w = wl.WORKLOADS[WORKLOAD]
    frames = args.warmup + args.steps
    forces = wl.tilt_schedule(1, frames, 1.0 / 120.0)
    dt = float(np.float32(1.0 / 120.0))

    # Substeps per frame: the reference's policy, substeps_for on the
    # one-frame-stale v_max with a cap of 16 (render.rs:57-106, :3090-3094),
    # which fluid_sim_frame applies when given no count. Each frame is
    # followed by a sync, so the stale v_max is exactly the previous frame's
    # in the device-timed loop as in the end-to-end loop and the reference
    # arm, and all three execute the same substeps on the same states.
    def frame(sim, k):
        f = forces[k]
        sim.frame((float(f[0]), float(f[1]), float(f[2])), dt, substeps=0, cap=SUBSTEP_CAP, seed=k)
        sim.sync()

    cfg = wl.make_config(fcu, WORKLOAD, device=local)
    sim = fcu.Sim(cfg)
    stream = torch.cuda.ExternalStream(sim.stream())
    for k in range(args.warmup):
        frame(sim, k)
    sim.sync()
    if args.profile_substeps:
        return profile_only(args, fcu, wl, sim, forces, dt / SUBSTEPS_PER_FRAME, w)
    before = sim.stats()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clocks:
        e0.record(stream)
        for k in range(args.warmup, frames):
            frame(sim, k)
        e1.record(stream)
        e1.synchronize()
    ms = e0.elapsed_time(e1)
    sim.sync()
    after = sim.stats()
    substeps = int(after.substeps - before.substeps)
    div_it = int(after.total_div_iters - before.total_div_iters)
    den_it = int(after.total_den_iters - before.total_den_iters)
    n = sim.n
    if world > 1:
        t = torch.tensor([ms, substeps], dtype=torch.float64, device="cuda")
        tmax = t.clone()
        torch.distributed.all_reduce(tmax[:1], op=torch.distributed.ReduceOp.MAX)
        tot = t.clone()
        torch.distributed.all_reduce(tot[1:], op=torch.distributed.ReduceOp.SUM)
        ms_max, all_substeps = float(tmax[0]), float(tot[1])
    else:
        ms_max, all_substeps = ms, float(substeps)
    value = n * all_substeps / (ms_max / 1000.0)

    # kernel launches inside the timed region: per substep the grid build
    # (keys, one per digit pass, starts scan), gather, density_div and its residual
    # step, forces pair, first density prediction and its residual step,
    # integrate; 3 per loop iteration; per frame stats (2) and tracers (3).
    passes = 1
    cells = sim.keyspace
    while (cells - 1) >> (8 * passes):
        passes += 1
    fixed = 2 + passes + 1 + 2 + 4 + 1
    launches = fixed * substeps + 3 * (div_it + den_it) + 5 * args.steps

    # e2e: a fresh replica, frames through the C ABI with a stats read back
    # to host memory after every frame (the frame's result), wall-clocked.
    # Per frame: the substeps' Step blocks up (160 B each), the stale-stats
    # copy, the statistics and the solver counters down (64 B each).
    if args.no_e2e:
        return finish_without_e2e(args, sim, value, ms_max, substeps, launches, clocks, world, rank)
    sim_e = fcu.Sim(wl.make_config(fcu, WORKLOAD, device=local))
    for k in range(args.warmup):
        frame(sim_e, k)
        sim_e.stats()
    if world > 1:
        torch.distributed.barrier()
    sb = sim_e.stats()
    t0 = time.perf_counter()
    for k in range(args.warmup, frames):
        frame(sim_e, k)
        sim_e.stats()
    t1 = time.perf_counter()
    se = sim_e.stats()
    e2e_sub = int(se.substeps - sb.substeps)
    e2e_s = t1 - t0
    if world > 1:
        t = torch.tensor([e2e_s, e2e_sub], dtype=torch.float64, device="cuda")
        tm = t.clone()
        torch.distributed.all_reduce(tm[:1], op=torch.distributed.ReduceOp.MAX)
        ts = t.clone()
        torch.distributed.all_reduce(ts[1:], op=torch.distributed.ReduceOp.SUM)
        e2e_s, e2e_all = float(tm[0]), float(ts[1])
    else:
        e2e_all = float(e2e_sub)
    e2e_value = n * e2e_all / e2e_s
    sim_e.close()

    # The same frames at a fixed four substeps (substeps_for's floor at 5 mm,
    # render.rs:63-65) on a fresh replica, device-timed without syncs: the
    # CFL clamp then catches the fast particles instead of more substeps.
    fixed = fixed_four_leg(args, fcu, wl, forces, dt, local) if not args.no_fixed else None

    # roofline: per-kernel CUDA-event times of a few substeps of this state
    prof = {}
    per_frame = max(1, int(round(substeps / args.steps)))
    for k in range(8):
        f = forces[(frames + k) % len(forces)]
        dts = float(np.float32(dt) / np.float32(per_frame))
        st = fcu.make_step(force=tuple(float(x) for x in f), dt=dts, v_clamp=wl.v_clamp(w["spacing"], dts))
        for name, t in sim.profile_step(st):
            prof.setdefault(name, []).append(t)
    # Each kernel's share of a timed substep: its mean duration times the
    # launches a substep of the timed run made (the tolerance loops' mean
    # iteration counts, not the profile's fixed schedule).
    mean = {k: sum(v) / len(v) for k, v in prof.items()}
    md, mk = div_it / max(substeps, 1), den_it / max(substeps, 1)
    # In the tolerance schedule density_div forms the first divergence
    # prediction and forces_eval, run after each divergence apply, forms the
    # next ones (no div_kappa sweep): forces_eval runs md times a substep.
    per_substep = {"grid": 1.0, "gather": 1.0, "density_div": 1.0, "div_apply": md,
                   "forces_eval": max(md, 1.0), "forces_den_apply": 1.0, "den_kappa": 1.0 + mk,
                   "den_apply": mk, "integrate": 1.0}
    share = {k: mean[k] * per_substep[k] for k in mean if k in per_substep}
    dom = max(share, key=lambda k: share[k])
    avg_ms = mean[dom]
    achieved = ALGO_BYTES[dom] * n / (avg_ms / 1000.0) / 1e9
    peak, peak_kind = peaks()
    copy_peak = copy_gbs(local)
    traffic = NCU_TRAFFIC_PER_PARTICLE.get(dom)

    # the CPU oracle on this host over one substep of the same state
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_sample(fcu, sim, dt, per_frame)

    # the neighbour list the sweeps stream: 8 bytes per entry
    mean_nbrs = float(np.mean(sim.field("nbr_n").astype(np.float64)))
    list_bytes = 8.0 * mean_nbrs
    sim.close()
    batched = None if args.no_batched else batched_leg(args, fcu, wl, world, rank, local, value / world)
    adjoint = None if args.no_adjoint else adjoint_leg(args, fcu, wl, world, local)
    grid = None if args.no_grid else grid_leg(fcu, wl, local, peak, copy_peak)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(w, n),
            "particle_frames_per_s": n * world * args.steps / (ms_max / 1000.0),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 160 * e2e_sub / args.steps,
                    "d2h_bytes_per_step": 64 + 64 + 64},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None if traffic is None else traffic * n,
                         "traffic_source": "constant from one ncu capture of this kernel on this "
                                           "workload (dram__bytes_read.sum + dram__bytes_write.sum), "
                                           "not measured in this run",
                         "peak_source": f"{peak_kind} MEASURED_PEAKS.json hbm_gbs" if peak_kind == "measured" else "fallback 6.65 TB/s",
                         "algorithmic": f"own records, list-free ({ALGO_BYTES[dom]:.0f} B per particle for {dom})",
                         "limiter": NCU_LIMITER.get(dom),
                         "mean_neighbours": mean_nbrs,
                         "achieved_with_list": (ALGO_BYTES[dom] + list_bytes) * n / (avg_ms / 1000.0) / 1e9,
                         "frac_with_list": (ALGO_BYTES[dom] + list_bytes) * n / (avg_ms / 1000.0) / 1e9 / peak,
                         "copy_gbs_measured_here": copy_peak,
                         "frac_of_copy_measured_here": achieved / copy_peak,
                         "kernel_ms": mean,
                         "ms_per_substep_by_kernel": share},
            "cpu_baseline": cpu,
            "clocks": clocks.summary(),
            "gpu_launches": launches,
            "fixed_four_substeps": fixed,
            "batched": batched,
            "adjoint": adjoint,
            "grid": grid,
            # last, so that the end of the line shows them
            "solve": {"substeps": substeps, "mean_div_iters": div_it / max(substeps, 1),
                      "mean_den_iters": den_it / max(substeps, 1),
                      "parallelism": f"replicas x{world}" if world > 1 else "single box"},
            # the last timed frame's statistics (reduce_stats runs every frame)
            "density_error": {"compression_avg": after.compression_avg,
                              "compression_max": after.compression_max,
                              "den_residual_last": after.den_residual,
                              "clamps_per_particle_substep": (after.clamp_count - before.clamp_count)
                              / float(n * max(substeps, 1))},
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


BATCH_WARMUP_FRAMES = 10
BATCH_FRAMES = 30


def batched_leg(args, fcu, wl, world, rank, local, plain_per_gpu):
    """The batched workload: 256 boxes of 4,096..65,536 particles (log-
    uniform, about 5.7M in all), each with its own tilt sequence and XSPH
    coefficient, tolerance solve. The boxes share one substep clock: each
    1/120 s frame runs the most substeps the reference's policy asks for
    any box (substeps_for on that box's one-frame-stale v_max, cap 16), all
    boxes at that frame's dt. Each rank steps its LPT shard of the boxes as
    one batch (no collective in the step); device time on the batch's
    stream, max over ranks; per-box statistics are summed across ranks at
    the end."""
    import torch
    sharding = load("sharding", os.path.join(PKG, "sharding.py"))
    cfgs_all = wl.batched_boxes(fcu, nboxes=args.boxes)
    counts = [c.block[0] * c.block[1] * c.block[2] for c in cfgs_all]
    mine = sharding.lpt_shards(counts, world)[rank]
    cfgs = [cfgs_all[b] for b in mine]
    for c in cfgs:
        c.device = local
    batch = fcu.Batch(cfgs)
    frames = BATCH_WARMUP_FRAMES + BATCH_FRAMES
    dt = float(np.float32(1.0 / 120.0))
    forces = [wl.tilt_schedule(3 * 100003 + b, frames, 1.0 / 120.0) for b in mine]
    v_max = [0.0] * len(mine)
    recorded = []

    def frame_steps(k):
        n = max(fcu.substeps_for(dt, v, wl.BATCH_SPACING, SUBSTEP_CAP) for v in v_max)
        dts = float(np.float32(dt) / np.float32(n))
        vc = wl.v_clamp(wl.BATCH_SPACING, dts)
        row = [fcu.make_step(force=tuple(float(x) for x in forces[q][k]), dt=dts, v_clamp=vc, seed=k)
               for q in range(len(mine))]
        return [row] * n

    def frame(k):
        steps = frame_steps(k)
        batch.run(steps)
        batch.reduce_stats()
        v_max[:] = [st.v_max for st in batch.stats()]  # synchronises: the next frame's stale v_max
        recorded.extend(steps)
        return len(steps)

    for k in range(BATCH_WARMUP_FRAMES):
        frame(k)
    nw = len(recorded)
    # block sizes from the autotuner (one timed substep per candidate on the
    # warmed-up state, which it restores)
    chosen, tune_ms = batch.autotune(frame_steps(BATCH_WARMUP_FRAMES)[0])
    before = batch.stats()
    stream = torch.cuda.ExternalStream(batch.stream())
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sub = sum(frame(k) for k in range(BATCH_WARMUP_FRAMES, frames))
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    after = batch.stats()
    local_rows = [[a.total_den_iters - b.total_den_iters, a.total_div_iters - b.total_div_iters,
                   a.compression_avg, a.compression_max, a.clamp_count - b.clamp_count]
                  for a, b in zip(after, before)]
    rows = sharding.gather_box_values(mine, local_rows, len(cfgs_all),
                                      device="cuda" if world > 1 else "cpu")
    work = float(sum(counts[b] for b in mine) * sub)  # particle-substeps of this rank
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t[0])
        wt = torch.tensor([work], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(wt, op=torch.distributed.ReduceOp.SUM)
        work = float(wt[0])
    total = int(sum(counts))
    value = work / (ms / 1000.0)
    batch.close()
    plain_boxes = None
    if world == 1 and not args.no_plain_boxes:
        plain_boxes = plain_boxes_leg(fcu, cfgs, recorded, nw, value)
    per_box_substeps = work / total
    return {"workload": "batched_256", "boxes": len(cfgs_all), "particles": total,
            "frames": BATCH_FRAMES, "substeps": sub, "substeps_per_frame": sub / BATCH_FRAMES,
            "warmup_substeps": nw, "ms_per_substep": ms / sub, "ms_per_frame": ms / BATCH_FRAMES,
            "value": value, "unit": UNIT,
            "step": "substeps_for on each box's one-frame-stale v_max, the most any box asks for, cap 16",
            "sharding": f"LPT over {world} rank(s)" if world > 1 else "one batch",
            "scaling": "strong",
            "mean_den_iters_per_box": float(rows[:, 0].mean() / per_box_substeps),
            "mean_div_iters_per_box": float(rows[:, 1].mean() / per_box_substeps),
            "compression_avg_mean": float(rows[:, 2].mean()),
            "compression_avg_worst_box": float(rows[:, 2].max()),
            "clamps_per_particle_substep": float(rows[:, 4].sum() / work),
            "vs_plain_tilt_1m_per_gpu": value / world / plain_per_gpu if plain_per_gpu else None,
            "vs_the_same_boxes_as_plain_sims": plain_boxes,
            "autotuned_blocks": chosen,
            "autotune_ms_by_block": {str(t): dict(zip(fcu.Batch.TUNED, [round(float(x), 4) for x in tune_ms[c]]))
                                     for c, t in enumerate((64, 128, 256))}}


PLAIN_BOX_SUBSTEPS = 12


def plain_boxes_leg(fcu, cfgs, steps, nw, batch_value):
    """The batched workload's boxes stepped by the plain step: one Sim per
    box (fluid_sim_*), warmed up over the same substeps as the batch, then
    the batch's first PLAIN_BOX_SUBSTEPS timed substeps, (a) one box after
    another, each box's substeps then a device sync, and (b) every box's
    substeps enqueued on its own stream, then one sync. Wall clock around
    device syncs (the work spans 256 streams). Same Step blocks and the same
    per-box results (each box bit-identical to the batch's); compared with
    the batch's rate over its timed frames."""
    import torch
    sims = [fcu.Sim(c) for c in cfgs]
    try:
        counts = [s.n for s in sims]
        for b, s in enumerate(sims):
            s.run([row[b] for row in steps[:nw]])
        torch.cuda.synchronize()
        timed = steps[nw:nw + PLAIN_BOX_SUBSTEPS]
        t0 = time.perf_counter()
        for b, s in enumerate(sims):
            s.run([row[b] for row in timed])
            s.sync()
        t1 = time.perf_counter()
        for b, s in enumerate(sims):
            s.run([row[b] for row in timed])
        torch.cuda.synchronize()
        t2 = time.perf_counter()
    finally:
        for s in sims:
            s.close()
    work = sum(counts) * len(timed)
    one_by_one, concurrent = work / (t1 - t0), work / (t2 - t1)
    return {"substeps": len(timed), "batch": batch_value,
            "one_box_at_a_time": one_by_one, "all_boxes_on_own_streams": concurrent,
            "batch_over_one_at_a_time": batch_value / one_by_one,
            "batch_over_concurrent": batch_value / concurrent}


ADJ_FRAMES = 120
ADJ_CHECKPOINT = 10


GRID_SIDE = 256
GRID_BUILDS = 10


def grid_leg(fcu, wl, local, peak, copy_peak):
    """The grid workload: 16,777,216 positions in a 256^3-cell box (cell 1),
    in the three seeded distributions (uniform; 90 % packed into the lowest
    tenth; eight Gaussian clusters of sigma 4 cells), each built into
    starts[C+1] and the stable permutation by fluid_grid_build. Three
    untimed builds, then ten timed on the device with CUDA events. The
    positions (268 MB) exceed L2, so no flush. Algorithmic bytes per build:
    positions 16 + key 4 + 4 (written, read back) + permutation 4 per
    position, 8 per cell for the counts and starts."""
    import torch
    dev = torch.device("cuda", local)
    n, side = 1 << 24, GRID_SIDE
    cells = side ** 3
    g = fcu.FluidGrid()
    g.min[:] = [0.0, 0.0, 0.0]
    g.cell = 1.0
    g.dims[:] = [side, side, side]
    ws_bytes = fcu.grid_workspace_bytes(n, g)
    ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
    starts = torch.empty(cells + 1, dtype=torch.int32, device=dev)
    perm = torch.empty(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    algo = 36.0 * n + 8.0 * cells
    out = {"workload": "grid_16m", "positions": n, "cells": cells,
           "algorithmic_bytes_per_build": algo, "builds_timed": GRID_BUILDS}
    for kind, seed in (("uniform", 1), ("packed", 2), ("gaussian", 3)):
        pos = torch.from_numpy(wl.grid_positions(kind, n, side, seed)).to(dev)

        def build():
            fcu.grid_build_device(pos.data_ptr(), n, g, 0, starts.data_ptr(), perm.data_ptr(),
                                  ws.data_ptr(), ws_bytes, stream.cuda_stream)

        for _ in range(3):
            build()
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(GRID_BUILDS):
            build()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / GRID_BUILDS
        gbs = algo / (ms / 1e3) / 1e9
        out[kind] = {"ms_per_build": ms, "positions_per_s": n / (ms / 1e3),
                     "achieved_gbs": gbs, "frac": gbs / peak,
                     "frac_of_copy_measured_here": gbs / copy_peak}
        del pos
    del ws, starts, perm
    torch.cuda.empty_cache()
    return out


def adjoint_leg(args, fcu, wl, world, local):
    """The adjoint workload: 65,536 particles (64x16x64 block), 120 frames of
    4 substeps, loss on the final centre of mass and density deviation,
    gradients with respect to the 120x3 force sequence and the XSPH
    coefficient, checkpoints every 10 frames. FP32. The first forward
    decides and freezes the iteration counts (not timed); then one forward
    and one backward are timed on the device. The production step on the
    same configuration, 480 substeps in tolerance mode, is timed beside it."""
    import torch
    cfg = wl.make_config(fcu, "adjoint_64k", device=local)
    dt = float(np.float32(1.0 / 120.0))
    dts = float(np.float32(dt) / np.float32(SUBSTEPS_PER_FRAME))
    vc = wl.v_clamp(0.005, dts)
    forces = wl.tilt_schedule(2, ADJ_FRAMES, 1.0 / 120.0).astype(np.float64)
    target = np.array([0.64, 0.05, 0.64])
    adj = fcu.Adjoint(cfg, ADJ_FRAMES, SUBSTEPS_PER_FRAME, dt, vc, ADJ_CHECKPOINT, precision=32)
    adj.forward(forces, 0.01, target)
    div_it, den_it = adj.schedule()
    loss = adj.forward(forces, 0.01, target)
    fwd_ms, _ = adj.timing()
    g, gx = adj.backward()
    _, bwd_ms = adj.timing()
    n = adj.n
    # the same forward and backward in FP64 on the same frozen schedule: its
    # gradient stays finite over the whole horizon where FP32 overflows
    a64 = fcu.Adjoint(cfg, ADJ_FRAMES, SUBSTEPS_PER_FRAME, dt, vc, ADJ_CHECKPOINT, precision=64)
    a64.set_schedule(div_it, den_it)
    loss64 = a64.forward(forces, 0.01, target)
    g64, gx64 = a64.backward()
    f64_ms, b64_ms = a64.timing()
    a64.close()
    gv64 = np.concatenate([g64.ravel(), [gx64]])
    adj.close()
    # the production step on the same box, same substeps
    sim = fcu.Sim(cfg)
    steps = [fcu.make_step(force=tuple(float(v) for v in forces[k // SUBSTEPS_PER_FRAME]), dt=dts,
                           v_clamp=vc, seed=k) for k in range(ADJ_FRAMES * SUBSTEPS_PER_FRAME)]
    sim.run(steps[:40])
    sim.sync()
    stream = torch.cuda.ExternalStream(sim.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.run(steps)
    e1.record(stream)
    e1.synchronize()
    prod_ms = e0.elapsed_time(e1)
    sim.close()
    sub = ADJ_FRAMES * SUBSTEPS_PER_FRAME
    gv = np.concatenate([g.ravel(), [gx]])
    return {"workload": "adjoint_64k", "particles": n, "frames": ADJ_FRAMES, "substeps": sub,
            "checkpoint_every_frames": ADJ_CHECKPOINT, "precision": "f32", "loss": loss,
            "forward_ms": fwd_ms, "backward_ms": bwd_ms,
            "value": n * sub / ((fwd_ms + bwd_ms) / 1000.0), "unit": UNIT,
            "backward_over_model_forward": bwd_ms / fwd_ms,
            "production_forward_ms": prod_ms,
            "backward_over_production_forward": bwd_ms / prod_ms,
            "mean_div_iters": float(div_it.mean()), "mean_den_iters": float(den_it.mean()),
            "grad_norm": float(np.linalg.norm(gv)) if np.all(np.isfinite(gv)) else None,
            "fp64": {"loss": loss64, "forward_ms": f64_ms, "backward_ms": b64_ms,
                     "grad_norm": float(np.linalg.norm(gv64)) if np.all(np.isfinite(gv64)) else None,
                     "grad_xsph": float(gx64)},
            "grad_note": "sensitivities grow exponentially with the horizon on this splashing "
                         "workload; the gradient is checked against FP64 central differences "
                         "on short horizons (tests/test_gpu_adjoint.py)"}


def profile_only(args, fcu, wl, sim, forces, dt_sub, w):
    """Substeps as direct kernel launches (visible to ncu), timed per kernel."""
    prof = {}
    vc = wl.v_clamp(w["spacing"], dt_sub)
    for k in range(args.profile_substeps):
        f = forces[k % len(forces)]
        st = fcu.make_step(force=tuple(float(x) for x in f), dt=dt_sub, v_clamp=vc)
        for name, t in sim.profile_step(st):
            prof.setdefault(name, []).append(t)
    sim.sync()
    sim.close()
    print(json.dumps({"profile_substeps": args.profile_substeps, "particles": int(sim.n),
                      "kernel_ms": {k: sum(v) / len(v) for k, v in prof.items()},
                      "launches": {k: len(v) for k, v in prof.items()}}), flush=True)


def finish_without_e2e(args, sim, value, ms_max, substeps, launches, clocks, world, rank):
    sim.close()
    if rank == 0:
        print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                          "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": ms_max / args.steps, "substeps": substeps,
                          "gpu_launches": launches, "clocks": clocks.summary(),
                          "note": "profiling run: no e2e, roofline or cpu baseline"}), flush=True)
    if world > 1:
        import torch
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def fixed_four_leg(args, fcu, wl, forces, dt, local):
    import torch
    sim = fcu.Sim(wl.make_config(fcu, WORKLOAD, device=local))

    def frame(k):
        f = forces[k]
        sim.frame((float(f[0]), float(f[1]), float(f[2])), dt, substeps=SUBSTEPS_PER_FRAME, cap=16, seed=k)

    for k in range(args.warmup):
        frame(k)
    sim.sync()
    b = sim.stats()
    stream = torch.cuda.ExternalStream(sim.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(args.warmup, args.warmup + args.steps):
        frame(k)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    a = sim.stats()
    sub = int(a.substeps - b.substeps)
    out = {"substeps_per_frame": SUBSTEPS_PER_FRAME, "value": sim.n * sub / (ms / 1000.0), "unit": UNIT,
           "ms_per_frame": ms / args.steps,
           "mean_den_iters": (a.total_den_iters - b.total_den_iters) / max(sub, 1),
           "clamps_per_particle_substep": (a.clamp_count - b.clamp_count) / float(sim.n * max(sub, 1)),
           "compression_avg": a.compression_avg}
    sim.close()
    return out


def cpu_sample(fcu, sim, dt, per_frame):
    """The oracle over one substep of the GPU's current state, all cores."""
    sys.path.insert(0, ROOT)
    from oracle import oracle as orc

    p = orc.OrParams()
    for name, _ in orc.OrParams._fields_:
        v = getattr(sim.params, name)
        if hasattr(v, "__len__"):
            getattr(p, name)[:] = list(v)
        else:
            setattr(p, name, v)
    o = orc.Sim(p, 0)
    st = sim.state()
    o.set_state(st["pos"], st["vel"], st["prev_vel"], st["prev_p"], st["temp"], st["id"])
    dts = float(np.float32(dt) / np.float32(per_frame))
    step = orc.make_step(force=(0.0, -9.81, 0.0), dt=dts,
                         v_clamp=float(np.float32(0.4) * np.float32(0.005) / np.float32(dts)))
    t0 = time.perf_counter()
    iters, _ = o.substep_tol(step, 0.01, 0.001, 100)
    t = time.perf_counter() - t0
    return {"value": sim.n / t, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": f"one substep of {sim.n} particles from the benchmark state "
                      f"({int(iters[0])} div + {int(iters[1])} den iterations), {t:.1f} s"}


def reference_arm(args):
    """The reference implementation on the host: the CPU oracle (this
    project's restatement of the reference's WGSL step, which exists only as
    shaders) on the same workload, the same frames and the same count as the
    CUDA arm: tilt_1m's 1,048,576-particle lattice and 4,096 tracers seeded
    as fluid_sim_create seeds them, `warmup` untimed frames, then `steps`
    timed frames, each the substeps the reference's policy picks from the
    one-frame-stale v_max (tolerance solves), reduce_stats and a tracer pass,
    with the same seeded tilt. All host threads (OpenMP)."""
    world, rank, local = dist_init()
    if rank != 0:
        return
    sys.path.insert(0, ROOT)
    from oracle import oracle as orc
    wl = load("workloads", os.path.join(PKG, "workloads.py"))
    w = wl.WORKLOADS[WORKLOAD]
    lattice, spacing = list(w["lattice"]), w["spacing"]
    pos = orc.seed_block([0, 0, 0], spacing, lattice, 0.005, 1)
    n = len(pos)
    p = orc.params_box([0, 0, 0], list(w["box_hi"]), spacing, 1.2, 1000.0, n)
    p.xsph_blend = 0.01
    o = orc.Sim(p, w["tracers"])
    o.set_state(pos4=pos)
    size = [float(np.float32(x) * np.float32(spacing)) for x in lattice]
    o.set_tracers(orc.seed_tracers_box(w["tracers"], [0, 0, 0], size, p))
    frames = args.warmup + args.steps
    forces = wl.tilt_schedule(1, frames, 1.0 / 120.0)
    dt = float(np.float32(1.0 / 120.0))
    iters = np.zeros(3, np.int64)  # divergence, density iterations, substeps
    v_max = [0.0]

    def frame(k):
        # the reference's policy on the one-frame-stale v_max (render.rs:3090-3094)
        f = tuple(float(x) for x in forces[k])
        m = orc.substeps_for(dt, v_max[0], spacing, SUBSTEP_CAP)
        dts = float(np.float32(dt) / np.float32(m))
        vc = float(np.float32(0.4) * np.float32(spacing) / np.float32(dts))
        st = orc.make_step(force=f, dt=dts, v_clamp=vc)
        for _ in range(m):
            it, _ = o.substep_tol(st, 0.01, 0.001, 100)
            iters[:2] += it
        iters[2] += m
        v_max[0] = float(o.stats()[6])
        o.tracer_pass(orc.make_step(force=f, dt=dt, seed=k))

    for k in range(args.warmup):
        frame(k)
    iters[:] = 0
    t0 = time.perf_counter()
    for k in range(args.warmup, frames):
        frame(k)
    t = time.perf_counter() - t0
    final = o.stats()
    substeps = int(iters[2])
    value = n * substeps / t
    cores = os.cpu_count()
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * t / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "impl": "reference",
        "config": workload_config(w, n),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"the whole workload: {args.steps} frames of {n} particles "
                                   f"({substeps} substeps) after {args.warmup} warm-up frames, "
                                   f"OpenMP over {cores} threads, {t:.1f} s"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "solve": {"substeps": substeps, "mean_div_iters": float(iters[0]) / substeps,
                  "mean_den_iters": float(iters[1]) / substeps},
        "density_error": {"compression_avg": float(final[0]), "compression_max": float(final[1])},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    # 20 timed frames after 5 warm-up frames: the CUDA arm's timed region is
    # then ~0.65 s and the reference arm (the oracle on the same frames) ~4 min.
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["cuda", "reference"], default="cuda")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="time the device loop only (profiling runs)")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-boxes leg")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint leg")
    ap.add_argument("--no-grid", action="store_true", help="skip the 16.7M-position grid leg")
    ap.add_argument("--no-fixed", action="store_true", help="skip the fixed-four-substep frames")
    ap.add_argument("--no-plain-boxes", action="store_true",
                    help="skip stepping the batched boxes as separate plain sims")
    ap.add_argument("--profile-substeps", type=int, default=0,
                    help="after the warm-up, run this many substeps as direct launches timed per kernel, then exit")
    ap.add_argument("--boxes", type=int, default=256,
                    help="boxes of the batched leg (256: the batched workload; fewer for profiling runs)")
    ap.add_argument("--batch-only", action="store_true",
                    help="run the batched leg alone and print it (profiling runs)")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="run the adjoint leg alone and print it (profiling runs)")
    ap.add_argument("--grid-only", action="store_true",
                    help="run the 16.7M-position grid leg alone and print it (profiling runs)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")
    if args.batch_only or args.adjoint_only:
        import torch
        torch.cuda.set_device(0)
        fcu = load("fluidcu", os.path.join(PKG, "fluidcu.py"))
        wl = load("workloads", os.path.join(PKG, "workloads.py"))
        if args.batch_only:
            print(json.dumps(batched_leg(args, fcu, wl, 1, 0, 0, None)), flush=True)
        else:
            print(json.dumps(adjoint_leg(args, fcu, wl, 1, 0)), flush=True)
    elif args.grid_only:
        import torch
        torch.cuda.set_device(0)
        fcu = load("fluidcu", os.path.join(PKG, "fluidcu.py"))
        wl = load("workloads", os.path.join(PKG, "workloads.py"))
        print(json.dumps(grid_leg(fcu, wl, 0, peaks()[0], copy_gbs(0))), flush=True)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        cuda_arm(args)


if __name__ == "__main__":
    main()
