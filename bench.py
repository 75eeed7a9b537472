#!/usr/bin/env python
"""Benchmark of the coarse-grid field step (air + Newtonian gravity) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload 1|2|4|5] [--ticks T]   (workloads C1, C2, C4, C5)
    python bench.py --voxel3d [--worlds W] ...   (the 3-D sandbox's field step)
    python bench.py --save-io                    (the .tptrs save codec, host only)

Metric: cell-ticks/s = sum over instances of xcells*ycells * ticks / time;
one tick is one air step plus one gravity solve of every instance (the
reference re-solves gravity every tick). One bench "step" is one pass of the
workload's tick count (1000 ticks for the batched workloads) over all its
instances. Inputs are seeded synthetic sandboxes with the workloads' shapes
(the reference publishes no dataset): see workloads.py.

`value` is device-timed (CUDA events on the launching stream, inputs
resident in HBM; the working set exceeds the 126 MB L2, so no flush is
needed). `e2e` is the same metric through the public C ABI with host
buffers: every step uploads the inputs from pinned host memory and reads the
results back inside the timed region. Multi-GPU runs (torchrun) give every
rank its own full copy of the workload (weak scaling, no collective in the
data path); time is the max over ranks.

`--impl reference` times the reference's CPU path -- the oracle's FP32
restatement of the reference kernels (the reference itself needs Rust and
wgpu, neither of which exists on these machines) -- on all host cores, on
bounded samples of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "the-powder-toy-rust-wgpu_b200"))

import numpy as np  # noqa: E402

B_AIR = 52  # algorithmic bytes per cell-tick of the air step (reference layout)
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one air tick
# (both tile-form launches) and of one gravity solve of the whole batch (the
# GEMM launches), from ncu captures; workloads without a capture report null.
# Air: 74.7 bytes per cell-tick measured on the first 32 instances of the
# 128-instance batch (2.88 M cells, well above L2) after 900 ticks, scaled by
# its 6,121,601 cells (traffic grows with the cells staged).
MEASURED_DRAM_BYTES = {5: {"air_tick": 457.3e6, "grav_solve": 418.4e6}}
WORKLOAD_NAMES = {
    1: "C1 plain FP32 air+gravity, 153x96 cells (612x384 canvas)",
    2: "C2 plain FP32 air+gravity, 400x225 cells (1600x900 canvas)",
    4: "C4 batched 256 instances, W,H log-uniform 32..512, FP32 air + FP32 gravity",
    5: "C5 batched 64x(400x225) + 64 Pareto(1.5) instances, FP32 air + split-BF16 gravity",
}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), d.get("bf16_tflops_sustained", 1400.0), "measured"
    return 6650.0, 1590.0, 1400.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def workload(cid: int):
    import workloads as W

    return W.config_instances(cid)


def dist_setup(gpus: int):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if gpus > 1 and world != gpus:
        raise SystemExit(f"--gpus {gpus} needs torchrun with {gpus} ranks (WORLD_SIZE={world})")
    if torch.cuda.is_available():
        torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(v: float, world: int) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ----------------------------------------------------------- CPU baseline --

def _strata(insts):
    """Instances grouped by shape class: equal-shape groups of eight or more
    (C5's 64 x 400x225) and the rest (the heavy tail, or all of C4)."""
    shapes = {}
    for i, inst in enumerate(insts):
        shapes.setdefault((inst.xcells, inst.ycells), []).append(i)
    groups = [v for v in shapes.values() if len(v) >= 8]
    rest = sorted(i for v in shapes.values() if len(v) < 8 for i in v)
    out = [g for g in groups]
    if rest:
        out.append(rest)
    return out


def cpu_rate(insts, target_s: float, threads: int | None = None):
    """The oracle's FP32 air + gravity (all host threads) on a stratified
    sample of `insts`: from each shape stratum (equal-shape groups, and the
    heavy tail) a few evenly spaced instances run the same number of ticks;
    each stratum's time per cell-tick is scaled by that stratum's share of the
    workload's cells, so the result estimates the whole workload's
    cell-ticks/s. Ticks are chosen so the timed sample takes about `target_s`.
    Returns (cell-ticks/s, cores, sample description)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    if threads:
        O.set_threads(threads)
    cores = O.num_threads()
    strata = []
    for idx in _strata(insts):
        k = min(len(idx), 4)
        pick = [idx[(j * len(idx)) // k] for j in range(k)]
        strata.append((idx, pick))

    def run(cur, ticks):
        for inst in cur:
            O.air_steps(inst, ticks)
            if inst.config.newton_grav:
                for _ in range(ticks):
                    O.grav_solve(inst.xcells, inst.ycells, inst.gmask, mass_fx=inst.mass_fx)

    t0 = time.perf_counter()
    run([insts[i] for _, pick in strata for i in pick], 1)
    t1 = time.perf_counter() - t0
    ticks = max(2, int(target_s / max(t1, 1e-6)))
    est_s_per_tick = 0.0
    parts = []
    for idx, pick in strata:
        cur = [insts[i].copy() for i in pick]
        t0 = time.perf_counter()
        run(cur, ticks)
        dt = time.perf_counter() - t0
        cells_s = sum(insts[i].cells for i in pick)
        cells_all = sum(insts[i].cells for i in idx)
        est_s_per_tick += dt / ticks / cells_s * cells_all
        parts.append(f"{len(pick)} of {len(idx)} instances ({cells_s} of {cells_all} cells)")
    total = sum(i.cells for i in insts)
    desc = (f"stratified sample, {ticks} ticks each: " + "; ".join(parts) +
            "; air + gravity solve per tick; each stratum's time scaled by its share of the cells")
    return total / est_s_per_tick, cores, desc


def ticks_of(cid: int) -> int:
    """Ticks of one bench step: the configs' stated horizon (C2 states 10000)."""
    return 10000 if cid == 2 else 1000


def config_of(cid: int, insts, ticks: int | None = None) -> dict:
    """The workload as both arms print it (the whole workload, all instances)."""
    return {"workload": WORKLOAD_NAMES[cid], "instances": len(insts), "cells": sum(i.cells for i in insts),
            "ticks_per_step": ticks or ticks_of(cid)}


# ------------------------------------------------------------------ ours --

def run_plain(ticks: int):
    """The plain FP32 single-instance form: one 400x225 grid (C2) stepped
    through the reference-shaped calls, step_air_gpu + GravityFft.solve
    (FP32) once per tick, stream ordered, no graph. Device time, inputs
    resident. Returns (cell-ticks/s, ms per tick)."""
    import torch

    import tpt_field as tf
    import workloads as W

    inst = W.config_instances(2)[0]
    b = tf.SimBuffers.from_instance(inst)
    solver = tf.GravityFft(tf.PRECISION_FP32)
    stream = torch.cuda.current_stream()

    def tick():
        tf.step_air_gpu(b, stream)
        solver.solve(b, b.grav_mass_prev, 1.0 / 65536.0, stream)

    for _ in range(20):
        tick()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(ticks):
        tick()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    solver.close()
    return inst.cells * ticks / (ms / 1e3), ms / ticks


def run_c3(solves: int):
    """The gravity-only configuration: one 512x512 grid with clustered f32
    mass (all cells unmasked), `solves` solves through GravityFft.solve in
    each precision, device time with the inputs resident. Returns
    {precision: {ms_per_solve, ...}}; the split-BF16 line adds the
    algorithmic rate 3F / time with F = 24 X^2 Y + 96 X Y^2 (the dense
    separable DFT-GEMM's flops, times the 3 split products)."""
    import torch

    import tpt_field as tf
    import workloads as W

    X = Y = 512
    mass = torch.from_numpy(W.clustered_mass(X, Y, W.instance_seed(3, 0))).cuda()
    cfg = tf.SimulationConfig(xres=4 * X, yres=4 * Y, newton_grav=True)
    b = tf.SimBuffers(cfg)
    b.grav_mask.fill_(-1)
    stream = torch.cuda.current_stream()
    out = {}
    for name, prec in (("split_bf16", tf.PRECISION_SPLIT_BF16), ("fp32", tf.PRECISION_FP32)):
        solver = tf.GravityFft(prec)
        for _ in range(5):
            solver.solve(b, mass, stream=stream)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(solves):
            solver.solve(b, mass, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / solves
        solver.close()
        out[name] = {"ms_per_solve": round(ms, 5)}
        if prec == tf.PRECISION_SPLIT_BF16:
            F = 24.0 * X * X * Y + 96.0 * X * Y * Y
            out[name]["algorithmic_tflops_3F"] = round(3.0 * F / (ms / 1e3) / 1e12, 1)
    out["config"] = "C3 gravity only, 512x512 cells, clustered f32 mass, %d solves" % solves
    return out


def air_launches(ticks, tuning, per_tick, chunk=1000):
    """Air launches of `ticks` ticks stepped in graphs of `chunk` ticks.
    `per_tick` is the profile's unblocked count (2, or 3 with a NoUpdate +
    heat instance in the tile form); the tile form at temporal depth k runs
    each block of n <= k ticks (cut at the chunk's end) as n + 1 launches,
    plus one settle launch per tick with a NoUpdate + heat instance."""
    import tpt_field as tf

    k = tuning.temporal_depth if tuning.air_form == tf.AIR_FORM_TILES else 1
    if k <= 1:
        return per_tick * ticks
    total, left = 0, ticks
    while left:
        c = min(chunk, left)
        left -= c
        t = 0
        while t < c:
            n = min(k, c - t)
            total += n + 1 + (per_tick - 2) * n
            t += n
    return total


def run_ours(args, rank, world, local):
    import torch

    import tpt_field as tf

    import sharding

    tf.lib()
    cid = args.workload
    insts = workload(cid)
    if args.instances:  # a prefix of the workload, for profiling captures
        insts = insts[: args.instances]
    total_cells = sum(i.cells for i in insts)
    cfg = config_of(cid, insts, args.ticks or None)
    if args.scaling == "strong" and world > 1:  # this rank's share, no exchange between ranks
        insts = [insts[i] for i in sharding.shard_of([(i.xcells, i.ycells) for i in insts], rank, world)]
    ticks = args.ticks or ticks_of(cid)
    precision = tf.PRECISION_SPLIT_BF16 if cid == 5 else tf.PRECISION_FP32
    stream = torch.cuda.current_stream()
    batch = tf.Batch(insts, precision)
    if not args.skip_tune:
        batch.tune()
    if args.air_form != "tuned":
        t = batch.tuning()
        t.air_form = tf.AIR_FORM_SWEEP if args.air_form == "sweep" else tf.AIR_FORM_TILES
        t.tile_x, t.tile_y = args.air_shape or ((224, 64) if args.air_form == "sweep" else tf.TILE_SHAPES[0])
        t.ctas_per_sm = 0
        t.temporal_depth = args.temporal_depth
        t.work_queue = args.work_queue
        batch.set_tuning(t)
    cells = sum(i.cells for i in insts)
    # cells all ranks advance per tick: every rank has a full copy (weak) or
    # a share of one copy (strong)
    job_cells = total_cells if args.scaling == "strong" else total_cells * world

    # device-timed: inputs resident
    for _ in range(args.warmup):
        batch.step(ticks)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        batch.step(ticks)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier(world)
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    value = job_cells * ticks * args.steps / (ms / 1e3)

    # end to end through the C ABI with pinned host buffers: each grid kind of
    # every instance in one dense buffer (tpt_batch_write_field /
    # tpt_batch_read_field)
    total = batch.total_cells
    host_in = {}
    for n, fid in tf.Batch.GRIDS:
        dt = getattr(insts[0], n).dtype
        t = torch.empty(total, dtype=torch.int32, pin_memory=True)
        t.numpy().view(dt)[:] = np.concatenate([getattr(inst, n).ravel() for inst in insts])
        host_in[fid] = t.numpy().view(dt)
    out_fields = (tf.FIELD_PV, tf.FIELD_VX, tf.FIELD_VY, tf.FIELD_HV, tf.FIELD_GX, tf.FIELD_GY)
    host_out = {fid: torch.empty(total, dtype=torch.float32, pin_memory=True).numpy() for fid in out_fields}
    h2d = sum(a.nbytes for a in host_in.values())
    d2h = sum(a.nbytes for a in host_out.values())

    def e2e_step():
        for fid, a in host_in.items():
            tf.check(tf.lib().tpt_batch_write_field(batch._h, fid, tf._ptr(a), a.nbytes, tf._stream(stream)))
        batch.step(ticks, stream)
        for fid, a in host_out.items():
            tf.check(tf.lib().tpt_batch_read_field(batch._h, fid, tf._ptr(a), a.nbytes, tf._stream(stream)))

    e2e_steps = 0 if args.no_e2e else max(1, min(args.steps, 3))
    e2e_value = None
    if e2e_steps:
        e2e_step()
        torch.cuda.synchronize()
        barrier(world)
        e0.record(stream)
        for _ in range(e2e_steps):
            e2e_step()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        e2e_ms = max_over_ranks(e0.elapsed_time(e1), world)
        e2e_value = job_cells * ticks * e2e_steps / (e2e_ms / 1e3)

    # per-phase device times for the roofline
    prof = batch.profile_phases(args.phase_ticks)
    hbm, bf16, bf16s, peak_src = load_peaks()
    air_gbs = prof.cells * prof.ticks * B_AIR / (prof.air_ms / 1e3) / 1e9
    tuning = batch.tuning()
    air_launch_ms = prof.air_ms / air_launches(prof.ticks, tuning, prof.air_launches_per_tick, chunk=prof.ticks)
    roof_air = {"kernel": "air tick (pressure+velocity, advection+heat+masks)", "bound": "hbm",
                "achieved": round(air_gbs, 1), "peak": hbm, "unit": "GB/s", "frac": round(air_gbs / hbm, 4),
                "peak_source": peak_src, "algorithmic_bytes_per_cell_tick": B_AIR,
                "traffic": MEASURED_DRAM_BYTES.get(cid, {}).get("air_tick"),
                "traffic_unit": "DRAM bytes per tick, both launches (ncu)",
                "ms_per_tick": round(prof.air_ms / prof.ticks, 5),
                "avg_launch_ms": round(air_launch_ms, 5)}
    phases = {"air_ms_per_tick": prof.air_ms / prof.ticks, "grav_ms_per_tick": prof.grav_ms / prof.ticks}
    if precision == tf.PRECISION_SPLIT_BF16 and prof.grav_ms > 0:
        tfl = prof.grav_flops_per_tick * prof.ticks / (prof.grav_ms / 1e3) / 1e12
        roof_grav = {"kernel": "split-BF16 DFT-GEMM gravity", "bound": "tensor", "achieved": round(tfl, 2),
                     "peak": bf16, "unit": "TFLOP/s", "frac": round(tfl / bf16, 4), "peak_source": peak_src,
                     "peak_sustained": bf16s, "frac_sustained": round(tfl / bf16s, 4),
                     "traffic": MEASURED_DRAM_BYTES.get(cid, {}).get("grav_solve"),
                     "traffic_unit": "DRAM bytes per solve of the batch, GEMM launches (ncu)"}
    else:
        roof_grav = None
    dominant = roof_grav if (roof_grav and prof.grav_ms > prof.air_ms) else roof_air
    launches = (air_launches(ticks, tuning, prof.air_launches_per_tick) + prof.grav_launches_per_tick * ticks) * \
        args.steps + (args.steps if ticks % 2 else 0)

    plain = None
    if rank == 0 and world == 1 and args.plain_ticks > 0:
        p_rate, p_ms = run_plain(args.plain_ticks)
        plain = {"workload": WORKLOAD_NAMES[2] + ", one instance, step_air_gpu + GravityFft.solve per tick",
                 "value": p_rate, "unit": "cell-ticks/s", "ms_per_tick": p_ms, "ticks": args.plain_ticks,
                 "speedup_of_this_line": value / world / p_rate}

    c3 = run_c3(args.c3_solves) if rank == 0 and world == 1 and args.c3_solves > 0 else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, cores, desc = cpu_rate(insts, args.cpu_seconds)
        cpu = {"value": rate, "unit": "cell-ticks/s", "cores": cores, "kind": "port", "sample": desc}

    if rank == 0:
        line = {
            "metric": "cell-ticks/s", "value": value, "unit": "cell-ticks/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": args.scaling, "vs_baseline": None,
            "dtype": "f32" if precision == tf.PRECISION_FP32 else "f32 air + bf16x3 gravity (f32 accumulate)",
            "data": "synthetic (seeded sandboxes, workloads.py)",
            "config": cfg,
            "l2": "working set > 126 MB L2, no flush",
            "tuning": batch.tuning_dict(),
            "e2e": {"value": e2e_value, "unit": "cell-ticks/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": e2e_steps,
                    "calls": f"tpt_batch_write_field x{len(host_in)}, tpt_batch_step, "
                             f"tpt_batch_read_field x{len(host_out)} from/to pinned host buffers"},
            "gpu_launches": launches,
            "roofline": dominant,
            "roofline_phases": {"air": roof_air, "gravity": roof_grav, **phases},
            "clocks": clk,
            "cpu_baseline": cpu,
            "plain_fp32_single_instance": plain,
            "gravity_c3": c3,
        }
        print(json.dumps(line), flush=True)
    batch.close()


# -------------------------------------------------------------- 3-D ----
# ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_grav_gather_rows
# launch on the bench's world with every brick listed (134.3 MB + 4.0 MB)
VOX_GRAV_GATHER_DRAM_BYTES = 138.3e6
VOX_NAME = ("3-D sandbox field step, 64^3 cells per world over 256^3 voxels with every brick active: air gather, "
            "air solve (12 Jacobi sweeps), gravity solve (24 sweeps), clear mass, gravity gather")


def _vox_cpu_rate(host: dict, target_s: float):
    """The oracle's 3-D tick (single-threaded C++) on one world; returns
    (cell-ticks/s, cores, sample description)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    d = {k: v.copy() for k, v in host.items()}

    def tick():
        O.vox_field_step(d, 12)
        O.vox_grav_gather(d)

    t0 = time.perf_counter()
    tick()
    t1 = time.perf_counter() - t0
    n = max(1, min(50, int(target_s / max(t1, 1e-6))))
    t0 = time.perf_counter()
    for _ in range(n):
        tick()
    dt = time.perf_counter() - t0
    return 262144 * n / dt, 1, f"1 world x {n} ticks, oracle restatement of the five passes"


def run_voxel3d(args, rank, world, local):
    """The 3-D field step (tpt_vox_field_step + tpt_vox_grav_gather per tick),
    `--worlds` worlds per rank, ticks captured in one CUDA graph per step.
    Metric: cell-ticks/s over the 64^3 coarse cells of every world."""
    import torch

    import tpt_field as tf
    import voxel3d as V
    import workloads as W

    tf.lib()
    host = W.voxel_world(0x3D00, active=1.0)
    nw = args.worlds
    ticks = args.ticks or 100
    stream = torch.cuda.Stream()
    plans = {"batched": V.Plan(tf.VOX_AUTO), "cluster": V.Plan(tf.VOX_CLUSTER),
             "per_sweep": V.Plan(tf.VOX_PER_SWEEP)}
    devs = [V.upload(host) for _ in range(nw)]
    nonempty = int(np.count_nonzero(host["voxel"] & 0xFF))

    def tick(plan):
        V.field_step(plan, devs, 12, stream)
        for b, _ in devs:
            V.gravity_gather(plan, b, stream)

    def graph_of(fn, n):
        with torch.cuda.stream(stream):
            for _ in range(2):
                fn()
        stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            for _ in range(n):
                fn()
        return g

    def time_graph(g, reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(reps):
                g.replay()
            e1.record(stream)
        stream.synchronize()
        return e0.elapsed_time(e1)

    L0 = tf.launch_count()
    g_tick = graph_of(lambda: tick(plans["batched"]), ticks)
    launches_per_tick = (tf.launch_count() - L0) / (ticks + 2)  # two warm-up ticks, then the captured ones
    for _ in range(args.warmup):
        g_tick.replay()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ms = time_graph(g_tick, args.steps)
    clk = clocks.stop()
    barrier(world)
    ms = max_over_ranks(ms, world)
    value = 262144 * nw * world * ticks * args.steps / (ms / 1e3)

    # phases, each alone in a graph of `ticks` launches (device time per launch)
    reps = 3
    phase = {}
    g = graph_of(lambda: [V.AirState.gather(a, plans["batched"], b, stream) for b, a in devs], ticks)
    phase["air_gather"] = time_graph(g, reps) / (reps * ticks * nw)
    g = graph_of(lambda: [V.gravity_gather(plans["batched"], b, stream) for b, _ in devs], ticks)
    phase["grav_gather"] = time_graph(g, reps) / (reps * ticks * nw)
    forms = {}
    for name, plan in plans.items():
        g = graph_of(lambda: V.field_step(plan, devs, 12, stream), ticks)
        step_ms = time_graph(g, reps) / (reps * ticks)
        forms[name] = {"field_step_ms": round(step_ms, 5),
                       "solves_ms": round(step_ms - phase["air_gather"] * nw, 5)}  # air + gravity solves, every world
    for name in forms:
        forms[name]["batched_speedup"] = round(forms[name]["solves_ms"] / forms["batched"]["solves_ms"], 3)
    del g

    # end to end: host buffers in, ticks, fields out, through the public calls
    in_keys = ("voxel", "aux_tmp", "vx", "vy", "vz", "p", "p_tmp", "temp", "solid", "pv", "grav_mass",
               "grav_potential", "grav_potential_tmp")
    out_keys = ("vx", "vy", "vz", "p", "pv", "grav_force_x", "grav_force_y", "grav_force_z")

    def pinned(a):
        t = torch.empty(a.size, dtype=torch.int32 if a.dtype != np.float32 else torch.float32, pin_memory=True)
        t.numpy().view(a.dtype)[:] = a
        return t

    h_in = {k: pinned(host[k]) for k in in_keys}
    h_out = [{k: torch.empty(262144, dtype=torch.int32 if k == "pv" else torch.float32, pin_memory=True)
              for k in out_keys} for _ in range(nw)]

    def dev_of(b, a, k):
        if k == "voxel":
            return b.voxel_a
        if k == "temp":
            return a.t
        return getattr(b, k) if hasattr(b, k) else getattr(a, k)

    def e2e_step():
        with torch.cuda.stream(stream):
            for b, a in devs:
                for k, t in h_in.items():
                    dev_of(b, a, k).copy_(t.view(dev_of(b, a, k).dtype), non_blocking=True)
            g_tick.replay()
            for (b, a), o in zip(devs, h_out):
                for k, t in o.items():
                    t.copy_(dev_of(b, a, k), non_blocking=True)

    e2e_steps = 0 if args.no_e2e else max(1, min(args.steps, 3))
    e2e_value = None
    if e2e_steps:
        e2e_step()
        stream.synchronize()
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(e2e_steps):
                e2e_step()
            e1.record(stream)
        stream.synchronize()
        barrier(world)
        e2e_ms = max_over_ranks(e0.elapsed_time(e1), world)
        e2e_value = 262144 * nw * world * ticks * e2e_steps / (e2e_ms / 1e3)
    h2d = sum(t.numel() * 4 for t in h_in.values()) * nw
    d2h = sum(t.numel() * 4 for o in h_out for t in o.values())

    hbm, bf16, bf16s, peak_src = load_peaks()
    # algorithmic DRAM bytes of the gathers with every brick listed: the
    # voxel words, the tmp words of the non-empty voxels, and the cell words
    # written (air: solid + temp; gravity: read-modify-write of the mass)
    b_air = 4 * W.VOX_VOXELS + 8 * W.VOX_CELLS
    b_grav = 4 * W.VOX_VOXELS + 4 * nonempty + 8 * W.VOX_CELLS
    gbs_air = b_air / (phase["air_gather"] / 1e3) / 1e9
    gbs_grav = b_grav / (phase["grav_gather"] / 1e3) / 1e9
    roof_grav = {"kernel": "gravity gather (k_brick_mult + k_grav_gather_rows)", "bound": "hbm",
                 "achieved": round(gbs_grav, 1), "peak": hbm,
                 "unit": "GB/s", "frac": round(gbs_grav / hbm, 4), "peak_source": peak_src,
                 "algorithmic_bytes_per_launch": b_grav, "avg_launch_ms": round(phase["grav_gather"], 5),
                 "traffic": VOX_GRAV_GATHER_DRAM_BYTES,
                 "traffic_unit": "DRAM bytes read + written by k_grav_gather_rows per launch (ncu)"}
    roof_air = {"kernel": "k_air_gather", "bound": "hbm", "achieved": round(gbs_air, 1), "peak": hbm,
                "unit": "GB/s", "frac": round(gbs_air / hbm, 4), "peak_source": peak_src,
                "algorithmic_bytes_per_launch": b_air, "avg_launch_ms": round(phase["air_gather"], 5),
                "traffic": None}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, cores, desc = _vox_cpu_rate(host, args.cpu_seconds)
        cpu = {"value": rate, "unit": "cell-ticks/s", "cores": cores, "kind": "port", "sample": desc}
    if rank == 0:
        line = {
            "metric": "cell-ticks/s", "value": value, "unit": "cell-ticks/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (i32 mass, pv)",
            "data": "synthetic (seeded 3-D world, workloads.voxel_world)",
            "config": {"workload": VOX_NAME, "worlds": nw, "ticks_per_step": ticks,
                       "l2": "gather inputs 128 MiB per world > 126 MB L2, no flush", "form": "batched"},
            "e2e": {"value": e2e_value, "unit": "cell-ticks/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": e2e_steps},
            "gpu_launches": round(launches_per_tick * ticks * args.steps),
            "roofline": roof_grav if phase["grav_gather"] >= phase["air_gather"] else roof_air,
            "roofline_phases": {"air_gather": roof_air, "grav_gather": roof_grav},
            "gather_ms_per_world_tick": {k: round(v, 5) for k, v in phase.items()},
            "solve_forms": forms,
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    for p in plans.values():
        p.close()


def run_reference(args, rank, world):
    if rank != 0:
        return
    cid = args.workload
    insts = workload(cid)
    rate_samples = []
    cores = desc = None
    # each step: a stratified sample of the workload, sized to about
    # --ref-step-seconds of host work
    for _ in range(args.warmup + args.steps):
        rate, cores, desc = cpu_rate(insts, args.ref_step_seconds)
        rate_samples.append(rate)
    rates = rate_samples[args.warmup:]
    value = statistics.median(rates)
    line = {
        "impl": "reference", "metric": "cell-ticks/s", "value": value, "unit": "cell-ticks/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded sandboxes, workloads.py)",
        "config": config_of(cid, insts, args.ticks or None),
        "spread": {"min": min(rates), "max": max(rates)},
        "cpu_baseline": {"value": value, "unit": "cell-ticks/s", "cores": cores, "kind": "port", "sample": desc},
        "e2e": {"value": value, "unit": "cell-ticks/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_save_io(args):
    """Host timing of the `.tptrs` codec (crates/tpt-save/src/lib.rs) on a
    C2-sized save: a 1600x900 canvas (90,000 cells, eight grids) with 50,000
    particle records. One step decodes the file, restores the field-step
    instance from it and encodes it again. Metric: decoded payload bytes per
    second."""
    import tpt_field as tf
    import workloads as W

    inst = W.make_stress_instance(400, 225, 77)
    sv = tf.SaveData.new(1600, 900)
    for name, key in (("air_pv", "pv"), ("air_vx", "vx"), ("air_vy", "vy"), ("air_hv", "hv"), ("fan_vx", "fan_vx"),
                      ("fan_vy", "fan_vy"), ("wall_bmap", "wall"), ("wall_emap", "emap")):
        sv.set_grid(name, getattr(inst, key))
    st = W.Stream(78)
    parts = np.zeros((50000, 16), np.uint32)
    parts[:, 0] = (st.u64(50000) % np.uint64(180) + np.uint64(1)).astype(np.uint32)
    parts[:, 3] = st.uniform(0, 1600, 50000).astype(np.float32).view(np.uint32)
    parts[:, 4] = st.uniform(0, 900, 50000).astype(np.float32).view(np.uint32)
    parts[:, 7] = st.uniform(250, 400, 50000).astype(np.float32).view(np.uint32)
    sv.set_particles(parts)
    data = sv.to_bytes()
    import zlib
    payload = len(zlib.decompress(data[8:]))

    def step():
        s2 = tf.SaveData.from_bytes(data)
        s2.to_instance()
        return s2.to_bytes()

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t0) / args.steps
    t0 = time.perf_counter()
    for _ in range(args.steps):
        tf.SaveData.from_bytes(data)
    dec = (time.perf_counter() - t0) / args.steps
    line = {
        "metric": "save payload bytes/s (decode + restore + encode)", "value": payload / dt, "unit": "B/s",
        "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3,
        "higher_is_better": True, "scaling": "none", "vs_baseline": None, "dtype": "bytes",
        "data": "synthetic (a C2 stress sandbox and 50,000 particle records)",
        "config": {"workload": ".tptrs codec, 1600x900 canvas, 50000 particles", "file_bytes": len(data),
                   "payload_bytes": payload, "decode_ms": dec * 1e3, "threads": 1},
    }
    print(json.dumps(line), flush=True)


def run_reference_voxel3d(args, rank, world):
    if rank != 0:
        return
    import workloads as W

    host = W.voxel_world(0x3D00, active=1.0)
    rates = []
    cores = desc = None
    for _ in range(args.warmup + args.steps):
        rate, cores, desc = _vox_cpu_rate(host, args.cpu_seconds / max(args.steps, 1))
        rates.append(rate)
    value = statistics.median(rates[args.warmup:])
    line = {
        "impl": "reference", "metric": "cell-ticks/s", "value": value, "unit": "cell-ticks/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (i32 mass, pv)", "data": "synthetic (seeded 3-D world, workloads.voxel_world)",
        "config": {"workload": VOX_NAME, "worlds": 1},
        "cpu_baseline": {"value": value, "unit": "cell-ticks/s", "cores": cores, "kind": "port", "sample": desc},
        "e2e": {"value": value, "unit": "cell-ticks/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", type=int, choices=(1, 2, 4, 5), default=5)
    ap.add_argument("--ticks", type=int, default=0)
    ap.add_argument("--plain-ticks", type=int, default=500, help="ticks of the plain FP32 comparison (0 = skip)")
    ap.add_argument("--c3-solves", type=int, default=100,
                    help="solves of the gravity-only 512x512 line, each precision (0 = skip)")
    ap.add_argument("--scaling", choices=("weak", "strong"), default="weak",
                    help="weak: every rank steps a full copy; strong: ranks split one copy's instances")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="host work of the GPU arm's cpu_baseline leg")
    ap.add_argument("--ref-step-seconds", type=float, default=2.0,
                    help="host work of one --impl reference step (a stratified sample of the workload)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer run (profiling captures)")
    ap.add_argument("--phase-ticks", type=int, default=200, help="even tick count of the per-phase timing")
    ap.add_argument("--air-form", choices=("tuned", "tiles", "sweep"), default="tuned",
                    help="air tick form of the batched workloads (default: the autotuner's choice)")
    ap.add_argument("--air-shape", type=lambda v: tuple(int(x) for x in v.split("x")), default=None,
                    help="with --air-form: tile (tiles) or lanes x rows (sweep), e.g. 64x16")
    ap.add_argument("--temporal-depth", type=int, default=1,
                    help="with --air-form tiles: ticks per temporally blocked run (1 = none)")
    ap.add_argument("--work-queue", type=int, choices=(0, 1), default=1,
                    help="with --air-form tiles: 1 = atomic tile queue (the library's default), 0 = static striding")
    ap.add_argument("--skip-tune", action="store_true", help="keep the batch's default tuning (profiling captures)")
    ap.add_argument("--instances", type=int, default=0,
                    help="only the first N instances of the workload (profiling captures on a smaller case)")
    ap.add_argument("--voxel3d", action="store_true", help="the 3-D sandbox's field step instead of the 2-D one")
    ap.add_argument("--worlds", type=int, default=1, help="3-D worlds per rank (--voxel3d)")
    ap.add_argument("--save-io", action="store_true", help="host timing of the .tptrs save codec")
    args = ap.parse_args()
    if args.save_io:
        run_save_io(args)
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        world = int(os.environ.get("WORLD_SIZE", "1"))
        if args.voxel3d:
            run_reference_voxel3d(args, rank, world)
        else:
            run_reference(args, rank, world)
        return
    rank, world, local = dist_setup(args.gpus)
    try:
        if args.voxel3d:
            run_voxel3d(args, rank, world, local)
        else:
            run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
