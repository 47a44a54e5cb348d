"""Throughput benchmark of the NICAM tracer-advection step on B200.

Workload (the configuration the headline metric is quoted on): glevel 8,
rlevel 0 (10 regions of 258x258, 655,362 columns), kall 96, 32 tracers, FP32
flux/limiter arithmetic with the FP64 rhogq/rhog mass update, dt = 150 s
(1200 s scaled by 2^(5-gl)).  One step advances every tracer cell-level once:
2,013,272,064 updates.  Synthetic seeded inputs of the reference's shapes
(there are no input snapshots to load).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--mode fast|plain] [--impl ours|reference]

value : updates/s of the device-resident step loop (CUDA events on the library's
        stream, max over ranks); e2e: the same metric through the host-pointer
        C ABI call with pinned host buffers, copies inside the timed region.
--impl reference: the CPU restatement of the reference (oracle) on all host
        cores, on a bounded sample of the workload (each step: the same glevel 8
        grid and 32 tracers, 10 of the 94 physical levels), reported in the same unit.
N > 1: one process per GPU, each running an independent replica of the workload
(the single-GPU path does not shard), value = total updates / max time.
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
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "tracer cell-level updates/s"
UNIT = "updates/s"


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measured_traffic(kernel, shape, updates):
    """DRAM bytes per launch of `kernel` from the committed ncu figure (profiles/dram_traffic.json),
    scaled by the updates per launch; None when no capture of this kernel and tile shape exists."""
    p = ROOT / "profiles" / "dram_traffic.json"
    if not p.exists():
        return None, None
    d = json.loads(p.read_text()).get(kernel)
    for c in (d or {}).get("captures", []):
        if list(c["tile_txtytg"]) == list(shape):
            return c["bytes_per_update"] * updates, "ncu " + c["capture"] + ", scaled by updates"
    return None, None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms in the background."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except FileNotFoundError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = [r for r in self.rows if len(r) >= 9]
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    """One process per GPU (torchrun env).  NCCL where CUDA is present, gloo on a host
    without GPUs (the multi-rank tests run there); a short timeout so that ranks waiting
    for a lost peer end with an error."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def allreduce_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------------------------
def cpu_reference(glevel, kall, ntr, steps, warmup, threads):
    """The oracle (C restatement of the reference) on `threads` host cores; returns updates/s.
    The grid's topology and halo plan come from the oracle too (oracle.GridTables), so this
    leg loads no part of the library under test."""
    import numpy as np

    from icoatmosbenchmark_v1_b200 import fields as F
    from icoatmosbenchmark_v1_b200.grid import Grid, default_dt
    from oracle import oracle as O
    g = Grid(glevel, 0, kall, tables=O.GridTables())
    f = {k: v.numpy() for k, v in F.make_fields(g).items()}
    S = {k: v.numpy().copy() for k, v in F.make_state(g, ntr, "mixed").items()}
    d = O.make_dims(glevel, 0, kall)
    topo = O.Topo(glevel, 0, 1)
    dt = default_dt(glevel)
    for _ in range(warmup):
        O.step(d, g.have_sgp, topo, dt, S, f, g.arrays, nthreads=threads)
    t0 = time.perf_counter()
    for _ in range(steps):
        O.step(d, g.have_sgp, topo, dt, S, f, g.arrays, nthreads=threads)
    el = time.perf_counter() - t0
    upd = (10 * 4 ** glevel + 2) * kall * ntr * steps
    return upd / el, el, upd, np


def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    ks = args.ref_kall
    val, el, upd, _ = cpu_reference(args.glevel, ks, args.ntr, args.steps, args.warmup, threads)
    sample = (f"each step: glevel {args.glevel}, all {args.ntr} tracers, {ks - 2} of the {args.kall - 2} "
              f"physical levels (kall {ks}); {args.steps} steps, {upd:.3e} updates")
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args),
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "sample_updates_per_step": upd // max(args.steps, 1),
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def workload_config(args):
    return {"workload": f"gl{args.glevel}_k{args.kall}_t{args.ntr}", "glevel": args.glevel, "rlevel": 0,
            "kall": args.kall, "tracers": args.ntr, "columns": 10 * 4 ** args.glevel + 2,
            "updates_per_step": (10 * 4 ** args.glevel + 2) * args.kall * args.ntr,
            "mode": args.mode, "dt": 1200.0 * 2.0 ** (5 - args.glevel),
            "l2": "inputs larger than L2 (state %.1f GB)" % ((10 * 4 ** args.glevel + 2) * args.kall * args.ntr * 8e-9)}


# ---------------------------------------------------------------------------------------------
def run_ours(args, world, rank, local):
    import numpy as np
    import torch

    from icoatmosbenchmark_v1_b200 import api
    from icoatmosbenchmark_v1_b200 import fields as F
    from icoatmosbenchmark_v1_b200.grid import Grid, default_dt

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    t_host = time.perf_counter()
    g = Grid(args.glevel, 0, args.kall)
    t_host = time.perf_counter() - t_host
    dt = default_dt(args.glevel)
    f = F.make_fields(g, device=dev)
    st = F.make_state(g, args.ntr, "mixed", device=dev, fields=f)
    del f["rhog"], f["rhog_pl"]
    ctx = api.IcoAdv(args.glevel, 0, args.kall - 2, device=local)
    ctx.set_grid(g)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    upd = (10 * 4 ** args.glevel + 2) * args.kall * args.ntr
    grid_setup = measure_grid_setup(ctx, g, stream, t_host)
    if args.shard and args.mode == "fast":
        return run_sharded(args, world, rank, local, ctx, g, st, f, dt, upd, grid_setup)

    if args.mode == "plain":
        def step():
            ctx.advect_step(dt, st["rhog"], st["rhog_pl"], st["rhogq"], st["rhogq_pl"], f["rhogvx"], f["rhogvx_pl"],
                            f["rhogvy"], f["rhogvy_pl"], f["rhogvz"], f["rhogvz_pl"], f["rhogw"], f["rhogw_pl"])
        dtype = "f64"
        s_bytes = 48
    else:
        runner = ctx.fast_runner(g, st, f, dt, autotune=args.tile_shape < 0)
        if args.tile_shape >= 0:
            ctx.fast_set_shape(args.tile_shape)
            runner.shape = args.tile_shape
        step = runner.step
        st = runner.state
        dtype = "f32"
        s_bytes = 32

    err = m0 = None
    extra = args.mode == "fast" and world == 1 and rank == 0 and not args.no_extra and not args.no_check
    init = ref = None
    if args.mode != "plain" and not args.no_check:
        # one FP64 plain-path step on a copy: the reference of the batched step's first step
        ref = {k: v.clone() for k, v in runner.state.items()}
        if extra:  # the FP64 variant starts from the same state later
            init = {k: v.clone() for k, v in runner.state.items()}
        ctx.advect_step(dt, ref["rhog"], ref["rhog_pl"], ref["rhogq"], ref["rhogq_pl"], f["rhogvx"], f["rhogvx_pl"],
                        f["rhogvy"], f["rhogvy_pl"], f["rhogvz"], f["rhogvz_pl"], f["rhogw"], f["rhogw_pl"])
        m0 = tracer_mass(g, runner.state)
        step()
        torch.cuda.synchronize()
        err = float(((runner.state["rhogq"] - ref["rhogq"]).abs().max() / ref["rhogq"].abs().max()).item())
        if not extra:
            ref = None
        torch.cuda.empty_cache()
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    sampler = ClockSampler(local)
    sampler.start()
    n0 = ctx.launch_count
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if args.mode != "plain":
        runner.start_timing()
    torch.cuda.synchronize()
    barrier(world)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    launches = ctx.launch_count - n0
    drift = None
    if m0 is not None:
        m1 = tracer_mass(g, runner.state)
        drift = float(((m1 - m0).abs() / m0.abs()).max().item())
    ms = e0.elapsed_time(e1) / args.steps
    ms = allreduce_max(ms, world)
    value = upd * world / (ms * 1e-3)
    peak, peak_kind = load_peaks()
    b_alg = 16.0 + s_bytes / args.ntr
    kern = None
    if args.mode != "plain":
        kern = runner.kernel_stats()
    if kern:  # dominant kernel timed with its own events inside the step loop
        achieved = kern["bytes_per_launch"] / (kern["ms_per_launch"] * 1e-3) / 1e9
        shape = list(ctx.fast_shapes()[runner.shape])
        traffic, tsrc = args.traffic, None
        if traffic is None:
            traffic, tsrc = measured_traffic(kern["name"], shape, upd)
        roof = {"bound": "hbm", "kernel": kern["name"], "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic, "traffic_source": tsrc,
                "alg_bytes_per_update": runner.alg_bytes}
    else:
        achieved = upd * b_alg / (ms * 1e-3) / 1e9
        roof = {"bound": "hbm", "kernel": "whole step", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind, "traffic": args.traffic,
                "alg_bytes_per_update": b_alg}
    # ---- e2e through the host-pointer C ABI (pinned host buffers, copies inside the timed region)
    e2e = None
    if not args.no_e2e:
        e2e = measure_e2e(args, ctx, g, st, f, dt, upd, world)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        cval, cel, cupd, _ = cpu_reference(args.glevel, args.ref_kall, args.ntr, 1, 0, threads)
        cpu = {"value": cval, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"oracle, glevel {args.glevel}, all {args.ntr} tracers, {args.ref_kall - 2} of the "
                         f"{args.kall - 2} physical levels (kall {args.ref_kall}), 1 step "
                         f"({cupd:.3e} updates, {cel:.1f} s)"}
    cfg = workload_config(args)
    shape_idx = runner.shape if args.mode != "plain" else None
    if args.mode != "plain":
        cfg["tile"] = {"shape_txtytg": list(ctx.fast_shapes()[runner.shape]),
                       "autotune_ms": [round(t["ms"], 3) for t in runner.tuning] or None}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": dtype, "data": "synthetic", "config": cfg,
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clocks,
                "grid_setup": grid_setup}
        if err is not None:
            line["max_rel_err_vs_fp64"] = err  # first step vs the FP64 plain path (bit-exact to the oracle)
            line["mass_drift"] = {"value": drift, "steps": 1 + args.warmup + args.steps}
    if extra:  # the FP64 variant of the batched step on the same workload, from the same state
        runner = step = None
        st = None
        import gc
        gc.collect()
        torch.cuda.empty_cache()
        line["fp64_variant"] = measure_fast64(args, ctx, g, init, ref, f, dt, shape_idx, ms)
        init = ref = None
        gc.collect()
        torch.cuda.empty_cache()
    ctx.close()
    if rank == 0 and world == 1 and not args.no_adjoint and args.mode == "fast":
        runner = st = f = step = None  # the bound step method holds the runner and its buffers
        import gc
        gc.collect()
        torch.cuda.empty_cache()
        line["adjoint"] = measure_adjoint(args, local, fast_ms=ms, steps=args.adjoint_steps,
                                          every=args.adjoint_every)
    if extra:
        import gc
        gc.collect()
        torch.cuda.empty_cache()
        line["uneven_batch"] = measure_uneven(args, local)
    if rank == 0:
        print(json.dumps(line), flush=True)


def measure_fast64(args, ctx, g, init, ref, f, dt, shape, ms32):
    """The FP64 variant of the batched step (FP64 fields, face values, bounds and limiters) on
    the workload of the line, from the line's initial state: its first step's max relative
    error against the plain FP64 step, its device time per step (CUDA events on the library's
    stream) and the relative mass drift over its steps."""
    import torch

    from icoatmosbenchmark_v1_b200 import api
    r = api.FastRunner(ctx, g, init, f, dt, autotune=False, f64=True)
    ctx.fast_set_shape(shape)
    r.shape = shape
    m0 = tracer_mass(g, r.state)
    r.step()
    torch.cuda.synchronize()
    err = float(((r.state["rhogq"] - ref["rhogq"]).abs().max() / ref["rhogq"].abs().max()).item())
    for _ in range(max(args.warmup - 1, 1)):
        r.step()
    n = max(1, min(args.steps, 5))
    stream = torch.cuda.ExternalStream(ctx.stream, device=init["rhog"].device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(n):
        r.step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / n
    m1 = tracer_mass(g, r.state)
    drift = float(((m1 - m0).abs() / m0.abs()).max().item())
    upd = (10 * 4 ** args.glevel + 2) * args.kall * args.ntr
    out = {"workload": f"gl{args.glevel}_k{args.kall}_t{args.ntr}", "dtype": "f64", "steps": n,
           "ms_per_step": ms, "value": upd / (ms * 1e-3), "unit": UNIT,
           "max_rel_err_vs_fp64_plain": err, "mass_drift": {"value": drift, "steps": 1 + max(args.warmup - 1, 1) + n},
           "time_vs_fp32_variant": ms / ms32}
    del r
    return out


def measure_grid_setup(ctx, g, stream, t_host):
    """The grid's positions and metrics built on the device (ica_grid_build_dev, timed with CUDA
    events after one warm build) beside the host (numpy) build the run uses, and the largest
    difference between the two relative to each array's largest magnitude."""
    import torch
    out = ctx.build_grid(g.R)  # warm: the context's scratch
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    out = ctx.build_grid(g.R)
    e1.record(stream)
    torch.cuda.synchronize()
    err = 0.0
    for k, v in out.items():
        ref = torch.as_tensor(g.arrays[k], device=v.device)
        err = max(err, float((v - ref).abs().max() / ref.abs().max().clamp_min(1e-300)))
    del out
    torch.cuda.empty_cache()
    return {"device_ms": e0.elapsed_time(e1), "host_numpy_s": t_host, "max_rel_diff": err,
            "what": "positions, GMTR_p/t/a, GRD_xr, coef_grad and pole arrays"}


def run_sharded(args, world, rank, local, ctx, g, st, f, dt, upd, grid_setup):
    """--shard: the workload region-sharded over the ranks (strong scaling: the same grid on
    every N), each rank computing its block of regions with the two exchanges of a step as NCCL
    send/recv (ShardedRunner).  value = the whole grid's updates / the max over ranks of the
    step time."""
    import torch

    from icoatmosbenchmark_v1_b200 import shard
    plan = shard.ShardPlan.build(args.glevel, 0, world)
    ctx.fast_set_shape(args.tile_shape if args.tile_shape >= 0 else 3)
    run = shard.ShardedRunner(ctx, plan, rank, st, f, dt)
    for _ in range(args.warmup):
        run.step()
    torch.cuda.synchronize()
    barrier(world)
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(local)
    sampler.start()
    n0 = ctx.launch_count
    e0.record(stream)
    for _ in range(args.steps):
        run.step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    ms = allreduce_max(e0.elapsed_time(e1) / args.steps, world)
    bval_b, halo_b = plan.bytes_per_step(args.kall, args.ntr)
    status = ctx.fast_status()
    if rank == 0:
        cfg = workload_config(args)
        cfg["parallelism"] = f"regions sharded over {world} ranks (blocks {plan.blocks}), NCCL send/recv"
        line = {"metric": METRIC, "value": upd / (ms * 1e-3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": cfg,
                "exchange_bytes_per_step": {"boundary_values": bval_b, "halo": halo_b},
                "gpu_launches": ctx.launch_count - n0, "clocks": clocks, "grid_setup": grid_setup,
                "status": status}
        print(json.dumps(line), flush=True)
    ctx.close()


UNEVEN = ((7, 96, 40), (6, 42, 12))  # (glevel, kall, tracers) of the two instances


def tracer_mass(g, S):
    """Global mass of every tracer (FP64): sum over interior cells and pole centres of
    rhogq * area * dz over the physical levels."""
    import torch
    dev = S["rhogq"].device
    m = torch.as_tensor(g.interior_mask(), device=dev)
    kk = slice(g.kmin - 1, g.kmax)
    area = torch.as_tensor(g.arrays["GMTR_p"][0], device=dev)
    dz = torch.as_tensor(g.arrays["dz"], device=dev)
    apl = torch.as_tensor(g.arrays["GMTR_p_pl"][0][:, 0], device=dev)
    a = (S["rhogq"][:, :, kk] * (area * m)[None, :, None] * dz[kk][None, None, :, None]).sum((1, 2, 3))
    return a + (S["rhogq_pl"][:, :, kk, 0] * apl[None, :, None] * dz[kk][None, None]).sum((1, 2))


def run_uneven(args, world, rank, local):
    """`--mode uneven`: the uneven batch (measure_uneven) as the line's workload."""
    out = measure_uneven(args, local)
    if rank == 0:
        line = {"metric": METRIC, "value": out["value"], "unit": UNIT, "n_gpus": world, "steps": out["steps"],
                "warmup": args.warmup, "ms_per_step": out["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": out["config"]}
        line.update({k: v for k, v in out.items() if k not in ("value", "ms_per_step", "steps", "config")})
        print(json.dumps(line), flush=True)


def measure_uneven(args, local):
    """Batch of two uneven grid instances (glevel 7 / kall 96 / 40 tracers and glevel 6 / kall 42 /
    12 tracers) advanced by the same launches and replayed from a CUDA graph, in the FP32 variant
    (`value`) and the FP64 variant (`fp64_variant`).  Each reports its max relative error
    against the plain FP64 step after one step and the relative mass drift over the timed
    steps; the plain FP64 step of both instances is timed beside them."""
    import torch

    from icoatmosbenchmark_v1_b200 import api
    from icoatmosbenchmark_v1_b200 import fields as F
    from icoatmosbenchmark_v1_b200.grid import Grid, default_dt
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    grids = [Grid(gl, 0, K) for gl, K, _ in UNEVEN]
    fs, sts, ctxs, dts = [], [], [], []
    for g, (gl, K, T) in zip(grids, UNEVEN):
        f = F.make_fields(g, device=dev)
        st = F.make_state(g, T, "mixed", device=dev, fields=f)
        ctx = api.IcoAdv(gl, 0, K - 2, device=local)
        ctx.set_grid(g)
        fs.append(f), sts.append(st), ctxs.append(ctx), dts.append(default_dt(gl))
    upd = sum((10 * 4 ** gl + 2) * K * T for gl, K, T in UNEVEN)

    def masses(states):
        return [tracer_mass(g, S) for g, S in zip(grids, states)]

    # FP64 variant (plain path) for one step: the error reference, and its time (after a
    # warm-up step on a copy, which sets up its buffers)
    for ctx, st, f, dt in zip(ctxs, sts, fs, dts):
        S = {k: v.clone() for k, v in st.items()}
        ctx.advect_step(dt, S["rhog"], S["rhog_pl"], S["rhogq"], S["rhogq_pl"], f["rhogvx"], f["rhogvx_pl"],
                        f["rhogvy"], f["rhogvy_pl"], f["rhogvz"], f["rhogvz_pl"], f["rhogw"], f["rhogw_pl"])
        del S
    ref = [{k: v.clone() for k, v in st.items()} for st in sts]
    init = [{k: v.clone() for k, v in st.items()} for st in sts]  # the FP32 runner advances sts in place
    torch.cuda.synchronize()
    t64 = time.perf_counter()
    for ctx, S, f, dt in zip(ctxs, ref, fs, dts):
        ctx.advect_step(dt, S["rhog"], S["rhog_pl"], S["rhogq"], S["rhogq_pl"], f["rhogvx"], f["rhogvx_pl"],
                        f["rhogvy"], f["rhogvy_pl"], f["rhogvz"], f["rhogvz_pl"], f["rhogw"], f["rhogw_pl"])
    torch.cuda.synchronize()
    ms64 = (time.perf_counter() - t64) * 1e3
    # tile shape: the fastest over two direct steps each
    best, tuning = None, []
    for shape in range(len(ctxs[0].fast_shapes())):
        br = api.BatchRunner(ctxs, [{k: v.clone() for k, v in st.items()} for st in sts], fs, dts, shape=shape)
        br.step()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        br.step(), br.step()
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 500.0
        tuning.append(round(ms, 3))
        if best is None or ms < best[1]:
            best = (shape, ms)
        br.close()
        del br
    br = api.BatchRunner(ctxs, sts, fs, dts, shape=best[0])
    m0 = masses(br.states)
    br.step()
    torch.cuda.synchronize()
    err = max(float(((a["rhogq"] - b["rhogq"]).abs().max() / b["rhogq"].abs().max()).item())
              for a, b in zip(br.states, ref))
    br.use_graph()
    for _ in range(args.warmup):
        br.step()
    stream = torch.cuda.ExternalStream(ctxs[0].stream, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(local)
    sampler.start()
    torch.cuda.synchronize()
    n0 = sum(c.launch_count for c in ctxs)
    e0.record(stream)
    for _ in range(args.steps):
        br.step()
    e1.record(stream)
    launches = sum(c.launch_count for c in ctxs) - n0
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1) / args.steps
    m1 = masses(br.states)
    drift = max(float(((b - a).abs() / a.abs()).max().item()) for a, b in zip(m0, m1))
    br.close()
    del br
    torch.cuda.empty_cache()
    # FP64 variant of the same batch: the same launches in FP64 (fields, faces, limiters)
    b64 = api.BatchRunner(ctxs, init, fs, dts, shape=best[0], f64=True)
    m0 = masses(b64.states)
    b64.step()
    torch.cuda.synchronize()
    err64 = max(float(((a["rhogq"] - b["rhogq"]).abs().max() / b["rhogq"].abs().max()).item())
                for a, b in zip(b64.states, ref))
    b64.use_graph()
    for _ in range(args.warmup):
        b64.step()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        b64.step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms_f64 = e0.elapsed_time(e1) / args.steps
    m1 = masses(b64.states)
    drift64 = max(float(((b - a).abs() / a.abs()).max().item()) for a, b in zip(m0, m1))
    b64.close()
    shape = list(ctxs[0].fast_shapes()[best[0]])
    out = {"value": upd / (ms * 1e-3), "unit": UNIT, "steps": args.steps, "ms_per_step": ms, "dtype": "f32",
           "config": {"workload": "uneven_gl7_k96_t40+gl6_k42_t12", "instances": [list(x) for x in UNEVEN],
                      "updates_per_step": upd, "launch": "one launch per stage over both instances, "
                      "persistent horizontal kernel, step replayed from a CUDA graph",
                      "tile": {"shape_txtytg": shape, "autotune_ms": tuning}},
           "fp64_plain_ms_per_step": ms64, "max_rel_err_vs_fp64": err,
           "mass_drift": {"value": drift, "steps": args.steps + args.warmup},
           "fp64_variant": {"ms_per_step": ms_f64, "value": upd / (ms_f64 * 1e-3),
                            "max_rel_err_vs_fp64_plain": err64,
                            "mass_drift": {"value": drift64, "steps": 1 + args.steps + args.warmup}},
           "gpu_launches": launches, "clocks": clocks}
    for c in ctxs:
        c.close()
    return out


def measure_adjoint(args, local, fast_ms=None, steps=12, every=4):
    """Adjoint of the plain FP64 step over a checkpointed run, on this GPU alone: the FP64
    forward timed over `steps` steps, then ica_adjoint_record (the same steps, a checkpoint
    every `every`) and ica_adjoint_sweep (segments recomputed from their checkpoints and
    transposed step by step), each timed with CUDA events on the context stream.  The adjoint
    is seeded with J = sum of squared q over region 0, levels 10-20."""
    import torch

    from icoatmosbenchmark_v1_b200 import api
    from icoatmosbenchmark_v1_b200 import fields as F
    from icoatmosbenchmark_v1_b200.grid import Grid, default_dt

    dev = torch.device("cuda", local)
    g = Grid(args.glevel, 0, args.kall)
    dt = default_dt(args.glevel)
    f = F.make_fields(g, device=dev)
    st = F.make_state(g, args.ntr, "mixed", device=dev, fields=f)
    del f["rhog"], f["rhog_pl"]
    torch.cuda.synchronize()
    torch.cuda.empty_cache()  # temporaries of the state set-up
    ctx = api.IcoAdv(args.glevel, 0, args.kall - 2, device=local)
    ctx.set_grid(g)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    a = {k: torch.zeros_like(v) for k, v in st.items()}
    aw = {k: torch.zeros_like(f[k]) for k in api.WIND_KEYS}
    kr = slice(9, 20)  # levels 10-20

    def seed():
        for v in a.values():
            v.zero_()
        q = st["rhogq"][:, 0, kr] / st["rhog"][None, 0, kr]
        a["rhogq"][:, 0, kr] = 2 * q / st["rhog"][None, 0, kr]
        a["rhog"][0, kr] = -(2 * q * q / st["rhog"][None, 0, kr]).sum(0)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    def fwd(n):
        for _ in range(n):
            ctx.advect_step(dt, st["rhog"], st["rhog_pl"], st["rhogq"], st["rhogq_pl"], f["rhogvx"], f["rhogvx_pl"],
                            f["rhogvy"], f["rhogvy_pl"], f["rhogvz"], f["rhogvz_pl"], f["rhogw"], f["rhogw_pl"])

    fwd(1)  # warm
    # warm the adjoint: allocates the scratch and the segment states
    ctx.adjoint_record(dt, every, every, st, f)
    seed()
    ctx.adjoint_sweep(f, a, aw)
    t_fwd = timed(lambda: fwd(steps))
    t_rec = timed(lambda: ctx.adjoint_record(dt, steps, every, st, f))
    seed()
    n1 = ctx.launch_count
    t_sweep = timed(lambda: ctx.adjoint_sweep(f, a, aw))
    launches = ctx.launch_count - n1
    free_gb = torch.cuda.mem_get_info(dev)[0] / 1e9
    finite = all(bool(torch.isfinite(v.sum()).item()) for v in (a["rhogq"], a["rhog"], aw["rhogvx"], aw["rhogvy"],
                                                                 aw["rhogvz"]))
    ctx.adjoint_release()
    ctx.close()
    del st, f, a, aw
    torch.cuda.empty_cache()
    out = {"workload": f"gl{args.glevel}_k{args.kall}_t{args.ntr}: {steps}-step sweep, checkpoint every {every}",
           "objective": "sum of squared q over region 0, levels 10-20", "dtype": "f64",
           "forward_fp64_ms_per_step": t_fwd / steps, "record_ms": t_rec, "sweep_ms": t_sweep,
           "sweep_ms_per_step": t_sweep / steps, "ratio_vs_fp64_forward": t_sweep / t_fwd,
           "gpu_launches_sweep": launches, "gradients_finite": finite,
           "device_free_gb_during_sweep": round(free_gb, 1)}
    if fast_ms:
        out["ratio_vs_batched_forward"] = t_sweep / (steps * fast_ms)
    return out


def measure_e2e(args, ctx, g, st, f, dt, upd, world):
    """Per step: pinned host -> device copy of the state and fields, the step, device -> host copy of
    the state, all inside one host-pointer C ABI call (ica_advect_step / ica_advect_fast)."""
    import numpy as np
    import torch
    n = max(1, min(args.steps, args.e2e_steps))
    host = {k: v.cpu().pin_memory() for k, v in st.items()}
    hf = {k: v.cpu().pin_memory() for k, v in f.items()}
    if args.mode != "plain":  # the batched path takes FP32 fields
        hf = {k: v.to(torch.float32).pin_memory() for k, v in hf.items()}
    hn = {k: v.numpy() for k, v in host.items()}
    hfn = {k: v.numpy() for k, v in hf.items()}
    h2d = sum(v.numel() * v.element_size() for v in host.values()) + sum(
        v.numel() * v.element_size() for v in hf.values())
    d2h = sum(v.numel() * v.element_size() for v in host.values())
    call = ctx.advect_step if args.mode == "plain" else ctx.advect_fast_host
    if args.mode != "plain":
        ctx.fast_set_host_chunk(args.host_chunk)
    call(dt, **_step_kwargs(hn, hfn))  # warm (allocates staging once)
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(n):
        call(dt, **_step_kwargs(hn, hfn))
    el = (time.perf_counter() - t0) / n
    el = allreduce_max(el, world)
    return {"value": upd * world / el, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "steps": n, "ms_per_step": el * 1e3}


def _step_kwargs(s, f):
    return dict(rhog=s["rhog"], rhog_pl=s["rhog_pl"], rhogq=s["rhogq"], rhogq_pl=s["rhogq_pl"],
                rhogvx=f["rhogvx"], rhogvx_pl=f["rhogvx_pl"], rhogvy=f["rhogvy"], rhogvy_pl=f["rhogvy_pl"],
                rhogvz=f["rhogvz"], rhogvz_pl=f["rhogvz_pl"], rhogw=f["rhogw"], rhogw_pl=f["rhogw_pl"])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--mode", choices=["fast", "plain", "uneven", "adjoint"], default="fast",
                    help="fast: batched step (headline, followed by the adjoint sweep); plain: FP64 per-tracer "
                         "path; uneven: batch of two grid levels; adjoint: the adjoint sweep alone")
    ap.add_argument("--glevel", type=int, default=8)
    ap.add_argument("--kall", type=int, default=96)
    ap.add_argument("--ntr", type=int, default=32)
    ap.add_argument("--ref-kall", type=int, default=12,
                    help="kall of the CPU sample (same grid level and tracers, fewer levels per step)")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-check", action="store_true", help="skip the error / mass-drift check")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint sweep measurement")
    ap.add_argument("--shard", action="store_true",
                    help="shard the grid's regions over the ranks (NCCL exchanges) instead of running replicas")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the FP64 variant and the uneven batch (extra keys of the default line)")
    ap.add_argument("--adjoint-steps", type=int, default=12, help="steps of the adjoint sweep")
    ap.add_argument("--adjoint-every", type=int, default=4, help="checkpoint interval of the adjoint sweep")
    ap.add_argument("--tile-shape", type=int, default=-1, help="tile shape index of the horizontal kernel (default: autotune)")
    ap.add_argument("--host-chunk", type=int, default=0,
                    help="tracers per chunk of the host-pointer step's overlapped copies (default 0: by size)")
    ap.add_argument("--traffic", type=float, default=None,
                    help="ncu dram bytes per launch of the dominant kernel, if measured")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference_arm(args, world, rank)
        elif args.mode == "uneven":
            run_uneven(args, world, rank, local)
        elif args.mode == "adjoint":
            import torch
            torch.cuda.set_device(local)
            if rank == 0:
                print(json.dumps({"adjoint": measure_adjoint(args, local, steps=args.adjoint_steps,
                                                             every=args.adjoint_every)}), flush=True)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
