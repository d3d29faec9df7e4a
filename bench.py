#!/usr/bin/env python
"""Benchmark of the B200 Bohrium vector engine.

Headline (one JSON line on rank 0): the Black-Scholes workload -- 10M float64 options,
S~U(5,30), K~U(1,100), T~U(0.25,10), r=0.02, vol=0.3, erf-based normal CDF -- run as 10 flushes
per step, each flush one iteration ending in a mean-price reduction. `value` is the algorithmic HBM
throughput of the flushes with the inputs resident in device memory (bytes of S, K and T read per
flush plus the result written, over the device time of the timed steps). `e2e` is the same metric
through the C ABI with the inputs handed over from page-locked host buffers every step and the 10
mean prices read back. `cpu_baseline` is the oracle (the restated ve/openmp engine) on the host
cores. `extra` adds the other workloads (plain chain, heat stencil, batching, streaming block,
axpy, transpose-add, scan, learned fuser); they are single-GPU measurements and run at N = 1 only.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--no-extra]

With N > 1 (torchrun) every rank runs the same workload on its own GPU ("replicas only": the path
has no data exchange between GPUs) and `value` is the sum over ranks divided by the slowest rank.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "flush wall-time & HBM GB/s (%peak): batched+learned vs plain ve/cuda; vs ve/openmp"
BS_OPTIONS = 10_000_000
BS_ITERS = 10
# DRAM bytes (read + written) per option of one Black-Scholes kernel launch, from an ncu capture
# of a 6,000,000-option launch (dram__bytes_read.sum 144.08 MB + dram__bytes_write.sum 4.84 MB;
# inputs of 144 MB, larger than L2): one pass over the three inputs plus the tile partials, so
# the traffic grows in proportion to the options and is scaled to the launch's option count.
BS_TRAFFIC_PER_OPTION = (144_081_152 + 4_843_776) / 6_000_000
# FP64 instructions per option of the same launch: sm__inst_executed_pipe_fp64.sum (28,608,514
# warp instructions) x 32 lanes / 6,000,000 options. The same capture shows the FP64 pipe
# 52.1 % busy over the kernel's active cycles (sm__inst_executed_pipe_fp64 pct_of_peak_sustained_active).
BS_FP64_PER_OPTION = 28_608_514 * 32 / 6_000_000
BS_FP64_PIPE_NCU = 0.521
# FP64 lanes per SM per clock on B200: the capture's 193,301 FP64 warp instructions per SM at
# 52.12 % of peak over 185,430 active cycles give 2.0 warp instructions (64 lanes) per cycle.
FP64_LANES_PER_SM = 64
SM_COUNT = 148


# Warm-up executions of every extra workload before its timed ones: enough for the autotuner to
# time all variants of a large kernel (3 launches each) and settle on one.
EXTRA_WARMUP = 20


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------------------------ clocks
class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv",
                                          "-lms", "50"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.15)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        try:
            lines = open(self.path).read().strip().splitlines()[1:]
        except OSError:
            lines = []
        for ln in lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1].split()[0]))
                mx = float(f[2].split()[0])
            except ValueError:
                continue
            for name, v in zip(["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"], f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if self.path:
            os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------------------- distributed
def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allreduce_max(world, x: float) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------------------------ workloads
def build_black_scholes(bh, W, rt, ex, n, pinned=False):
    S, K, T = W.black_scholes_inputs(n, 0)
    arrays, hosts = [], []
    for x in (S, K, T):
        a = bh.empty(rt, (n,), np.float64)
        if pinned:
            hosts.append(ex.set_pinned(a.base, x))
        else:
            ex.set_data(a.base, x)
        arrays.append(a)
    s, k, t = arrays
    rt.flush()
    irs, outs = [], []
    for it in range(BS_ITERS):
        m = W.black_scholes_iteration(rt, s, k, t, it)
        flush = rt.take()
        irs.append(ex.compile(flush))
        outs.append(m)
    return (s, k, t), hosts, irs, outs, (S, K, T)


def bs_bytes(n):
    return 3 * 8 * n + 8


def stats(ex) -> dict:
    out = {}
    for line in ex.message("statistic").splitlines():
        if ":" in line and not line.startswith(" "):
            k, v = line.split(":", 1)
            try:
                out[k.strip()] = float(v)
            except ValueError:
                pass
    return out


def sync_read(bh, ex, outs):
    """One flush that syncs every result base, then read the host copies."""
    ex.execute(bh.ir.Flush([], syncs=[o.base for o in outs]))
    return [ex.lib.bhb_base_data(o.base.handle) for o in outs]


def run_ours(args, world, rank, local):
    os.environ["BH_CUDA_DEVICE_NUMBER"] = str(local)
    import bohrium_b200 as bh
    from bohrium_b200 import workloads as W
    ex = bh.NativeExecutor()
    rt = bh.Runtime(ex)
    peak, peak_kind = peaks()

    # ---- device-resident throughput -----------------------------------------------------
    n = args.bs_options
    inputs, _, irs, outs, host_inputs = build_black_scholes(bh, W, rt, ex, n)
    step = lambda: [ir.execute() for ir in irs]
    # The clock sampler runs from the warm-up through the timed steps (all under load): the timed
    # region alone can be shorter than a sampling interval.
    with Clocks(local) as clk:
        for _ in range(max(args.warmup, 3)):
            step()
        ex.message("CUDA: sync")
        barrier(world)
        launches0 = int(ex.message("CUDA: launches"))
        host0 = stats(ex)
        ex.message("CUDA: timer start")
        t0 = time.perf_counter()
        for _ in range(args.steps):
            step()
        dev_ms = float(ex.message("CUDA: timer stop"))
        wall = time.perf_counter() - t0
    launches = int(ex.message("CUDA: launches")) - launches0
    host1 = stats(ex)
    clocks = clk.summary()
    nflush = args.steps * BS_ITERS
    host_us = {k: round((host1.get(k, 0) - host0.get(k, 0)) * 1e6 / nflush, 2)
               for k in ("time_exec_host", "time_prepare", "time_launch")}
    # Per-launch kernel durations with CUDA events (one profiled step after the timed region).
    ex.message("CUDA: prof on")
    ex.message("statistic_enable_and_reset")
    step()
    ex.message("CUDA: sync")
    stat = ex.message("statistic")
    ex.message("CUDA: prof off")
    per_kernel = {}
    for line in stat.splitlines():
        if line.strip().startswith("- {name"):
            name = line.split("name:")[1].split(",")[0].strip()
            per_kernel.setdefault(name, []).append(float(line.split("ms:")[1].strip(" }")))
    # the dominant kernel: the one with the largest total device time
    kernel_ms = max(per_kernel.values(), key=sum) if per_kernel else []
    dev_ms_max = allreduce_max(world, dev_ms)
    bytes_step = BS_ITERS * bs_bytes(n)
    value = world * bytes_step * args.steps / (dev_ms_max / 1e3) / 1e9
    got = [float(v) for v in (ex.peek(o.base)[0] for o in outs[:3])]
    want = [W.black_scholes_numpy(*host_inputs, it) for it in range(3)] if rank == 0 else got
    check_ok = all(abs(g - w) <= 1e-10 * abs(w) for g, w in zip(got, want))
    avg_kernel_ms = statistics.mean(kernel_ms) if kernel_ms else dev_ms / args.steps / BS_ITERS
    achieved = bs_bytes(n) / (avg_kernel_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": round(BS_TRAFFIC_PER_OPTION * n),
                "traffic_source": "ncu DRAM bytes of a 6e6-option launch, scaled to the launch's options",
                "peak_kind": peak_kind,
                "kernel": "bh_grid_reduce (Black-Scholes flush)", "kernel_ms": round(avg_kernel_ms, 5),
                "algorithmic_bytes_per_launch": bs_bytes(n)}
    # The kernel's real ceiling is the FP64 pipe, not HBM: FP64 instructions per launch over the
    # kernel time, against 64 lanes x 148 SMs at the SM clock sampled during the timed region.
    mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 1965.0
    fp64_achieved = BS_FP64_PER_OPTION * n / (avg_kernel_ms / 1e3) / 1e9
    fp64_peak = FP64_LANES_PER_SM * SM_COUNT * mhz / 1e3
    roofline["fp64"] = {"unit": "G FP64 lane-instructions/s", "per_option": round(BS_FP64_PER_OPTION, 1),
                        "achieved": round(fp64_achieved, 1), "peak": round(fp64_peak, 1),
                        "frac": round(fp64_achieved / fp64_peak, 4), "sm_mhz": mhz,
                        "ncu_pipe_active_6e6": BS_FP64_PIPE_NCU,
                        "source": "per-option count and pipe share from an ncu capture of a 6e6-option launch"}
    del irs, outs, inputs

    # ---- end to end through the C ABI with page-locked host buffers ---------------------
    # Every step hands page-locked host inputs (240 MB) to the engine with bhb_data_set, runs the
    # 10 flushes and reads the 10 means back. Two forms:
    #   serial     a step hands over its own inputs, then computes on them;
    #   pipelined  two input sets alternate: a step hands over the NEXT step's inputs before running
    #              its own flushes, so the engine's eager upload (a copy stream) overlaps them. The
    #              clock stops after the last upload has landed, so the timed region holds exactly
    #              one 240 MB upload and one read-back per step.
    sets = [build_black_scholes(bh, W, rt, ex, n, pinned=True) for _ in range(2)]

    def hand_over(st):
        (s_, k_, t_), hosts, _, _, _ = st
        for arr, h in zip((s_, k_, t_), hosts):
            if ex.lib.bhb_data_set(ex.rt, arr.base.handle, 1, h.ctypes.data) != 0:  # new host data: re-upload
                raise RuntimeError("bhb_data_set failed")

    def run_set(st):
        for ir in st[2]:
            ir.execute()
        return sync_read(bh, ex, st[3])

    def serial_step():
        hand_over(sets[0])
        return run_set(sets[0])

    cur = [0]

    def pipelined_step():
        hand_over(sets[1 - cur[0]])
        r = run_set(sets[cur[0]])
        cur[0] = 1 - cur[0]
        return r

    def timed(step_fn, prime=None):
        if prime:
            prime()
        for _ in range(2):
            step_fn()
        ex.message("CUDA: sync")
        barrier(world)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            step_fn()
        ex.message("CUDA: sync")  # both streams: the last upload has landed
        return allreduce_max(world, time.perf_counter() - t0)

    e2e_serial_s = timed(serial_step)
    e2e_s = timed(pipelined_step, prime=lambda: hand_over(sets[0]))
    want_means = [W.black_scholes_numpy(*sets[0][4], it) for it in range(2)] if rank == 0 else None
    got_means = [float(v) for v in (ex.peek(o.base)[0] for o in sets[0][3][:2])]
    e2e_check = rank != 0 or all(abs(g - w) <= 1e-10 * abs(w) for g, w in zip(got_means, want_means))
    e2e = {"value": round(world * bytes_step * args.steps / e2e_s / 1e9, 2), "unit": "GB/s",
           "h2d_bytes_per_step": 3 * 8 * n, "d2h_bytes_per_step": 8 * BS_ITERS,
           "ms_per_step": round(e2e_s * 1e3 / args.steps, 3), "form": "pipelined",
           "serial": {"value": round(world * bytes_step * args.steps / e2e_serial_s / 1e9, 2),
                      "ms_per_step": round(e2e_serial_s * 1e3 / args.steps, 3)},
           "result_check": e2e_check,
           "note": "pipelined: the next step's inputs are handed over before this step's flushes and "
                   "uploaded on the engine's copy stream while they run; serial: hand-over, upload, "
                   "flushes, read-back in turn"}
    del sets

    extra = {}
    # The other workloads are single-GPU measurements: they run at N = 1 only (under torchrun the
    # other ranks would wait for rank 0 at the final barrier for the whole of them).
    if args.extra and rank == 0 and world == 1:
        extra = run_extra(bh, W, ex, rt, peak, heat_n=args.heat_n, learned_train=args.learned_train,
                          learned_eval=args.learned_eval, learned_holdout=args.learned_holdout)

    cpu = None
    if rank == 0 and world == 1 and args.cpu_baseline:
        cpu = cpu_baseline(n=args.cpu_options)

    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(dev_ms_max / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded uniform inputs)",
        "config": {"workload": "black_scholes_f64_10M_options_x10_flushes", "options": n, "flushes_per_step": BS_ITERS,
                   "bytecodes_per_flush": 44, "l2": "inputs (240 MB) larger than L2",
                   "parallelism": "replicas" if world > 1 else "single GPU",
                   "flush_ms_device": round(dev_ms_max / args.steps / BS_ITERS, 4),
                   "flush_ms_wall": round(wall * 1e3 / args.steps / BS_ITERS, 4),
                   "frac_of_peak": round(value / world / peak, 4), "result_check": check_ok,
                   "host_us_per_flush": host_us},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clocks,
    }
    if extra:
        line["extra"] = extra
    if rank == 0:
        print(json.dumps(line), flush=True)


def extra_plain_chain(bh, W, ex, rt, out):
    """The plain chain over three float64 arrays of 2^20 elements. Its 25 MB working set fits in
    L2, so before every timed flush another flush writes a 512 MB array (four times L2), and only
    the chain's flush is timed: the GB/s are HBM figures."""
    n = 1 << 20
    A, B, C = W.plain_chain_inputs(n, 0)
    a, b, c = (bh.array(rt, x) for x in (A, B, C))
    rt.flush()
    r = W.plain_chain(rt, a, b, c)
    ir = ex.compile(rt.take())
    junk = bh.zeros(rt, (1 << 27,), np.float32)
    rt.flush()
    junk2 = junk + np.float32(1)
    evict = ex.compile(rt.take())
    for _ in range(EXTRA_WARMUP):
        ir.execute()
    reps = 50
    cold = []
    for _ in range(reps):
        evict.execute()
        ex.message("CUDA: sync")
        ex.message("CUDA: timer start")
        ir.execute()
        cold.append(float(ex.message("CUDA: timer stop")))
    ms = statistics.median(cold)
    reps = 200
    ex.message("CUDA: sync")
    ex.message("CUDA: timer start")
    t0 = time.perf_counter()
    for _ in range(reps):
        ir.execute()
    warm_ms = float(ex.message("CUDA: timer stop")) / reps
    wall = (time.perf_counter() - t0) * 1e3 / reps
    out["plain_chain_f64_2^20"] = {"flush_ms_device": round(ms, 4), "GB/s": round((3 * 8 * n + 8) / (ms / 1e3) / 1e9, 1),
                                   "l2": "evicted before every timed flush (512 MB written); median of 50",
                                   "l2_resident": {"flush_ms_device": round(warm_ms, 4), "flush_ms_wall": round(wall, 4),
                                                   "note": "back-to-back flushes, 25 MB in L2: launch-bound, not an HBM figure"}}
    del ir, r, a, b, c, evict, junk2, junk


def extra_transpose(bh, W, ex, rt, out, n=8192):
    """C = A + B^T over float32 n x n (12 B per element: A and B read, C written; 805 MB per
    flush at n = 8192). B is read through a transposed view."""
    A = bh.random_sample(rt, (n, n), start=3, key=21, dtype=np.float32)
    B = bh.random_sample(rt, (n, n), start=4, key=22, dtype=np.float32)
    rt.flush()
    C = A + B.T
    ir = ex.compile(rt.take())
    for _ in range(EXTRA_WARMUP):
        ir.execute()
    ex.message("CUDA: sync")
    reps = 10
    ex.message("CUDA: timer start")
    for _ in range(reps):
        ir.execute()
    ms = float(ex.message("CUDA: timer stop")) / reps
    a, b, c = (ex.peek(x.base).reshape(n, n) for x in (A, B, C))
    ok = bool(np.array_equal(c[:: 97, :: 89], (a + b.T)[:: 97, :: 89]))
    gbs = 12 * n * n / (ms / 1e3) / 1e9
    out["transpose_add_f32_%d^2" % n] = {"flush_ms_device": round(ms, 4), "GB/s": round(gbs, 1),
                                         "frac_of_peak": round(gbs / peaks()[0], 3), "result_check": ok}
    del ir, A, B, C


def extra_heat(bh, W, ex, rt, out, n=4096):
    """2-D heat stencil, float32 n^2, 100 iterations as one flush repeated 50 times over a
    two-step (a->b, b->a) bytecode; device time per 100 iterations, the mean of 5 such flushes."""
    g = W.heat_grid(n, 0)
    ga, gb = bh.array(rt, g), bh.array(rt, g)
    d1 = W.heat_step(ga, gb)
    d2 = W.heat_step(gb, ga)
    rt.flush()
    # rebuild the same two steps as a repeatable flush
    d1 = W.heat_step(ga, gb)
    d2 = W.heat_step(gb, ga)
    flush = rt.take()
    flush.nrepeats = 50
    ir = ex.compile(flush)
    for _ in range(3):  # 300 launches: past the autotuner's variant timings
        ir.execute()
    ex.message("CUDA: sync")
    reps = 5
    ex.message("CUDA: timer start")
    t0 = time.perf_counter()
    for _ in range(reps):
        ir.execute()
    ms = float(ex.message("CUDA: timer stop")) / reps
    wall = (time.perf_counter() - t0) * 1e3 / reps
    per_iter = (n * n * 4 + (n - 2) * (n - 2) * 4)
    out[f"heat_f32_{n}^2_x100"] = {"flush_ms_device": round(ms, 3), "flush_ms_wall": round(wall, 3),
                                   "GB/s": round(100 * per_iter / (ms / 1e3) / 1e9, 1),
                                   "iterations": 100}
    del ir, d1, d2, ga, gb


def extra_batching(bh, W, ex, rt, out):
    """4096 float32 systems of uneven length in one flush, plain vs grouped launches."""
    lengths = W.batching_lengths(4096, 256, 65536, 0)
    xs = []
    for i, L in enumerate(lengths):
        f = bh.random_sample(rt, (int(L),), start=int(i) << 32, key=7, dtype=np.float32)
        xs.append(f)
    rt.flush()
    outs = []
    for x in xs:
        y = W.batching_chain(x)
        outs += [y, y.sum(), y.max()]
    ir = ex.compile(rt.take())
    total = int(lengths.sum())
    res = {}
    for mode in ["off", "grouped", "graph"]:
        ex.message(f"CUDA: batch {mode}")
        for _ in range(EXTRA_WARMUP):
            ir.execute()
        ex.message("CUDA: sync")
        l0 = int(ex.message("CUDA: launches"))
        h0 = stats(ex)
        reps = 5
        ex.message("CUDA: timer start")
        t0 = time.perf_counter()
        for _ in range(reps):
            ir.execute()
        ms = float(ex.message("CUDA: timer stop")) / reps
        wall = (time.perf_counter() - t0) * 1e3 / reps
        res[mode] = {"flush_ms_device": round(ms, 3), "flush_ms_wall": round(wall, 3),
                     "launches_per_flush": (int(ex.message("CUDA: launches")) - l0) // reps,
                     "host_ms_per_flush": None,
                     "GB/s": round((8 * total + 8 * 4096) / (max(ms, wall) / 1e3) / 1e9, 1)}
        h1 = stats(ex)
        res[mode]["host_ms_per_flush"] = {k: round((h1.get(k, 0) - h0.get(k, 0)) * 1e3 / reps, 3)
                                          for k in ("time_exec_host", "time_prepare", "time_launch")}
    ex.message("CUDA: batch off")
    # bit-identical results between the forms (every output of every system)
    got = {}
    for mode in ["graph", "grouped", "off"]:
        ex.message(f"CUDA: batch {mode}")
        ir.execute()
        ir.execute()
        got[mode] = [ex.peek(o.base).tobytes() for o in outs]
    ex.message("CUDA: batch off")
    res["bit_identical"] = got["graph"] == got["off"] and got["grouped"] == got["off"]
    res["speedup_wall"] = round(res["off"]["flush_ms_wall"] / res["grouped"]["flush_ms_wall"], 2)
    res["speedup_wall_graph"] = round(res["off"]["flush_ms_wall"] / res["graph"]["flush_ms_wall"], 2)
    res["systems"] = 4096
    res["elements"] = total
    out["batching_4096_systems_f32"] = res


def extra_stream(bh, W, ex, rt, out, n=100_000_000):
    """One fused streaming block on a large array: the 12-operation float32 chain of the batching
    workload over 1e8 elements, keeping y and reducing sum(y) and max(y) (8 B per element)."""
    x = bh.random_sample(rt, (n,), start=0, key=7, dtype=np.float32)
    rt.flush()
    y = W.batching_chain(x)
    outs = [y, y.sum(), y.max()]
    ir = ex.compile(rt.take())
    for _ in range(EXTRA_WARMUP):
        ir.execute()
    ex.message("CUDA: sync")
    reps = 10
    ex.message("CUDA: timer start")
    for _ in range(reps):
        ir.execute()
    ms = float(ex.message("CUDA: timer stop")) / reps
    ex.message("CUDA: prof on")
    ex.message("statistic_enable_and_reset")
    ir.execute()
    ex.message("CUDA: sync")
    stat = ex.message("statistic")
    ex.message("CUDA: prof off")
    kernels = [line for line in stat.splitlines() if line.strip().startswith("- {name")]
    k_ms = max((float(k.split("ms:")[1].strip(" }")) for k in kernels), default=ms)
    name = max(kernels, key=lambda k: float(k.split("ms:")[1].strip(" }"))).split("name:")[1].split(",")[0].strip() \
        if kernels else ""
    bytes_ = 8 * n + 8
    out["stream_f32_1e8"] = {"flush_ms_device": round(ms, 4), "GB/s": round(bytes_ / (ms / 1e3) / 1e9, 1),
                             "kernel": name, "kernel_ms": round(k_ms, 4),
                             "kernel_GB/s": round(bytes_ / (k_ms / 1e3) / 1e9, 1),
                             "frac_of_peak": round(bytes_ / (k_ms / 1e3) / 1e9 / peaks()[0], 3),
                             "launches_per_flush": len(kernels)}
    del ir, outs, x


def extra_axpy(bh, W, ex, rt, out, n=200_000_000):
    """A memory-bound fused map: z = 2.5 * x + y over 2e8 float32 (FLAT, 12 B per element:
    x and y read, z written)."""
    x = bh.random_sample(rt, (n,), start=1, key=11, dtype=np.float32)
    y = bh.random_sample(rt, (n,), start=2, key=12, dtype=np.float32)
    rt.flush()
    z = x * np.float32(2.5) + y
    ir = ex.compile(rt.take())
    for _ in range(EXTRA_WARMUP):
        ir.execute()
    ex.message("CUDA: sync")
    reps = 10
    ex.message("CUDA: timer start")
    for _ in range(reps):
        ir.execute()
    ms = float(ex.message("CUDA: timer stop")) / reps
    gbs = 12 * n / (ms / 1e3) / 1e9
    out["axpy_f32_2e8"] = {"flush_ms_device": round(ms, 4), "GB/s": round(gbs, 1),
                           "frac_of_peak": round(gbs / peaks()[0], 3)}
    del ir, z, x, y


def extra_scan(bh, W, ex, rt, out, n=50_000_000):
    """A fused 1-D cumulative sum (SCAN1D): y = cumsum(2x + 1) over 5e7 float64 (8 B read + 8 B
    written per element, algorithmically)."""
    x = bh.random_sample(rt, (n,), start=5, key=3, dtype=np.float64)
    rt.flush()
    y = bh.accumulate("ADD_ACCUMULATE", x * 2.0 + 1.0, 0)
    ir = ex.compile(rt.take())
    for _ in range(EXTRA_WARMUP):
        ir.execute()
    ex.message("CUDA: sync")
    reps = 10
    ex.message("CUDA: timer start")
    for _ in range(reps):
        ir.execute()
    ms = float(ex.message("CUDA: timer stop")) / reps
    out["scan_f64_5e7"] = {"flush_ms_device": round(ms, 4), "GB/s": round(16 * n / (ms / 1e3) / 1e9, 1),
                           "frac_of_peak": round(16 * n / (ms / 1e3) / 1e9 / peaks()[0], 3)}
    del ir, y, x


def extra_learned(bh, W, ex, rt, out, train_seeds=24, eval_seeds=12, holdout_seeds=48):
    """The learned-fuser workload: seeded random bytecode DAGs (50-400 operations, 1e3-1e8
    elements, float32/float64/int32, transposed/reversed/broadcast views, 0-3 reductions). The
    engine records per-kernel device times on the training DAGs, the cost model is trained on the
    GPU, its prediction error is measured on the recorded kernels of other DAGs (held out), and
    held-out DAGs are timed under the plain engine (greedy plan, one launch per kernel), the
    batched engine (CUDA-graph replay) and the batched + learned engine."""
    from bohrium_b200 import learn
    t0 = time.perf_counter()
    X, t = learn.collect(ex, seeds=range(train_seeds), max_elems=1e7)
    t1 = time.perf_counter()
    model, loss = learn.train(X, t, epochs=300)
    t2 = time.perf_counter()
    train_s = t2 - t1
    Xh, th = learn.collect(ex, seeds=range(5000, 5000 + holdout_seeds), max_elems=1e7, variants=learn.VARIANTS[:2])
    holdout = learn.holdout_error(model, Xh, th)
    holdout.update({"dags": holdout_seeds, "train_r2": learn.holdout_error(model, X, t)["r2"],
                    "collect_s": round(time.perf_counter() - t2, 1)})
    t2 = time.perf_counter()
    fd, path = tempfile.mkstemp(suffix=".cm")
    os.close(fd)
    try:
        model.save(path)
        s0 = stats(ex)
        rows = learn.evaluate(ex, seeds=range(1000, 1000 + eval_seeds), model_path=path, max_elems=1e8, reps=3)
        s1 = stats(ex)
    finally:
        os.unlink(path)
    res = learn.summary(rows)
    # Inference: the cost model's share of building the learned plans (block features, GPU
    # inference, merge choice) per plan and per predicted block; and the whole learned plan
    # building (contraction, lowering, NVRTC compilation of new kernels) per plan.
    preds = s1.get("learned_predictions", 0) - s0.get("learned_predictions", 0)
    fusion_s = s1.get("time_learned_fusion", 0) - s0.get("time_learned_fusion", 0)
    choose_s = s1.get("time_learned_choose", 0) - s0.get("time_learned_choose", 0)
    plans = s1.get("learned_trials", 0) + s1.get("learned_same_plan", 0) + s1.get("learned_order_differs", 0) - (
        s0.get("learned_trials", 0) + s0.get("learned_same_plan", 0) + s0.get("learned_order_differs", 0))
    res["inference"] = {"predictions": int(preds), "plans": int(plans),
                        "model_ms_per_plan": round(choose_s * 1e3 / plans, 3) if plans else None,
                        "model_us_per_prediction": round(choose_s * 1e6 / preds, 3) if preds else None,
                        "plan_build_ms_per_plan": round(fusion_s * 1e3 / plans, 3) if plans else None}
    res.update({"records": int(X.shape[0]), "train_loss": round(loss, 4), "holdout": holdout,
                "collect_s": round(t1 - t0, 1),
                "train_s": round(train_s, 2), "eval_s": round(time.perf_counter() - t2, 1),
                "per_dag_speedup_vs_plain": [round(r["plain_ms"] / r["learned_ms"], 2) for r in rows]})
    out["learned_fuser_random_dags"] = res


EXTRAS = {"plain_chain": extra_plain_chain, "heat": extra_heat, "batching": extra_batching, "stream": extra_stream,
          "axpy": extra_axpy, "transpose": extra_transpose, "scan": extra_scan, "learned": extra_learned}


def run_extra(bh, W, ex, rt, peak, only=None, heat_n=4096, learned_train=24, learned_eval=12, learned_holdout=48):
    out = {}
    for name, fn in EXTRAS.items():
        if only is None or name == only:
            if name == "heat":
                fn(bh, W, ex, rt, out, n=heat_n)
            elif name == "learned":
                fn(bh, W, ex, rt, out, train_seeds=learned_train, eval_seeds=learned_eval, holdout_seeds=learned_holdout)
            else:
                fn(bh, W, ex, rt, out)
    return out


def cpu_baseline(n=BS_OPTIONS, iters=BS_ITERS):
    """The oracle (restated ve/openmp) on the host cores: kernel time of the compiled OpenMP code."""
    import bohrium_b200 as bh
    from bohrium_b200 import workloads as W
    from oracle.ve_openmp import OracleExecutor
    threads = os.cpu_count() or 1
    ex = OracleExecutor(threads=threads)
    rt = bh.Runtime(ex)
    S, K, T = W.black_scholes_inputs(n, 0)
    s, k, t = (bh.array(rt, x) for x in (S, K, T))
    W.black_scholes_iteration(rt, s, k, t, 0).numpy()  # compile
    ex.exec_seconds = 0.0
    for it in range(iters):
        W.black_scholes_iteration(rt, s, k, t, it).numpy()
    secs = ex.exec_seconds
    return {"value": round(iters * bs_bytes(n) / secs / 1e9, 3), "unit": "GB/s", "cores": threads, "kind": "port",
            "sample": f"Black-Scholes {n} float64 options x {iters} flushes (the full workload); time of the "
                      f"compiled OpenMP kernels, fusion and compilation excluded as the reference's caches hit",
            "flush_ms": round(secs * 1e3 / iters, 3)}


def run_reference(args, world, rank):
    """The reference arm: the reference's CPU engine for this path (the oracle's restatement of
    ve/openmp) on all host cores. Inputs are made once; each step is one Black-Scholes flush (one
    of the 10 iterations, in turn) over the full 10M options, timed as the compiled OpenMP
    kernels' time (fusion and compilation excluded, as the reference's caches would hit)."""
    if rank != 0:
        return
    import bohrium_b200 as bh
    from bohrium_b200 import workloads as W
    from oracle.ve_openmp import OracleExecutor
    n = args.cpu_options
    threads = os.cpu_count() or 1
    ex = OracleExecutor(threads=threads)
    rt = bh.Runtime(ex)
    S, K, T = W.black_scholes_inputs(n, 0)
    s, k, t = (bh.array(rt, x) for x in (S, K, T))
    for it in range(max(args.warmup, 1)):
        W.black_scholes_iteration(rt, s, k, t, it % BS_ITERS).numpy()  # compiles the kernels
    times = []
    for i in range(args.steps):
        ex.exec_seconds = 0.0
        W.black_scholes_iteration(rt, s, k, t, i % BS_ITERS).numpy()
        times.append(ex.exec_seconds)
    secs = sum(times)
    value = round(args.steps * bs_bytes(n) / secs / 1e9, 3)
    sample = (f"Black-Scholes {n} float64 options, one flush (iteration) per step; compiled OpenMP kernel time "
              f"on {threads} threads")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(secs * 1e3 / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded uniform inputs)",
            "config": {"workload": "black_scholes_f64_10M_options_x10_flushes", "options": n,
                       "flushes_per_step": 1},
            "cpu_baseline": {"value": value, "unit": "GB/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-extra", dest="extra", action="store_false")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--cpu-options", type=int, default=BS_OPTIONS)
    ap.add_argument("--bs-options", type=int, default=BS_OPTIONS, help="options of the headline workload")
    ap.add_argument("--only", choices=sorted(EXTRAS), default=None,
                    help="run one of the other workloads alone (no headline line; for profiling)")
    ap.add_argument("--heat-n", type=int, default=4096, help="grid side of the heat workload")
    ap.add_argument("--learned-train", type=int, default=24, help="training DAGs of the learned-fuser workload")
    ap.add_argument("--learned-eval", type=int, default=12, help="held-out DAGs of the learned-fuser workload")
    ap.add_argument("--learned-holdout", type=int, default=48,
                    help="DAGs whose recorded kernel timings measure the cost model's held-out prediction error")
    args = ap.parse_args()
    world, rank, local = dist_init()
    if args.only:
        import bohrium_b200 as bh
        from bohrium_b200 import workloads as W
        ex = bh.NativeExecutor()
        res = run_extra(bh, W, ex, bh.Runtime(ex), peaks()[0], only=args.only, heat_n=args.heat_n,
                        learned_train=args.learned_train, learned_eval=args.learned_eval,
                        learned_holdout=args.learned_holdout)
        if rank == 0:
            print(json.dumps({"only": args.only, **res}), flush=True)
    elif args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_ours(args, world, rank, local)
    if world > 1:
        import torch.distributed as dist
        if args.impl != "reference":  # the reference arm runs on rank 0 alone; the others leave at once
            dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
