"""Learned fusion on the learned-fuser workload: seeded random bytecode DAGs of 50-400 operations
over 1e3-1e8 elements (float32, float64 or int32; contiguous, transposed, reversed and broadcast
views; 0-3 reductions).

    collect(ex, seeds)      run every DAG under several fusion plans with per-kernel timing on
                            and return the engine's records (features, device microseconds)
    train(X, t)             fit the cost model on the GPU (bohrium_b200.costmodel)
    holdout_error(m, X, t)  R^2 and median |log error| of the model on records of other DAGs
    evaluate(ex, seeds)     per DAG: device time of a flush with the plain greedy plan and with
                            the learned engine (the greedy plan and the learned plan timed on the
                            device, the faster kept), plus a check that the outputs are identical

The plain plan is the greedy fuser's; the learned plan only reorders and stops merges that
mergeable() allows and is only tried when every floating-point sum and product folds in the same
order, so the learned engine's outputs equal the greedy engine's bit for bit.
"""
from __future__ import annotations

import math
import os
import tempfile

import numpy as np

from .runtime import Runtime
from .costmodel import CostModel, read_records
from .workloads import random_dag

GREEDY = "greedy,push_reductions_inwards,collapse_redundant_axes"
WARMUP = 9  # executions before timing: plan building, the learned trials (3 + 3), graph capture
# Plans used to collect training timings: the greedy plan, no DAG fusion (pre-fuser groups
# only), no fusion at all, and two other contraction orders.
VARIANTS = [
    ("lossy", GREEDY),
    ("lossy", "push_reductions_inwards,collapse_redundant_axes"),
    ("singleton", "collapse_redundant_axes"),
    ("lossy", "breadth_first,push_reductions_inwards,collapse_redundant_axes"),
    ("lossy", "serial,collapse_redundant_axes"),
]


def dag_params(seed: int, max_elems: float = 1e8):
    rng = np.random.default_rng([seed, 5])
    nops = int(rng.integers(50, 401))
    nelem = int(10 ** rng.uniform(3.0, math.log10(max_elems)))
    dtype = [np.float32, np.float64, np.int32][int(rng.integers(3))]
    nred = int(rng.integers(0, 4))
    return nops, nelem, dtype, nred


def build(ex, seed: int, max_elems: float = 1e8):
    """Inputs registered and uploaded; returns (runtime, compiled DAG flush, output arrays)."""
    nops, nelem, dtype, nred = dag_params(seed, max_elems)
    rt = Runtime(ex)
    ins, outs = random_dag(rt, seed, nops, nelem, dtype=dtype, nreductions=nred)
    flush = rt.take()
    flush.syncs = []
    return rt, ex.compile(flush), outs, (nops, nelem, np.dtype(dtype).name, nred)


def _set_fusion(ex, pre: str, fusers: str):
    ex.message(f"CUDA: pre_fuser {pre}")
    ex.message(f"CUDA: fuser {fusers}")


def collect(ex, seeds, max_elems: float = 2e7, variants=VARIANTS):
    """Per-kernel (features, microseconds) rows of every DAG under every plan variant."""
    ex.message("CUDA: records clear")
    ex.message("CUDA: autotune off")  # no variant compilation while collecting
    for seed in seeds:
        rt, dag, outs, _ = build(ex, seed, max_elems)
        for pre, fusers in variants:
            _set_fusion(ex, pre, fusers)
            dag.execute()  # compile, upload inputs (not recorded)
            ex.message("CUDA: record on")
            dag.execute()
            ex.message("CUDA: record off")
        del dag, outs, rt
    _set_fusion(ex, "lossy", GREEDY)
    ex.message("CUDA: autotune on")
    fd, path = tempfile.mkstemp(suffix=".rec")
    os.close(fd)
    try:
        ex.message(f"CUDA: records dump {path}")
        return read_records(path)
    finally:
        os.unlink(path)


def holdout_error(model: CostModel, X, t_us) -> dict:
    """Prediction error of `model` on records it was not trained on: R^2 of the log device time
    and the median |log(predicted / measured)|."""
    y = np.log(np.maximum(np.asarray(t_us, dtype=np.float64), 1e-3))
    p = np.log(np.maximum(model.predict_us(X), 1e-30))
    ss_tot = float(np.sum((y - y.mean()) ** 2))
    r2 = 1.0 - float(np.sum((y - p) ** 2)) / ss_tot if ss_tot > 0 else float("nan")
    return {"records": int(len(y)), "r2": round(r2, 4), "median_abs_log_err": round(float(np.median(np.abs(y - p))), 4)}


def train(X, t_us, epochs: int = 300, seed: int = 0) -> tuple[CostModel, float]:
    m = CostModel(seed=seed)
    loss = m.fit(X, t_us, epochs=epochs, batch=256, lr=2e-3, seed=seed)
    return m, loss


def _timed(ex, dag, reps: int) -> float:
    ex.message("CUDA: sync")
    ex.message("CUDA: timer start")
    for _ in range(reps):
        dag.execute()
    return float(ex.message("CUDA: timer stop")) / reps


def evaluate(ex, seeds, model_path: str, max_elems: float = 1e8, reps: int = 5):
    """Device ms per flush of every DAG under three engines -- plain (greedy plan, one launch per
    kernel), batched (greedy plan replayed as a CUDA graph of grouped launches) and batched +
    learned (the learned plan where it is bit-identical and measured faster) -- with the outputs
    of all three compared bit for bit."""
    rows = []
    # The autotuner stays off while the three engines are timed: tuning launches (variants timed
    # on a kernel's first launches) would otherwise fall into whichever engine runs a kernel first.
    ex.message("CUDA: autotune off")
    for seed in seeds:
        rt, dag, outs, shape = build(ex, seed, max_elems)
        times, results = {}, {}
        stats0 = _stats(ex)
        for name, batch, learned in (("plain", "off", False), ("batched", "graph", False),
                                     ("batched_learned", "graph", True)):
            _set_fusion(ex, "lossy", GREEDY)  # forget plans, replays and graphs
            ex.message(f"CUDA: batch {batch}")
            if learned:
                ex.message(f"CUDA: costmodel load {model_path}")
            ex.message("CUDA: learned " + ("on" if learned else "off"))
            for _ in range(WARMUP):  # plan building, learned trials, graph capture
                dag.execute()
            times[name] = _timed(ex, dag, reps)
            results[name] = [ex.peek(o.base).tobytes() for o in outs]
        stats1 = _stats(ex)
        ex.message("CUDA: learned off")
        ex.message("CUDA: batch off")
        rows.append({"seed": seed, "ops": shape[0], "elements": shape[1], "dtype": shape[2], "reductions": shape[3],
                     "plain_ms": times["plain"], "batched_ms": times["batched"],
                     "learned_ms": times["batched_learned"],
                     "identical": results["plain"] == results["batched"] == results["batched_learned"],
                     "learned_kept": stats1.get("learned_kept", 0) - stats0.get("learned_kept", 0),
                     "tried": stats1.get("learned_trials", 0) - stats0.get("learned_trials", 0)})
        del dag, outs, rt
    _set_fusion(ex, "lossy", GREEDY)
    ex.message("CUDA: autotune on")
    return rows


def summary(rows) -> dict:
    """Geometric-mean speed-ups over the DAGs and the total flush times."""
    p = np.array([r["plain_ms"] for r in rows])
    b = np.array([r["batched_ms"] for r in rows])
    l = np.array([r["learned_ms"] for r in rows])
    g = lambda x: float(np.exp(np.mean(np.log(x))))
    return {"dags": len(rows), "geomean_speedup_batched_learned_vs_plain": round(g(p / l), 3),
            "geomean_speedup_batched_vs_plain": round(g(p / b), 3),
            "geomean_speedup_learned_vs_batched": round(g(b / l), 3),
            "total_ms": {"plain": round(float(p.sum()), 3), "batched": round(float(b.sum()), 3),
                         "batched_learned": round(float(l.sum()), 3)},
            "learned_plans_kept": int(sum(r["learned_kept"] for r in rows)),
            "learned_plans_tried": int(sum(r["tried"] for r in rows)),
            "bit_identical": all(r["identical"] for r in rows)}


def _stats(ex) -> dict:
    out = {}
    for line in ex.message("statistic").splitlines():
        if ":" in line and not line.startswith(" "):
            k, v = line.split(":", 1)
            try:
                out[k.strip()] = float(v)
            except ValueError:
                pass
    return out
