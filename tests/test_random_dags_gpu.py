"""The learned-fuser workload against the oracle: seeded random bytecode DAGs (float32, float64 and
int32; contiguous, transposed, reversed and broadcast views; 0-3 reductions) run on the CUDA engine
under every plan it has -- the plain greedy plan with one launch per kernel, grouped launches,
CUDA-graph replay, and the learned plan -- and on the CPU oracle (the restated ve/openmp).

Tolerances:
  * int32: bit-exact.
  * reductions: 1e-5 relative (float32), 1e-12 relative (float64), per output element.
  * elementwise outputs: within `float_tol`'s relative bound of each element, or within that same
    relative bound of the output's largest magnitude (a norm-wise bound). A DAG chains up to 400
    dependent operations; a one-ulp difference in one of them (CUDA's vs glibc's exp, the CPU
    compiler's multiply-add contraction) is carried forward and, after a cancellation, is large
    relative to a small element but stays at the ulp scale of the output's magnitude. Two CPU runs
    of the same DAGs that differ only in multiply-add contraction already show 2e-6 of the output's
    magnitude on float32 outputs.
  * all four engine plans: bit-identical to each other.
"""
import numpy as np
import pytest

import bohrium_b200 as bh
from bohrium_b200 import learn
from bohrium_b200.workloads import random_dag
from tests.harness import float_tol, reduce_tol

pytestmark = pytest.mark.gpu

DTYPES = (np.float32, np.float64, np.int32)
# Square shapes let the generator take transposes (it transposes only when rows == cols).
SIZES = (447 * 447, 300 * 300, 1000 * 37, 200_000)


def dag_case(k: int):
    """Case k of 24: dtype k % 3, reductions (k // 3) % 4, so every (dtype, reductions) pair
    appears twice, with 50-400 operations."""
    rng = np.random.default_rng([k, 11])
    nops = int(rng.integers(50, 401))
    return nops, SIZES[k % 4], DTYPES[k % 3], (k // 3) % 4


PLANS = (("plain", "off", False), ("grouped", "grouped", False), ("graph", "graph", False),
         ("learned", "graph", True))


@pytest.fixture(scope="module")
def learned_model(gpu_executor, tmp_path_factory):
    """A cost model trained on this engine's own timings of a few small DAGs, so that the learned
    engine has plans to try."""
    X, t = learn.collect(gpu_executor, seeds=range(1000, 1004), max_elems=5e4)
    model, _ = learn.train(X, t, epochs=60)
    path = str(tmp_path_factory.mktemp("cm") / "cm.bin")
    model.save(path)
    return path


def _engine_outputs(ex, seed, nops, nelem, dt, nred, model_path):
    rt = bh.Runtime(ex)
    _, outs = random_dag(rt, seed, nops, nelem, dtype=dt, nreductions=nred)
    flush = rt.take()
    flush.syncs = []
    dag = ex.compile(flush)
    got = {}
    try:
        for name, batch, learned in PLANS:
            learn._set_fusion(ex, "lossy", learn.GREEDY)  # forget plans, replays and graphs
            ex.message(f"CUDA: batch {batch}")
            if learned:
                ex.message(f"CUDA: costmodel load {model_path}")
            ex.message("CUDA: learned " + ("on" if learned else "off"))
            for _ in range(learn.WARMUP if batch != "off" else 1):
                dag.execute()
            got[name] = [ex.peek(o.base).reshape(o.shape) for o in outs]
    finally:
        ex.message("CUDA: learned off")
        ex.message("CUDA: batch off")
        learn._set_fusion(ex, "lossy", learn.GREEDY)
    return got


def _check(g, o, dt, reduction, what):
    assert g.shape == o.shape and g.dtype == o.dtype, (what, g.shape, o.shape, g.dtype, o.dtype)
    if np.dtype(dt).kind == "i":
        bad = np.flatnonzero(g.reshape(-1) != o.reshape(-1))
        assert bad.size == 0, f"{what}: {bad.size} mismatches, first at {bad[:5]}"
        return
    g64, o64 = g.astype(np.float64), o.astype(np.float64)
    assert np.array_equal(np.isnan(g64), np.isnan(o64)), what
    fin = ~np.isnan(o64)
    d = np.abs(g64 - o64)[fin]
    mag = np.abs(o64)[fin]
    if reduction:
        rtol = reduce_tol(dt)
        bound = rtol * mag
    else:
        rtol, _ = float_tol(dt, transcendental=True)
        bound = rtol * np.maximum(mag, mag.max(initial=0.0))
    worst = float(np.max(d - bound, initial=-1.0))
    assert worst <= 0.0, f"{what}: max |diff| {d.max():.3g} over the bound (rtol {rtol})"


@pytest.mark.parametrize("k", range(24))
def test_random_dag_matches_oracle_under_every_plan(gpu_executor, oracle_rt, learned_model, k):
    nops, nelem, dt, nred = dag_case(k)
    seed = 500 + k
    got = _engine_outputs(gpu_executor, seed, nops, nelem, dt, nred, learned_model)
    _, outs = random_dag(oracle_rt, seed, nops, nelem, dtype=dt, nreductions=nred)
    want = [o.numpy() for o in outs]
    ref = got["plain"]
    assert len(ref) == len(want) == 3 + nred
    for name, _, _ in PLANS:
        for i, (a, b) in enumerate(zip(got[name], ref)):
            assert a.tobytes() == b.tobytes(), f"plan {name} output {i} differs from the plain plan"
    for i, (g, o) in enumerate(zip(ref, want)):
        _check(np.asarray(g), np.asarray(o), dt, i >= 3, f"case {k} ({np.dtype(dt).name}, {nelem}, {nops} ops, "
                                                          f"{nred} reductions) output {i}")
