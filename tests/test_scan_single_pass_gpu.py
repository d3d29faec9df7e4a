"""The single-pass SCAN1D (scan_single_pass = true; chunk tickets, look-back over published chunk
totals with bounded waits): bit-identical to the three-unit scan (the default) and to its order
model, across repeated and graph-
replayed launches (its flags and counters reset themselves), and through its fallback, forced by
a negative wait cap: every chunk that must wait gives up, and the CTA that leaves last redoes the
whole scan alone."""
import numpy as np
import pytest

import bohrium_b200 as bh
from tests.harness import run, scan1d_cumsum

pytestmark = pytest.mark.gpu


def _prog(x):
    def prog(rt):
        a = bh.array(rt, x)
        c = bh.accumulate("ADD_ACCUMULATE", a * x.dtype.type(1) + x.dtype.type(0), 0)
        return [c, c - a]
    return prog


def _with(monkeypatch, **keys):
    for k, v in keys.items():
        monkeypatch.setenv("BH_CUDA_" + k.upper(), str(v))
    return bh.NativeExecutor(stack="cuda")


@pytest.mark.parametrize("n,dtype", [(4_500_001, np.float64), (9_000_000, np.float32), (70_000, np.float64)])
def test_single_pass_equals_three_units_and_model(gpu_rt, monkeypatch, n, dtype):
    x = np.random.default_rng(n).standard_normal(n).astype(dtype)
    three = run(gpu_rt, _prog(x))  # the default: three units
    ex = _with(monkeypatch, scan_single_pass="true", cache_dir="NONE")
    try:
        got = run(bh.Runtime(ex), _prog(x))
    finally:
        ex.close()
    want = scan1d_cumsum(x)
    assert np.asarray(got[0]).tobytes() == want.tobytes()
    assert np.asarray(got[1]).tobytes() == (want - x).tobytes()
    for a, b in zip(got, three):
        assert np.asarray(a).tobytes() == np.asarray(b).tobytes()


@pytest.mark.parametrize("cap", [-1, 0])
def test_fallback_when_waits_give_up(monkeypatch, cap):
    """cap -1: every wait gives up at once (the fallback always runs); cap 0: a wait gives up at
    its first unanswered poll (the fallback runs whenever a chunk found a predecessor not done)."""
    n = 3_000_017
    x = np.random.default_rng(5).standard_normal(n)
    ex = _with(monkeypatch, scan_single_pass="true", scan_spin_cap=cap, cache_dir="NONE")
    try:
        rt = bh.Runtime(ex)
        for _ in range(3):  # the reset after a fallback leaves the next launch clean
            got = run(rt, _prog(x))
            want = scan1d_cumsum(x)
            assert np.asarray(got[0]).tobytes() == want.tobytes()
            assert np.asarray(got[1]).tobytes() == (want - x).tobytes()
    finally:
        ex.close()


def test_repeated_and_graph_replayed_launches(monkeypatch):
    n = 5_000_000
    x = np.random.default_rng(9).standard_normal(n)
    gpu_executor = _with(monkeypatch, scan_single_pass="true", cache_dir="NONE")
    rt = bh.Runtime(gpu_executor)
    a = bh.array(rt, x)
    rt.flush()
    c = bh.accumulate("ADD_ACCUMULATE", a * 1.0 + 0.0, 0)
    ir = gpu_executor.compile(rt.take())
    want = scan1d_cumsum(x).tobytes()
    for mode in ("off", "graph"):
        gpu_executor.message(f"CUDA: batch {mode}")
        try:
            for _ in range(6):
                ir.execute()
                assert gpu_executor.peek(c.base).tobytes() == want, mode
        finally:
            gpu_executor.message("CUDA: batch off")
    del ir, c, a
    gpu_executor.close()
