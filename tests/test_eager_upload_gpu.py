"""Eager uploads: page-locked host data handed to the engine with setMemoryPointer (bhb_data_set)
is copied at once on a copy stream, and every later use on the engine's stream waits for it. The
results must be those of the data handed over, whatever overlaps with what."""
import numpy as np
import pytest

import bohrium_b200 as bh
from bohrium_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _stats(ex):
    out = {}
    for line in ex.message("statistic").splitlines():
        if ":" in line and not line.startswith(" "):
            k, v = line.split(":", 1)
            try:
                out[k.strip()] = float(v)
            except ValueError:
                pass
    return out


def _pinned_set(ex, rt, n, seed):
    S, K, T = W.black_scholes_inputs(n, seed)
    arrays, hosts = [], []
    for x in (S, K, T):
        a = bh.empty(rt, (n,), np.float64)
        hosts.append(ex.set_pinned(a.base, x))
        arrays.append(a)
    rt.flush()
    irs, outs = [], []
    for it in range(3):
        outs.append(W.black_scholes_iteration(rt, *arrays, it))
        irs.append(ex.compile(rt.take()))
    return arrays, hosts, irs, outs, (S, K, T)


def _hand_over(ex, st, data=None):
    arrays, hosts = st[0], st[1]
    for k, (a, h) in enumerate(zip(arrays, hosts)):
        if data is not None:
            h[:] = data[k]
        assert ex.lib.bhb_data_set(ex.rt, a.base.handle, 1, h.ctypes.data) == 0


def test_alternating_sets_overlap_and_stay_correct(gpu_executor):
    ex = gpu_executor
    rt = bh.Runtime(ex)
    n = 3_000_017
    sets = [_pinned_set(ex, rt, n, seed) for seed in (1, 2)]
    u0 = _stats(ex).get("eager_uploads", 0)
    _hand_over(ex, sets[0])
    cur = 0
    for step in range(6):
        nxt = sets[1 - cur]
        # new values for the next set each time, so a stale upload would show
        data = W.black_scholes_inputs(n, 100 + step)
        _hand_over(ex, nxt, data)
        for ir in sets[cur][2]:
            ir.execute()
        got = [float(ex.peek(o.base)[0]) for o in sets[cur][3]]
        src = sets[cur][4] if step == 0 else W.black_scholes_inputs(n, 100 + step - 1)
        want = [W.black_scholes_numpy(*src, it) for it in range(3)]
        assert all(abs(g - w) <= 1e-10 * abs(w) for g, w in zip(got, want)), (step, got, want)
        cur = 1 - cur
    ex.message("CUDA: sync")
    assert _stats(ex)["eager_uploads"] - u0 == 3 * 7


def test_freed_and_replaced_while_uploading(gpu_executor):
    """A base freed, or handed new data, while its upload is in flight."""
    ex = gpu_executor
    rt = bh.Runtime(ex)
    n = 1 << 22
    a = bh.empty(rt, (n,), np.float64)
    h = ex.set_pinned(a.base, np.arange(n, dtype=np.float64))
    rt.flush()
    for v in (1.0, 2.0, 3.0):
        h[:] = v
        assert ex.lib.bhb_data_set(ex.rt, a.base.handle, 1, h.ctypes.data) == 0
    s = a.sum()
    assert float(s.numpy()) == 3.0 * n
    b = bh.empty(rt, (n,), np.float64)
    hb = ex.set_pinned(b.base, np.ones(n))
    rt.flush()
    assert ex.lib.bhb_data_set(ex.rt, b.base.handle, 1, hb.ctypes.data) == 0
    del b, hb
    rt.flush()  # BH_FREE of b with its upload possibly still in flight
    ex.message("CUDA: sync")
