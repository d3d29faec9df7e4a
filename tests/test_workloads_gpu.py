"""The benchmark workloads on the GPU: parity with the oracle at small sizes, and size-independent
properties at the benchmark sizes."""
import numpy as np
import pytest

import bohrium_b200 as bh
from bohrium_b200 import workloads as W
from tests.harness import assert_close

pytestmark = pytest.mark.gpu


def test_plain_chain_parity(gpu_rt, oracle_rt):
    A, B, C = W.plain_chain_inputs(1 << 20, 0)
    res = []
    for rt in (gpu_rt, oracle_rt):
        a, b, c = (bh.array(rt, x) for x in (A, B, C))
        res.append(W.plain_chain(rt, a, b, c).numpy())
    want = np.sum(np.sqrt(A * A + B * B) * np.exp(-C))
    assert abs(res[0] - res[1]) <= 1e-12 * abs(res[1])
    assert abs(res[0] - want) <= 1e-12 * abs(want)


def test_black_scholes_parity(gpu_rt, oracle_rt):
    S, K, T = W.black_scholes_inputs(100_000, 1)
    for it in range(3):
        res = []
        for rt in (gpu_rt, oracle_rt):
            s, k, t = (bh.array(rt, x) for x in (S, K, T))
            res.append(W.black_scholes_iteration(rt, s, k, t, it).numpy())
        assert abs(res[0] - res[1]) <= 1e-12 * abs(res[1]), (it, res)


def test_heat_parity(gpu_rt, oracle_rt):
    G = W.heat_grid(130, 3)
    grids, deltas = [], []
    for rt in (gpu_rt, oracle_rt):
        a, b = bh.array(rt, G), bh.array(rt, G)
        d = []
        for _ in range(6):
            d.append(W.heat_step(a, b).numpy())
            a, b = b, a
        grids.append(a.numpy())
        deltas.append(np.array(d, dtype=np.float32))
    assert_close(grids[0], grids[1], 1e-5, 1e-6, "grid")
    assert_close(deltas[0], deltas[1], 1e-5, 1e-6, "deltas")


def test_batching_parity(gpu_rt, oracle_rt):
    lengths = W.batching_lengths(24, 256, 5000, 4)
    xs = [np.random.default_rng(i).random(int(n), dtype=np.float32) for i, n in enumerate(lengths)]
    res = []
    for rt in (gpu_rt, oracle_rt):
        out = []
        arrs = []
        for x in xs:
            y = W.batching_chain(bh.array(rt, x))
            arrs += [y, y.sum(), y.max()]
        out = [a.numpy() for a in arrs]
        res.append(out)
    for k, (g, o) in enumerate(zip(*res)):
        tol = 1e-5 if k % 3 == 1 else 1e-6
        assert_close(g, o, tol, 1e-6, f"batching[{k}]")


def test_plain_chain_full_size_property(gpu_rt):
    """Linearity at 2^24 elements: sum(f(a)) over the two halves adds up to the whole."""
    n = 1 << 24
    A, B, C = W.plain_chain_inputs(n, 5)
    a, b, c = (bh.array(gpu_rt, x) for x in (A, B, C))
    whole = W.plain_chain(gpu_rt, a, b, c).numpy()
    h1 = W.plain_chain(gpu_rt, a[: n // 2], b[: n // 2], c[: n // 2]).numpy()
    h2 = W.plain_chain(gpu_rt, a[n // 2:], b[n // 2:], c[n // 2:]).numpy()
    assert abs(whole - (h1 + h2)) <= 1e-12 * abs(whole)
    want = np.sum(np.sqrt(A * A + B * B) * np.exp(-C))
    assert abs(whole - want) <= 1e-12 * abs(want)


def test_black_scholes_full_size_against_numpy(gpu_rt):
    S, K, T = W.black_scholes_inputs(10_000_000, 0)
    s, k, t = (bh.array(gpu_rt, x) for x in (S, K, T))
    got = W.black_scholes_iteration(gpu_rt, s, k, t, 0).numpy()
    want = W.black_scholes_numpy(S, K, T, 0)
    assert abs(got - want) <= 1e-12 * abs(want)


def test_heat_full_size_properties(gpu_rt):
    """4096^2 float32: the boundary stays 1.0 and every delta is a max of absolute values."""
    G = W.heat_grid(4096, 0)
    a, b = bh.array(gpu_rt, G), bh.array(gpu_rt, G)
    deltas = []
    for _ in range(4):
        deltas.append(float(W.heat_step(a, b).numpy()))
        a, b = b, a
    g = a.numpy()
    assert (g[0] == 1).all() and (g[-1] == 1).all() and (g[:, 0] == 1).all() and (g[:, -1] == 1).all()
    assert all(d >= 0 for d in deltas)
    final, want = W.heat_numpy(G, 4)
    assert_close(g, final, 1e-5, 1e-6, "grid")
