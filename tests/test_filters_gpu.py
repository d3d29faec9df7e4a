"""Programs through the stack with the bytecode filter components (bcexp, bccon, node, cuda):
the filtered bytecode gives NumPy's results (integers bit-exact)."""
import numpy as np
import pytest

import bohrium_b200 as bh

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def filtered():
    return bh.NativeExecutor(stack="filtered_cuda")


def test_filtered_stack_integer_programs(filtered):
    rt = bh.Runtime(filtered)
    X = np.random.default_rng(0).integers(-20, 20, 100_000).astype(np.int64)
    x = bh.array(rt, X)
    outs = [bh.binary("POWER", x, np.int64(3)) + np.int64(1),
            x * np.int64(1) + np.int64(0),
            ((x + np.int64(3)) - np.int64(5)) + np.int64(7),
            x * np.int64(2) + x * np.int64(3)]
    want = [X ** 3 + 1, X, X + 5, 5 * X]
    for o, w in zip(outs, want):
        assert np.array_equal(o.numpy(), w)


def test_filtered_stack_float_power(filtered):
    rt = bh.Runtime(filtered)
    X = np.random.default_rng(1).random(50_000)
    x = bh.array(rt, X)
    y = bh.binary("POWER", x, np.int64(5)).sum()
    np.testing.assert_allclose(float(y.numpy()), float(np.sum(X ** 5)), rtol=1e-12)


def test_filtered_stack_reduce1d(monkeypatch):
    """With the reference's GPU-stack setting reduce1d = 32000 the 1-D reductions reach the engine
    as a [32, 32768] axis-0 reduction plus a 32768-element one: results within the float64
    reduction tolerance of NumPy, integer and max results bit-exact."""
    monkeypatch.setenv("BH_BCEXP_REDUCE1D", "32000")
    ex = bh.NativeExecutor(stack="filtered_cuda")
    rt = bh.Runtime(ex)
    rng = np.random.default_rng(2)
    X = rng.standard_normal(1 << 20)
    I = rng.integers(-1000, 1000, 1 << 20).astype(np.int64)
    x, i = bh.array(rt, X), bh.array(rt, I)
    s, m, t = x.sum(), x.max(), i.sum()
    np.testing.assert_allclose(float(s.numpy()), float(np.sum(X)), rtol=1e-12, atol=1e-9)
    assert float(m.numpy()) == float(X.max())
    assert int(t.numpy()) == int(I.sum())
