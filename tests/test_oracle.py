"""The CPU oracle pinned against golden vectors and NumPy (no GPU needed)."""
import ctypes
import json
import os

import numpy as np
import pytest

import bohrium_b200 as bh
from oracle.ve_openmp import OracleExecutor
from tests import programs as P
from tests.harness import assert_close, float_tol, reduce_tol, run

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def golden(name):
    with open(os.path.join(HERE, "golden", name)) as f:
        return json.load(f)


def test_oracle_random123_matches_reference_vectors(oracle_rt):
    for case in golden("random123.json")["cases"]:
        n = len(case["values"])
        r = bh.random123(oracle_rt, (n,), case["start"], case["key"]).numpy()
        assert r.tolist() == case["values"], (case["start"], case["key"])


def test_known_answer_vector():
    # counter 0, key 42 -> words (624017136, 4231775638)
    v = golden("random123.json")["cases"][0]["values"][0]
    assert (v & 0xFFFFFFFF, v >> 32) == (624017136, 4231775638)


def test_reference_build_matches_golden_when_present():
    so = os.path.join(ROOT, "oracle", "_ref", "libref_random123.so")
    if not os.path.exists(so):
        pytest.skip("oracle/_ref not built (make -C oracle)")
    lib = ctypes.CDLL(so)
    lib.ref_random123.restype = ctypes.c_uint64
    lib.ref_random123.argtypes = [ctypes.c_uint64] * 3
    for case in golden("random123.json")["cases"]:
        assert [lib.ref_random123(case["start"], case["key"], i) for i in range(len(case["values"]))] == case["values"]


@pytest.mark.parametrize("dt", ["int8", "int16", "int32", "int64", "uint8", "uint32", "uint64"])
def test_oracle_integer_division_and_remainder(oracle_rt, dt):
    case = golden("integer_semantics.json")["cases"][dt]
    a = bh.array(oracle_rt, np.array(case["a"], dtype=dt))
    b = bh.array(oracle_rt, np.array(case["b"], dtype=dt))
    assert (a // b).numpy().tolist() == case["floor_divide"]
    assert (a % b).numpy().tolist() == case["remainder"]


@pytest.mark.parametrize("name", ["ADD", "SUBTRACT", "MULTIPLY", "DIVIDE", "MAXIMUM", "POWER", "REMAINDER"])
@pytest.mark.parametrize("dtype", [np.int32, np.float64])
def test_oracle_binary_vs_numpy(oracle_rt, name, dtype):
    prog = P.binary_program(name, dtype, n=200)
    got = run(oracle_rt, prog)
    rng_a = P.data(200, dtype, 0, 0.05, 4.0) if np.dtype(dtype).kind == "f" else P.data(200, dtype, 0, 0 if name == "POWER" else None, 20 if name == "POWER" else 100)
    fn = {"ADD": np.add, "SUBTRACT": np.subtract, "MULTIPLY": np.multiply, "MAXIMUM": np.maximum,
          "REMAINDER": np.remainder, "POWER": np.power,
          "DIVIDE": np.floor_divide if np.dtype(dtype).kind == "i" else np.true_divide}[name]
    if np.dtype(dtype).kind == "f":
        B = P.data(200, dtype, 1, 0.05 if name in ("DIVIDE", "REMAINDER", "POWER") else -2.0, 3.0)
    else:
        B = P.data(200, dtype, 1, 0 if name == "POWER" else None, 5 if name == "POWER" else None,
                   nonzero=name in ("DIVIDE", "REMAINDER"))
    with np.errstate(all="ignore"):
        want = fn(rng_a, B).astype(dtype)
    rtol, atol = float_tol(dtype, name == "POWER")
    assert_close(got[0], want, rtol, atol, name)


@pytest.mark.parametrize("axis", [None, 0, 1, 2])
def test_oracle_reductions_vs_numpy(oracle_rt, axis):
    A = P.data((5, 6, 7), np.float64, 3)
    a = bh.array(oracle_rt, A)
    assert_close(a.sum(axis).numpy(), A.sum(axis), reduce_tol(np.float64), 0, "sum")
    assert_close(a.max(axis).numpy(), A.max(axis), 0, 0, "max")


def test_oracle_accumulate_and_views(oracle_rt):
    A = P.data((4, 9), np.float64, 5, 0.5, 1.5)
    a = bh.array(oracle_rt, A)
    assert_close(a.cumsum(1).numpy(), np.cumsum(A, 1), 1e-14, 0, "cumsum axis 1")
    assert_close(a.cumsum(0).numpy(), np.cumsum(A, 0), 1e-14, 0, "cumsum axis 0")
    assert_close(a[::-1, 1::2].numpy(), A[::-1, 1::2], 0, 0, "view")


def test_oracle_black_scholes_vs_numpy(oracle_rt):
    from bohrium_b200 import workloads as W
    S, K, T = W.black_scholes_inputs(1000, 1)
    s, k, t = (bh.array(oracle_rt, x) for x in (S, K, T))
    got = W.black_scholes_iteration(oracle_rt, s, k, t, 3).numpy()
    want = W.black_scholes_numpy(S, K, T, 3)
    assert abs(got - want) <= 1e-12 * abs(want)


def test_oracle_heat_vs_numpy(oracle_rt):
    from bohrium_b200 import workloads as W
    G = W.heat_grid(34, 2)
    a = bh.array(oracle_rt, G)
    b = bh.array(oracle_rt, G)
    deltas = []
    for _ in range(4):
        deltas.append(W.heat_step(a, b).numpy())
        a, b = b, a
    final, want = W.heat_numpy(G, 4)
    assert_close(a.numpy(), final, 1e-6, 1e-7, "grid")
    assert_close(np.array(deltas, dtype=np.float32), np.array(want, dtype=np.float32), 1e-6, 1e-7, "deltas")


def test_oracle_repeat_with_sliding_views():
    """flush-and-repeat with a sliding view (the reference's do_while, test/python/tests/test_loop.py)."""
    from bohrium_b200 import ir
    ex = OracleExecutor(threads=2)
    rt = bh.Runtime(ex)
    A = np.arange(10, dtype=np.float64)
    a = bh.array(rt, A)
    acc = bh.zeros(rt, (1,), np.float64)
    rt.flush()
    # acc += a[i] for i = 0..9 by sliding a one-element view of `a`
    ins = ir.Instr(ir.OPCODES["ADD"], [acc.view(), acc.view(), ir.View(a.base, 0, (1,), (1,))])
    ins.slides[2] = ([ir.Slide(0, 1, 0, 1, 10)], {})
    rt.ex.execute(ir.Flush([ins], nrepeats=10))
    assert acc.numpy()[0] == A.sum()


def test_costmodel_oracle_gradient_matches_finite_differences():
    """Pins the float64 network restatement (the checker of the GPU backward kernel)."""
    from oracle import costmodel as O
    rng = np.random.default_rng(0)
    p = rng.standard_normal(O.NPARAMS) * 0.3
    X = rng.standard_normal((9, O.F))
    t = rng.standard_normal(9)
    loss, g = O.loss_and_grad(p, X, t)
    assert abs(loss - np.mean((O.forward(p, X) - t) ** 2)) < 1e-12
    idx = np.concatenate([rng.choice(O.NPARAMS, 40, replace=False), [O.OFF_B3, O.OFF_W3, O.OFF_B1]])
    h = 1e-6
    for i in idx:
        e = np.zeros(O.NPARAMS)
        e[i] = h
        fd = (O.loss_and_grad(p + e, X, t)[0] - O.loss_and_grad(p - e, X, t)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])
