"""The benchmark workloads, written as Bohrium programs with the array front end.

Each builder takes a Runtime and returns the arrays it reads back; all inputs are seeded
synthetic data of the documented shapes (no dataset is involved).

  plain_chain     r = sum(sqrt(a*a + b*b) * exp(-c)) over three float64 arrays (one fused block)
  black_scholes   European call prices of float64 options with an erf-based normal CDF
                  (Abramowitz & Stegun 7.1.26), each iteration ending in a mean-price reduction
  heat            5-point Jacobi stencil on a float32 grid with a fixed boundary of 1.0, ping-pong
                  between two grids, each iteration recording max(abs(new - old))
  batching        many independent float32 systems of uneven length in one flush, each with a
                  12-operation elementwise chain kept in an output array plus its sum and max
  random_dag      seeded random bytecode DAGs (config of the learned fuser cost model)
"""
from __future__ import annotations

import math

import numpy as np

from . import ir
from .array import (BhArray, absolute, array, empty, exp, full, log, maximum, sign, sqrt, random_sample, reduce)
from .runtime import Runtime


# -------------------------------------------------------------------------------- plain chain
def plain_chain_inputs(n: int, seed: int = 0):
    rng = np.random.default_rng(seed)
    return rng.random(n), rng.random(n), rng.random(n)


def plain_chain(rt: Runtime, a: BhArray, b: BhArray, c: BhArray) -> BhArray:
    return (sqrt(a * a + b * b) * exp(-c)).sum()


# ------------------------------------------------------------------------------ Black-Scholes
AS_P = 0.3275911
AS_A = (0.254829592, -0.284496736, 1.421413741, -1.453152027, 1.061405429)


def erf_as(x: BhArray) -> BhArray:
    """erf(x) by Abramowitz & Stegun 7.1.26: sign(x) * (1 - poly(t) * exp(-x^2)), t = 1/(1+p|x|)."""
    a = absolute(x)
    t = 1.0 / (1.0 + AS_P * a)
    poly = ((((AS_A[4] * t + AS_A[3]) * t + AS_A[2]) * t + AS_A[1]) * t + AS_A[0]) * t
    y = 1.0 - poly * exp(-(a * a))
    return sign(x) * y


def cnd(x: BhArray) -> BhArray:
    return 0.5 * (1.0 + erf_as(x * (1.0 / math.sqrt(2.0))))


def black_scholes_inputs(n: int, seed: int = 0):
    rng = np.random.default_rng(seed)
    S = rng.uniform(5.0, 30.0, n)
    K = rng.uniform(1.0, 100.0, n)
    T = rng.uniform(0.25, 10.0, n)
    return S, K, T


def black_scholes_iteration(rt: Runtime, S: BhArray, K: BhArray, T: BhArray, it: int, r: float = 0.02,
                            vol: float = 0.3) -> BhArray:
    """Mean call price with maturities scaled by (1 + 0.01*it): one flush worth of bytecode."""
    Ti = T * (1.0 + 0.01 * it)
    sq = sqrt(Ti)
    d1 = (log(S / K) + (r + 0.5 * vol * vol) * Ti) / (vol * sq)
    d2 = d1 - vol * sq
    call = S * cnd(d1) - K * exp(-r * Ti) * cnd(d2)
    return call.sum() / float(S.size)


def black_scholes_numpy(S, K, T, it, r=0.02, vol=0.3):
    """float64 NumPy version of the same formula (with the same erf approximation)."""
    def erf(x):
        a = np.abs(x)
        t = 1.0 / (1.0 + AS_P * a)
        poly = ((((AS_A[4] * t + AS_A[3]) * t + AS_A[2]) * t + AS_A[1]) * t + AS_A[0]) * t
        return np.sign(x) * (1.0 - poly * np.exp(-(a * a)))
    Ti = T * (1.0 + 0.01 * it)
    sq = np.sqrt(Ti)
    d1 = (np.log(S / K) + (r + 0.5 * vol * vol) * Ti) / (vol * sq)
    d2 = d1 - vol * sq
    c = lambda x: 0.5 * (1.0 + erf(x * (1.0 / math.sqrt(2.0))))
    return np.mean(S * c(d1) - K * np.exp(-r * Ti) * c(d2))


# ------------------------------------------------------------------------------------- heat 2-D
def heat_grid(n: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    g = np.ones((n, n), dtype=np.float32)
    g[1:-1, 1:-1] = rng.random((n - 2, n - 2), dtype=np.float32)
    return g


def heat_step(src: BhArray, dst: BhArray) -> BhArray:
    """dst interior = 0.2 * (5-point stencil of src); returns max(abs(dst - src)) over the interior."""
    c = src[1:-1, 1:-1]
    work = (c + src[:-2, 1:-1] + src[2:, 1:-1] + src[1:-1, :-2] + src[1:-1, 2:]) * np.float32(0.2)
    dst[1:-1, 1:-1] = work
    return absolute(work - c).max()


def heat_numpy(g: np.ndarray, iterations: int):
    a = g.copy()
    b = g.copy()
    deltas = []
    for _ in range(iterations):
        c = a[1:-1, 1:-1]
        w = (c + a[:-2, 1:-1] + a[2:, 1:-1] + a[1:-1, :-2] + a[1:-1, 2:]) * np.float32(0.2)
        b[1:-1, 1:-1] = w
        deltas.append(np.abs(w - c).max())
        a, b = b, a
    return a, deltas


# ------------------------------------------------------------------------------------ batching
def batching_lengths(nsys: int, lo: int = 256, hi: int = 65536, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.integers(lo, hi + 1, nsys)


def batching_chain(x: BhArray) -> BhArray:
    """A 12-operation elementwise chain on float32 data in [0, 1)."""
    f = np.float32
    y = x * f(1.5) + f(0.25)
    y = y * y - f(0.125)
    y = sqrt(absolute(y))
    y = exp(-y) * f(2.0)
    y = maximum(y, f(0.5)) + x
    y = y * f(0.75) - f(0.0625)
    return y


def batching_numpy(x: np.ndarray):
    f = np.float32
    y = x * f(1.5) + f(0.25)
    y = y * y - f(0.125)
    y = np.sqrt(np.abs(y))
    y = np.exp(-y) * f(2.0)
    y = np.maximum(y, f(0.5)) + x
    y = y * f(0.75) - f(0.0625)
    return y


# ------------------------------------------------------------------------------- random DAGs
_UNARY = ["SQRT_ABS", "EXP_NEG", "ABS", "NEG"]
_BINARY = ["ADD", "SUBTRACT", "MULTIPLY", "MAXIMUM", "MINIMUM"]


def random_dag(rt: Runtime, seed: int, nops: int, nelem: int, dtype=np.float32, nreductions: int = 1,
               inputs: int = 3):
    """A seeded random DAG of `nops` elementwise operations over arrays of `nelem` elements.

    Views mix contiguous, transposed, sliced and broadcast forms of 2-D arrays; the DAG ends in
    `nreductions` reductions of random nodes and keeps a few nodes as outputs. Returns
    (inputs, outputs): lists of (BhArray, numpy value) for the inputs and BhArrays for the outputs.
    """
    rng = np.random.default_rng(seed)
    dtype = np.dtype(dtype)
    rows = max(1, int(round(math.sqrt(nelem))))
    cols = max(1, nelem // rows)
    ins = []
    for _ in range(inputs):
        v = rng.random((rows, cols)).astype(dtype)
        if dtype.kind == "i":
            v = (v * 100).astype(dtype)
        ins.append((array(rt, v), v))
    nodes = [a for a, _ in ins]
    for k in range(nops):
        if rng.random() < 0.3:
            name = _UNARY[rng.integers(len(_UNARY))]
            x = nodes[rng.integers(len(nodes))]
            if name == "SQRT_ABS":
                y = sqrt(absolute(x)) if dtype.kind == "f" else absolute(x)
            elif name == "EXP_NEG":
                y = exp(-absolute(x)) if dtype.kind == "f" else x * 2
            elif name == "ABS":
                y = absolute(x)
            else:
                y = -x
        else:
            name = _BINARY[rng.integers(len(_BINARY))]
            x = nodes[rng.integers(len(nodes))]
            z = nodes[rng.integers(len(nodes))]
            form = rng.integers(4)
            if form == 1 and rows == cols:
                z = z.T
            elif form == 2:
                z = z[:, ::-1] if cols > 1 else z
            elif form == 3:
                r0, _ = rng.integers(rows), rng.integers(rows)
                z = z[r0:r0 + 1, :] if rows > 1 else z
            from .array import binary
            y = binary(name, x, z)
        nodes.append(y)
        if len(nodes) > 24:
            nodes.pop(int(rng.integers(inputs, len(nodes) - 4)))
    outs = nodes[-3:]
    for _ in range(nreductions):
        src = nodes[rng.integers(len(nodes))]
        axis = int(rng.integers(3)) - 1
        outs.append(src.sum(axis=None if axis < 0 else axis))
    return ins, outs
