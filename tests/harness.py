"""Helpers to run one program on two runtimes and compare the results."""
from __future__ import annotations

import numpy as np


def run(rt, prog):
    outs = prog(rt)
    return [o.numpy() for o in outs]


def assert_close(got, want, rtol, atol=0.0, what=""):
    got = np.asarray(got)
    want = np.asarray(want)
    assert got.shape == want.shape, f"{what}: shape {got.shape} != {want.shape}"
    assert got.dtype == want.dtype, f"{what}: dtype {got.dtype} != {want.dtype}"
    if got.dtype.kind in "biu":
        bad = np.flatnonzero(got.reshape(-1) != want.reshape(-1))
        assert bad.size == 0, f"{what}: {bad.size} integer mismatches, first at {bad[:5]}: " \
                              f"{got.reshape(-1)[bad[:5]]} vs {want.reshape(-1)[bad[:5]]}"
    else:
        np.testing.assert_allclose(got, want, rtol=rtol, atol=atol, equal_nan=True, err_msg=what)


def float_tol(dtype, transcendental=False):
    """Tolerances for elementwise floating-point results of the CUDA engine vs the CPU oracle:
    a few ulps (CUDA's and glibc's math functions, and FMA contraction on the CPU side)."""
    if np.dtype(dtype) == np.float32:
        return (1e-5, 1e-6) if transcendental else (1e-6, 1e-7)
    return (1e-12, 1e-14) if transcendental else (1e-14, 1e-15)


def reduce_tol(dtype):
    """Reductions change summation order: 1e-5 relative for float32, 1e-12 for float64."""
    return 1e-5 if np.dtype(dtype) == np.float32 else 1e-12


def compare(a_results, b_results, tol=None, what=""):
    assert len(a_results) == len(b_results)
    for k, (x, y) in enumerate(zip(a_results, b_results)):
        if tol is None:
            rtol, atol = float_tol(np.asarray(y).dtype)
        else:
            rtol, atol = tol
        assert_close(x, y, rtol, atol, f"{what}[{k}]")
