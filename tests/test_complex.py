"""Complex element types in the CPU oracle, pinned against NumPy (no GPU needed).

The expectations follow the reference's semantics where they differ from NumPy's
(core/jitk/instruction.cpp): ISNAN/ISINF/ISFINITE test the real part only, SIGN is csgn
(sgn of the real part, or of the imaginary part where the real part is 0, with a zero imaginary
part), and LOG10 divides the complex log by log(10.0f), ln 10 rounded to float.
"""
import numpy as np
import pytest

from tests import programs as P
from tests.harness import assert_close, run


def _tol(dtype, transcendental):
    if np.dtype(dtype) in (np.complex64, np.float32):
        return (2e-5, 2e-6) if transcendental else (1e-6, 1e-7)
    return (1e-12, 1e-14) if transcendental else (1e-14, 1e-15)


def _expect_unary(name, A):
    rdt = P.real_dtype(A.dtype)
    if name == "ISNAN":
        return np.isnan(A.real)
    if name == "ISINF":
        return np.isinf(A.real)
    if name == "ISFINITE":
        return np.isfinite(A.real)
    if name == "SIGN":
        s = np.where(A.real == 0, np.sign(A.imag), np.sign(A.real))
        return s.astype(A.dtype)
    if name == "LOG10":
        return (np.log(A.astype(np.complex128)) / np.float64(np.float32(np.log(10.0)))).astype(A.dtype)
    if name == "CONJ":
        return np.conj(A)
    if name == "ABSOLUTE":
        return np.abs(A.astype(np.complex128)).astype(rdt)
    if name == "REAL":
        return A.real.astype(rdt)
    if name == "IMAG":
        return A.imag.astype(rdt)
    f = {"COS": np.cos, "SIN": np.sin, "TAN": np.tan, "COSH": np.cosh, "SINH": np.sinh, "TANH": np.tanh,
         "EXP": np.exp, "LOG": np.log, "SQRT": np.sqrt}[name]
    return f(A.astype(np.complex128)).astype(A.dtype)


@pytest.mark.parametrize("dtype", P.COMPLEX_TYPES)
@pytest.mark.parametrize("name", P.COMPLEX_UNARY + P.COMPLEX_TO_REAL + P.COMPLEX_PREDICATES)
def test_oracle_complex_unary_vs_numpy(oracle_rt, name, dtype):
    A = P.cdata(1000, dtype, 0)
    if name == "SIGN":
        A.real[::5] = 0
        A[::25] = 0
    if name in P.COMPLEX_PREDICATES:
        A.real[::7] = np.nan
        A.imag[3::7] = np.nan
        A.real[1::11] = np.inf
        A.imag[5::11] = np.inf
    (got,) = run(oracle_rt, P.complex_unary_program(name, dtype))
    want = _expect_unary(name, A)
    rtol, atol = _tol(dtype, name in P.COMPLEX_TRANSCENDENTAL)
    assert_close(got, want, rtol, atol * 10, name)


@pytest.mark.parametrize("dtype", P.COMPLEX_TYPES)
@pytest.mark.parametrize("name", P.COMPLEX_BINARY)
def test_oracle_complex_binary_vs_numpy(oracle_rt, name, dtype):
    A = P.cdata(1000, dtype, 0, 0.1, 2.0)
    B = P.cdata(1000, dtype, 1, 0.1 if name in ("DIVIDE", "POWER") else -2.0, 1.5)
    f = {"ADD": np.add, "SUBTRACT": np.subtract, "MULTIPLY": np.multiply, "DIVIDE": np.divide,
         "POWER": np.power}[name]
    wide = np.complex128
    got, got_c = run(oracle_rt, P.complex_binary_program(name, dtype))
    rtol, atol = _tol(dtype, name in P.COMPLEX_TRANSCENDENTAL)
    assert_close(got, f(A.astype(wide), B.astype(wide)).astype(dtype), rtol, atol, name)
    assert_close(got_c, f(A.astype(wide), wide(B[3])).astype(dtype), rtol, atol, name + " constant")


@pytest.mark.parametrize("dtype", P.COMPLEX_TYPES)
@pytest.mark.parametrize("name", ["EQUAL", "NOT_EQUAL"])
def test_oracle_complex_compare_vs_numpy(oracle_rt, name, dtype):
    A = P.cdata(1000, dtype, 0)
    B = P.cdata(1000, dtype, 1)
    B[::3] = A[::3]
    B.real[1::5] = A.real[1::5]
    (got,) = run(oracle_rt, P.complex_compare_program(name, dtype))
    assert_close(got, (A == B) if name == "EQUAL" else (A != B), 0, 0, name)


@pytest.mark.parametrize("src,dst", [(np.float64, np.complex128), (np.float32, np.complex64),
                                     (np.int32, np.complex128), (np.bool_, np.complex64),
                                     (np.complex64, np.complex128), (np.complex128, np.complex64),
                                     (np.uint64, np.complex64)])
def test_oracle_complex_identity_vs_numpy(oracle_rt, src, dst):
    s = np.dtype(src)
    A = P.cdata(500, s, 0, -100.0, 100.0) if s.kind == "c" else (
        P.data(500, s, 0, -100.0, 100.0) if s.kind == "f" else P.data(500, s, 0))
    (got,) = run(oracle_rt, P.complex_identity_program(src, dst))
    assert_close(got, A.astype(dst), 0, 0, f"{s}->{np.dtype(dst)}")


@pytest.mark.parametrize("dtype", P.COMPLEX_TYPES)
@pytest.mark.parametrize("name", ["ADD_REDUCE", "MULTIPLY_REDUCE"])
@pytest.mark.parametrize("shape,axis", [((5000,), 0), ((40, 30), 0), ((40, 30), 1)])
def test_oracle_complex_reduce_vs_numpy(oracle_rt, name, dtype, shape, axis):
    (got,) = run(oracle_rt, P.complex_reduce_program(name, dtype, shape, axis))
    rng = np.random.default_rng(0)
    if name == "MULTIPLY_REDUCE":
        A = ((0.95 + 0.1 * rng.random(shape)) * np.exp(0.05j * (rng.random(shape) - 0.5))).astype(dtype)
        want = np.prod(A.astype(np.complex128), axis=axis)
    else:
        A = P.cdata(shape, dtype, 0)
        want = np.sum(A.astype(np.complex128), axis=axis)
    rtol = 2e-5 if np.dtype(dtype) == np.complex64 else 1e-12
    assert_close(got, want.astype(dtype), rtol, rtol, name)


@pytest.mark.parametrize("dtype", P.COMPLEX_TYPES)
@pytest.mark.parametrize("name", ["ADD_ACCUMULATE", "MULTIPLY_ACCUMULATE"])
def test_oracle_complex_accumulate_vs_numpy(oracle_rt, name, dtype):
    shape = (300,)
    (got,) = run(oracle_rt, P.complex_accumulate_program(name, dtype, shape, 0))
    rng = np.random.default_rng(0)
    if name == "MULTIPLY_ACCUMULATE":
        A = ((0.98 + 0.04 * rng.random(shape)) * np.exp(0.05j * (rng.random(shape) - 0.5))).astype(dtype)
        want = np.cumprod(A, axis=0)
    else:
        A = P.cdata(shape, dtype, 0)
        want = np.cumsum(A, axis=0)
    rtol = 2e-5 if np.dtype(dtype) == np.complex64 else 1e-12
    assert_close(got, want, rtol, rtol, name)


def test_oracle_complex_chain_vs_numpy(oracle_rt):
    n = 4096
    x = P.cdata(n, np.complex128, 0)
    theta = P.data(n, np.float64, 1, -3.0, 3.0)
    z = np.exp(theta * 1j) * x + np.conj(x) * 0.5
    p = z.real * z.real + z.imag * z.imag
    got = run(oracle_rt, P.complex_chain_program(n))
    for g, w in zip(got, [z, z.sum(), p, p.sum(), np.abs(z)]):
        assert_close(g, np.asarray(w), 1e-12, 1e-12, "chain")


def test_oracle_complex_gather_scatter(oracle_rt):
    for dtype in P.COMPLEX_TYPES:
        g, dst = run(oracle_rt, P.complex_gather_scatter_program(dtype))
        src = P.cdata(1000, dtype, 0)
        idx = np.random.default_rng(0).permutation(1000)
        assert_close(g, src[idx], 0, 0, "gather")
        want = np.zeros(1000, dtype)
        want[idx] = src[idx]
        assert_close(dst, want, 0, 0, "scatter")
