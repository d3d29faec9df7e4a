"""Every elementwise opcode of the parity suite, for every element type it takes, on the oracle
against NumPy (the witness of the reference's own opcode tests, test/python/tests/
test_primitives.py test_bh_opcodes). The GPU tests compare the engine with the oracle on the same
programs, so together they tie the engine to NumPy. CPU only.

Integer, boolean and comparison results must be exact. Float results get the tolerances of the
GPU tests: glibc's and NumPy's math functions differ by ulps, and gcc contracts FMAs in the
oracle's remainder a - floor(a/b)*b."""
import numpy as np
import pytest

from tests import programs as P
from tests.harness import assert_close, float_tol, run

BINARY_NUMPY = {
    "ADD": np.add, "SUBTRACT": np.subtract, "MULTIPLY": np.multiply, "MAXIMUM": np.maximum,
    "MINIMUM": np.minimum, "BITWISE_AND": np.bitwise_and, "BITWISE_OR": np.bitwise_or,
    "BITWISE_XOR": np.bitwise_xor, "LEFT_SHIFT": np.left_shift, "RIGHT_SHIFT": np.right_shift,
    # MOD is C's % / fmod (sign of the dividend); REMAINDER is Python's (sign of the divisor)
    "MOD": np.fmod, "REMAINDER": np.remainder, "POWER": np.power, "ARCTAN2": np.arctan2,
}

UNARY_NUMPY = {
    "COS": np.cos, "SIN": np.sin, "TAN": np.tan, "COSH": np.cosh, "SINH": np.sinh, "TANH": np.tanh,
    "ARCSIN": np.arcsin, "ARCCOS": np.arccos, "ARCTAN": np.arctan, "ARCSINH": np.arcsinh,
    "ARCCOSH": np.arccosh, "ARCTANH": np.arctanh, "EXP": np.exp, "EXP2": np.exp2, "EXPM1": np.expm1,
    "LOG": np.log, "LOG2": np.log2, "LOG10": np.log10, "LOG1P": np.log1p, "SQRT": np.sqrt,
    "CEIL": np.ceil, "TRUNC": np.trunc, "FLOOR": np.floor, "RINT": np.rint, "ABSOLUTE": np.abs,
    "SIGN": np.sign, "ISNAN": np.isnan, "ISINF": np.isinf, "ISFINITE": np.isfinite, "INVERT": np.invert,
    "LOGICAL_NOT": np.logical_not,
}

COMPARE_NUMPY = {"GREATER": np.greater, "GREATER_EQUAL": np.greater_equal, "LESS": np.less,
                 "LESS_EQUAL": np.less_equal, "EQUAL": np.equal, "NOT_EQUAL": np.not_equal}

LOGICAL_NUMPY = {"LOGICAL_AND": np.logical_and, "LOGICAL_OR": np.logical_or, "LOGICAL_XOR": np.logical_xor}


def _binary_numpy(name, A, B):
    if name == "DIVIDE":
        return np.floor_divide(A, B) if A.dtype.kind in "iu" else np.true_divide(A, B)
    return BINARY_NUMPY[name](A, B)


@pytest.mark.parametrize("name", sorted(P.BINARY))
def test_binary_opcodes_vs_numpy(oracle_rt, name):
    for dt in P.BINARY[name]:
        A, B = P.binary_inputs(name, dt, n=777)
        got = run(oracle_rt, P.binary_program(name, dt, n=777))
        with np.errstate(all="ignore"):
            want = [_binary_numpy(name, A, B).astype(dt), _binary_numpy(name, A, np.full_like(B, B[3])).astype(dt)]
        rtol, atol = float_tol(dt, name in P.TRANSCENDENTAL or name in ("REMAINDER", "MOD"))
        if np.dtype(dt).kind == "f" and name in ("REMAINDER", "MOD"):
            atol = 4 * float(np.finfo(dt).eps) * 4.0  # an ulp or so of |a| <= 4
        for g, w in zip(got, want):
            assert_close(g, w, rtol, atol, f"{name} {np.dtype(dt)}")


@pytest.mark.parametrize("name", P.COMPARE)
def test_comparisons_vs_numpy(oracle_rt, name):
    for dt in P.INT_TYPES + P.FLOAT_TYPES:
        A, B = P.compare_inputs(dt, n=500)
        (got,) = run(oracle_rt, P.compare_program(name, dt, n=500))
        assert_close(got, COMPARE_NUMPY[name](A, B), 0, 0, f"{name} {np.dtype(dt)}")


@pytest.mark.parametrize("name", P.LOGICAL)
def test_logical_vs_numpy(oracle_rt, name):
    A, B = P.data(500, np.bool_, 0), P.data(500, np.bool_, 1)
    (got,) = run(oracle_rt, P.logical_program(name, n=500))
    assert_close(got, LOGICAL_NUMPY[name](A, B), 0, 0, name)


@pytest.mark.parametrize("name", P.UNARY_FLOAT)
def test_unary_float_vs_numpy(oracle_rt, name):
    for dt in P.FLOAT_TYPES:
        A = P.unary_inputs(name, dt)
        (got,) = run(oracle_rt, P.unary_program(name, dt))
        rtol, atol = float_tol(dt, name in P.TRANSCENDENTAL)
        assert_close(got, UNARY_NUMPY[name](A).astype(dt), rtol, atol, f"{name} {np.dtype(dt)}")


@pytest.mark.parametrize("name", P.UNARY_ANY)
def test_unary_any_vs_numpy(oracle_rt, name):
    types = {"INVERT": P.INT_TYPES + [np.bool_], "LOGICAL_NOT": [np.bool_]}.get(name, P.INT_TYPES + P.FLOAT_TYPES)
    for dt in types:
        A = P.unary_inputs(name, dt, n=500)
        (got,) = run(oracle_rt, P.unary_program(name, dt, n=500))
        with np.errstate(all="ignore"):
            want = UNARY_NUMPY[name](A)
        assert_close(got, want.astype(got.dtype), 0, 0, f"{name} {np.dtype(dt)}")


def test_type_conversions_vs_numpy(oracle_rt):
    """BH_IDENTITY between every pair of the GPU suite's types (test_typecast.py of the
    reference), against NumPy's astype on values every destination type holds."""
    types = [np.bool_, np.int8, np.int32, np.int64, np.uint8, np.uint64, np.float32, np.float64]
    for s in types:
        for d in types:
            if s == d:
                continue
            A = P.identity_inputs(s, d)
            (got,) = run(oracle_rt, P.identity_program(s, d))
            assert_close(got, A.astype(d), 0, 0, f"{np.dtype(s)}->{np.dtype(d)}")
