"""The reference's hot-path test cases (test/python/tests/test_reduce.py, test_accumulate.py,
test_summations.py, test_negatives.py, test_emptiness.py and test_loop.py: reduce primitives per
type, reductions of views along every axis, cumsum/cumprod, sum/prod/all/any/mean, division and
remainders of negative integers, empty arrays, flush-and-repeat with sliding views)
run on the oracle, with NumPy as the witness as in the reference's harness
(test/python/run.py:42-59). CPU only. Integer, bitwise and boolean results must be exact;
float sums and products are held to 1e-5 (float32) and 1e-12 (float64) relative, since the oracle's
summation order differs from NumPy's pairwise one."""
import numpy as np
import pytest

import bohrium_b200 as bh
from tests import programs as P

NORMAL = [np.int32, np.int64, np.uint32, np.uint64, np.float32, np.float64]

REDUCE_CASES = ([(op, dt) for op in ("ADD", "MULTIPLY") for dt in (np.float64, np.complex128)]
                + [(op, dt) for op in ("ADD", "MULTIPLY", "MINIMUM", "MAXIMUM") for dt in NORMAL]
                + [(op, np.uint64) for op in ("BITWISE_OR", "BITWISE_XOR")]
                + [(op, np.bool_) for op in ("ADD", "LOGICAL_OR", "LOGICAL_AND", "LOGICAL_XOR")])

NUMPY_UFUNC = {"ADD": np.add, "MULTIPLY": np.multiply, "MINIMUM": np.minimum, "MAXIMUM": np.maximum,
               "BITWISE_OR": np.bitwise_or, "BITWISE_XOR": np.bitwise_xor, "LOGICAL_OR": np.logical_or,
               "LOGICAL_AND": np.logical_and, "LOGICAL_XOR": np.logical_xor}


def random_of_dtype(shape, dtype, seed=42):
    """Seeded values of each type: small positive integers, floats in [0, 1), complex with both
    parts in [0, 1), random booleans."""
    rng = np.random.default_rng(seed)
    dt = np.dtype(dtype)
    if dt == np.bool_:
        return rng.random(shape) < 0.5
    if dt.kind in "iu":
        return rng.integers(1, 10, shape).astype(dt)
    if dt.kind == "c":
        return (rng.random(shape) + 1j * rng.random(shape)).astype(dt)
    return rng.random(shape).astype(dt)


def _check(got, want, dtype):
    got, want = np.asarray(got), np.asarray(want)
    kind = np.dtype(dtype).kind
    if kind in "biu":
        assert np.array_equal(got.astype(np.float64), want.astype(np.float64)), (got, want)
    else:
        tol = 1e-5 if np.dtype(dtype) in (np.float32, np.complex64) else 1e-12
        np.testing.assert_allclose(got, want, rtol=tol, atol=tol * 1e-3)


@pytest.mark.parametrize("op,dtype", REDUCE_CASES)
@pytest.mark.parametrize("scale", [1, 10 ** 6])
def test_reduce_primitives(oracle_rt, op, dtype, scale):
    """test_reduce.py test_primitives: a 10-element vector (test_vector) and the same times 1e6
    (test_vector_large; booleans are not scaled)."""
    host = random_of_dtype((10,), dtype)
    if np.dtype(dtype) != np.bool_ and scale != 1:
        host = (host * scale).astype(dtype)
    got = bh.reduce(op + "_REDUCE", bh.array(oracle_rt, host)).numpy()
    if np.dtype(dtype) == np.bool_ and op == "ADD":
        want = np.add.reduce(host)  # the count, as NumPy gives it
    else:
        with np.errstate(over="ignore"):  # float32 products of values near 1e6 overflow to inf
            want = NUMPY_UFUNC[op].reduce(host, dtype=host.dtype)
    _check(got, want, dtype)


def _views(rt, host):
    """Views of one 4-D float32 array of the kinds the reference's gen_random_arrays makes: the
    whole array, a strided slice, a reversed axis, a transposition and a sub-block."""
    a = bh.array(rt, host)
    yield a, host
    yield a[:, ::2, :, 1:], host[:, ::2, :, 1:]
    yield a[::-1, :, ::-1, :], host[::-1, :, ::-1, :]
    yield a.transpose((3, 1, 0, 2)), host.transpose((3, 1, 0, 2))
    yield a[1:3, 2:5, 1:, :2], host[1:3, 2:5, 1:, :2]


@pytest.mark.parametrize("axis", [0, 1, 2, 3, -1, -2, -3])
def test_reduce_views(oracle_rt, axis):
    """test_reduce.py test_views: add.reduce of views along every axis, positive and negative."""
    host = random_of_dtype((4, 6, 5, 3), np.float32)
    for view, ref in _views(oracle_rt, host):
        got = bh.reduce("ADD_REDUCE", view, axis).numpy()
        _check(got, np.add.reduce(ref, axis=axis), np.float32)


@pytest.mark.parametrize("axis", [0, 1, 2, 3, -1, -2, -3])
def test_accumulate_views(oracle_rt, axis):
    """test_accumulate.py test_views: add.accumulate of views along every axis."""
    host = random_of_dtype((4, 6, 5, 3), np.float32)
    for view, ref in _views(oracle_rt, host):
        ax = axis + view.ndim if axis < 0 else axis
        got = bh.accumulate("ADD_ACCUMULATE", view, ax).numpy()
        _check(got, np.add.accumulate(ref, axis=axis), np.float32)


@pytest.mark.parametrize("method", ["cumsum", "cumprod"])
def test_cumsum_cumprod_methods(oracle_rt, method):
    """test_accumulate.py test_sum: cumsum and cumprod along every axis of 3-D float32 arrays."""
    host = random_of_dtype((5, 4, 6), np.float32) + np.float32(0.5)
    for axis in range(3):
        got = getattr(bh.array(oracle_rt, host), method)(axis).numpy()
        _check(got, getattr(np, method)(host, axis=axis), np.float32)


@pytest.mark.parametrize("op,dtype", [("ADD", np.float64), ("MULTIPLY", np.float64),
                                      ("ADD", np.bool_), ("MULTIPLY", np.bool_)])
def test_accumulate_primitives(oracle_rt, op, dtype):
    """test_accumulate.py test_primitives: add/multiply.accumulate of a 10-element vector."""
    host = random_of_dtype((10,), dtype)
    got = bh.accumulate(op + "_ACCUMULATE", bh.array(oracle_rt, host), 0).numpy()
    _check(got, NUMPY_UFUNC[op].accumulate(host, dtype=host.dtype), dtype)


@pytest.mark.parametrize("op", ["sum", "prod", "all", "any", "mean"])
def test_summations(oracle_rt, op):
    """test_summations.py test_sums: sum, prod, all, any and mean of 3-D float32 arrays and views,
    over the whole array and along every axis (prod of values near 1, so it stays finite)."""
    host = (random_of_dtype((5, 4, 6), np.float32) * np.float32(0.2) + np.float32(0.9)).astype(np.float32)
    if op in ("all", "any"):
        host[1, 2, :] = 0
    a = bh.array(oracle_rt, host)
    views = [(a, host), (a[::-1, 1:, ::2], host[::-1, 1:, ::2]), (a.transpose((2, 0, 1)), host.transpose((2, 0, 1)))]
    for view, ref in views:
        for axis in [None, 0, 1, 2]:
            got = getattr(view, op)(axis).numpy()
            want = getattr(ref, op)(axis=axis)
            if op in ("all", "any"):
                assert np.array_equal(np.asarray(got).astype(bool), want), (op, axis)
            else:
                _check(got, want, np.float32)


@pytest.mark.parametrize("dtype", [np.int8, np.int16, np.int32, np.int64])
@pytest.mark.parametrize("swap", [False, True])
def test_negative_operands(oracle_rt, dtype, swap):
    """test_negatives.py: a = arange(-11, -1), b = arange(1, 11) and the other way round, through
    true division, floor division, % / remainder (the divisor's sign) and fmod (the dividend's)."""
    x, y = np.arange(-11, -1, dtype=dtype), np.arange(1, 11, dtype=dtype)
    A, B = (y, x) if swap else (x, y)
    a, b = bh.array(oracle_rt, A), bh.array(oracle_rt, B)
    np.testing.assert_array_equal((a / b).numpy(), A / B)
    np.testing.assert_array_equal((a // b).numpy(), A // B)
    np.testing.assert_array_equal((a % b).numpy(), np.remainder(A, B))
    np.testing.assert_array_equal(bh.binary("MOD", a, b).numpy(), np.fmod(A, B))


def test_empty_arrays(oracle_rt):
    """test_emptiness.py: a + a of empty arrays is an empty array."""
    a = bh.array(oracle_rt, np.array([], dtype=np.float64))
    res = (a + a).numpy()
    assert res.shape == (0,) and res.dtype == np.float64


def test_loop_sliding_views_triangular_numbers(oracle_rt):
    """test_loop.py test_loop_faculty_function_using_sliding_views: a[i+1] += a[i] for 10
    iterations of one flush, both views sliding by one element per iteration."""
    got, want = P.loop_triangular_numbers(oracle_rt)
    np.testing.assert_array_equal(got, want)


def test_loop_one_and_two_dimensional_sliding_views(oracle_rt):
    """test_loop.py test_loop_one_and_two_dimensional_sliding_views: res[i] += b[i, i], the
    element of b sliding along both axes at once."""
    got, want = P.loop_diagonal(oracle_rt)
    np.testing.assert_array_equal(got, want)
