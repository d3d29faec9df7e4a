"""Complex element types on the CUDA engine against the CPU oracle (the restated ve/openmp, whose
complex arithmetic is C99's and glibc's).

Tolerances: the engine's complex functions are written from the textbook identities and its
division is Smith's algorithm, so elementwise results differ from glibc's by a few ulps (complex
modulus of the difference relative to the modulus of the oracle's value); reductions change the
summation order (1e-12 complex128, 1e-5 complex64). Comparisons, conversions, REAL/IMAG/CONJ,
gathers and scatters are exact.
"""
import numpy as np
import pytest

from tests import programs as P
from tests.harness import assert_close, run

pytestmark = pytest.mark.gpu


def _tol(dtype, transcendental):
    if np.dtype(dtype) in (np.complex64, np.float32):
        return (2e-5, 2e-6) if transcendental else (1e-6, 1e-7)
    return (1e-12, 1e-14) if transcendental else (1e-14, 1e-15)


def _compare(gpu, ora, rtol, atol, what):
    assert len(gpu) == len(ora)
    for k, (g, o) in enumerate(zip(gpu, ora)):
        assert_close(g, o, rtol, atol, f"{what}[{k}]")


@pytest.mark.parametrize("dtype", P.COMPLEX_TYPES)
@pytest.mark.parametrize("name", P.COMPLEX_BINARY)
def test_complex_binary(gpu_rt, oracle_rt, name, dtype):
    prog = P.complex_binary_program(name, dtype, n=5000)
    _compare(run(gpu_rt, prog), run(oracle_rt, prog), *_tol(dtype, name in P.COMPLEX_TRANSCENDENTAL), name)


@pytest.mark.parametrize("dtype", P.COMPLEX_TYPES)
@pytest.mark.parametrize("name", P.COMPLEX_UNARY + P.COMPLEX_TO_REAL + P.COMPLEX_PREDICATES)
def test_complex_unary(gpu_rt, oracle_rt, name, dtype):
    prog = P.complex_unary_program(name, dtype, n=5000)
    exact = name in ("CONJ", "REAL", "IMAG", "SIGN") or name in P.COMPLEX_PREDICATES
    tol = (0, 0) if exact else _tol(dtype, name in P.COMPLEX_TRANSCENDENTAL)
    _compare(run(gpu_rt, prog), run(oracle_rt, prog), *tol, name)


@pytest.mark.parametrize("dtype", P.COMPLEX_TYPES)
@pytest.mark.parametrize("name", ["EQUAL", "NOT_EQUAL"])
def test_complex_compare(gpu_rt, oracle_rt, name, dtype):
    prog = P.complex_compare_program(name, dtype)
    _compare(run(gpu_rt, prog), run(oracle_rt, prog), 0, 0, name)


@pytest.mark.parametrize("src,dst", [(np.float64, np.complex128), (np.float32, np.complex64),
                                     (np.int32, np.complex128), (np.bool_, np.complex64),
                                     (np.complex64, np.complex128), (np.complex128, np.complex64),
                                     (np.uint64, np.complex64), (np.int8, np.complex128)])
def test_complex_identity(gpu_rt, oracle_rt, src, dst):
    prog = P.complex_identity_program(src, dst)
    _compare(run(gpu_rt, prog), run(oracle_rt, prog), 0, 0, f"{np.dtype(src)}->{np.dtype(dst)}")


# Shapes reaching every reduction schedule: GRID_REDUCE (1-D), SPLIT_REDUCE (axis 0 of a tall or
# short matrix), the in-thread loop (axis 1 of a narrow matrix), LANE_REDUCE (axis 1 of wide rows).
@pytest.mark.parametrize("dtype", P.COMPLEX_TYPES)
@pytest.mark.parametrize("name", ["ADD_REDUCE", "MULTIPLY_REDUCE"])
@pytest.mark.parametrize("shape,axis", [((5000,), 0), ((1_000_003,), 0), ((40, 30), 0), ((40, 30), 1),
                                        ((512, 4096), 1), ((4096, 64), 0)])
def test_complex_reduce(gpu_rt, oracle_rt, name, dtype, shape, axis):
    """complex128 within 1e-12 of the oracle. For complex64 the oracle's own float32 running sums
    (OpenMP threads over up to 1e6 elements) carry an error of about eps32 sqrt(n) rms|x| per
    thread partial, so the engine is held to 1e-5 of the sum plus 2e-5 sqrt(n) rms|x| against the
    oracle, and to 1e-5 relative against the same inputs summed in complex128."""
    prog = P.complex_reduce_program(name, dtype, shape, axis)
    gpu, ora = run(gpu_rt, prog), run(oracle_rt, prog)
    what = f"{name}{shape}/{axis}"
    if np.dtype(dtype) == np.complex128:
        _compare(gpu, ora, 1e-12, 1e-12, what)
        return
    if name == "ADD_REDUCE":
        A = P.cdata(shape, dtype, 0).astype(np.complex128)
        n = shape[axis]
        rms = float(np.sqrt(np.mean(np.abs(A) ** 2)))
        _compare(gpu, ora, 1e-5, 2e-5 * np.sqrt(n) * rms, what)
        exact = A.sum(axis=axis)
        assert_close(gpu[0].astype(np.complex128), exact, 1e-5, 1e-5 * np.sqrt(n) * rms, what + " vs complex128")
    else:
        _compare(gpu, ora, 1e-5, 1e-5, what)


@pytest.mark.parametrize("dtype", P.COMPLEX_TYPES)
@pytest.mark.parametrize("name", ["ADD_ACCUMULATE", "MULTIPLY_ACCUMULATE"])
@pytest.mark.parametrize("shape,axis", [((300,), 0), ((4099,), 0), ((1_000_003,), 0), ((20, 30), 1)])
def test_complex_accumulate(gpu_rt, oracle_rt, name, dtype, shape, axis):
    """The oracle scans sequentially and the engine in its own fixed order, so their running sums
    differ by rounding. complex128: against each other at 1e-12 relative (1e-9 absolute). complex64:
    each against the exact prefix sums and products (complex128) within its own rounding-error
    bound -- gamma_d * sum|x| per component for sums, with d the roundings an input passes through
    (the position for the oracle, SCAN1D's depth for the engine), ((1 + 3u)^i - 1)|p_i| for
    products -- and against each other within the sum of the two bounds."""
    prog = P.complex_accumulate_program(name, dtype, shape, axis)
    gpu, ora = run(gpu_rt, prog), run(oracle_rt, prog)
    if np.dtype(dtype) == np.complex128:
        _compare(gpu, ora, 1e-12, 1e-9, name)
        return
    from tests.harness import U32, assert_cumprod_within_bound, assert_cumsum_within_bound, scan1d_depth
    A = P.complex_accumulate_input(name, dtype, shape)
    g = np.moveaxis(np.asarray(gpu[0]), axis, -1).reshape(-1, shape[axis])
    o = np.moveaxis(np.asarray(ora[0]), axis, -1).reshape(-1, shape[axis])
    x = np.moveaxis(A, axis, -1).reshape(-1, shape[axis])
    n = shape[axis]
    for r in range(x.shape[0]):
        what = f"{name} row {r}"
        if name == "ADD_ACCUMULATE":
            assert_cumsum_within_bound(g[r], x[r], min(n, scan1d_depth(n)) if len(shape) > 1 else scan1d_depth(n),
                                       U32, what + " engine")
            assert_cumsum_within_bound(o[r], x[r], np.arange(1, n + 1), U32, what + " oracle")
        else:
            assert_cumprod_within_bound(g[r], x[r], U32, what=what + " engine")
            assert_cumprod_within_bound(o[r], x[r], U32, what=what + " oracle")


@pytest.mark.parametrize("dtype", P.COMPLEX_TYPES)
def test_complex_gather_scatter(gpu_rt, oracle_rt, dtype):
    prog = P.complex_gather_scatter_program(dtype)
    _compare(run(gpu_rt, prog), run(oracle_rt, prog), 0, 0, "gather/scatter")


@pytest.mark.parametrize("n", [1000, 1 << 20])
def test_complex_fused_chain(gpu_rt, oracle_rt, n):
    prog = P.complex_chain_program(n)
    _compare(run(gpu_rt, prog), run(oracle_rt, prog), 1e-12, 1e-12, "chain")


def test_complex_special_values(gpu_rt, oracle_rt):
    """Zeros, signed zeros and pure real/imaginary inputs through the functions whose formulas
    branch on them (sqrt of negative reals, log of reals, sign, division by a real)."""
    import bohrium_b200 as bh
    vals = np.array([0, -0.0, 1, -1, 1j, -1j, 4, -4, 2 + 0j, -2 + 1e-300j, 1e-8 + 1e-8j, 1 + 1e-9j, 0.6 + 0.8j,
                     3 - 4j, -3 + 4j, 0.5j], dtype=np.complex128)

    def prog(rt):
        a = bh.array(rt, vals)
        out = [bh.sqrt(a), bh.sign(a), bh.exp(a), bh.absolute(a), a / (a * 0 + 2.0)]
        nz = bh.array(rt, vals[2:])
        out.append(bh.log(nz))
        return out
    _compare(run(gpu_rt, prog), run(oracle_rt, prog), 1e-12, 1e-14, "special")
