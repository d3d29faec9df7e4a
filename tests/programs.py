"""Small Bohrium programs shared by the parity tests (GPU engine vs CPU oracle vs NumPy).

The cases follow the reference's own test-suite: every elementwise opcode over its type
signatures (test/python/tests/test_primitives.py), reductions over every axis of views
(test_reduce.py), cumulative sums (test_accumulate.py), sliding views in repeated flushes
(test_loop.py) and BH_RANDOM (test_random.py). Each program takes a Runtime and returns the
arrays to compare; inputs are seeded.
"""
from __future__ import annotations

import numpy as np

import bohrium_b200 as bh
from bohrium_b200 import ir

INT_TYPES = [np.int8, np.int16, np.int32, np.int64, np.uint8, np.uint16, np.uint32, np.uint64]
FLOAT_TYPES = [np.float32, np.float64]


def data(shape, dtype, seed, lo=None, hi=None, nonzero=False):
    rng = np.random.default_rng(seed)
    dt = np.dtype(dtype)
    if dt == np.bool_:
        return rng.random(shape) < 0.5
    if dt.kind == "f":
        lo = 0.0 if lo is None else lo
        hi = 1.0 if hi is None else hi
        return (rng.random(shape) * (hi - lo) + lo).astype(dt)
    info = np.iinfo(dt)
    lo = max(info.min, -100) if lo is None else lo
    hi = min(info.max, 100) if hi is None else hi
    v = rng.integers(lo, hi, shape, endpoint=True).astype(dt)
    if nonzero:
        v[v == 0] = 1
    return v


# Binary opcodes with the element types they accept (the reference's opcode signatures).
BINARY = {
    "ADD": INT_TYPES + FLOAT_TYPES + [np.bool_],
    "SUBTRACT": INT_TYPES + FLOAT_TYPES,
    "MULTIPLY": INT_TYPES + FLOAT_TYPES + [np.bool_],
    "DIVIDE": INT_TYPES + FLOAT_TYPES,
    "MAXIMUM": INT_TYPES + FLOAT_TYPES + [np.bool_],
    "MINIMUM": INT_TYPES + FLOAT_TYPES + [np.bool_],
    "BITWISE_AND": INT_TYPES + [np.bool_],
    "BITWISE_OR": INT_TYPES + [np.bool_],
    "BITWISE_XOR": INT_TYPES + [np.bool_],
    "LEFT_SHIFT": INT_TYPES,
    "RIGHT_SHIFT": INT_TYPES,
    "MOD": INT_TYPES + FLOAT_TYPES,
    "REMAINDER": INT_TYPES + FLOAT_TYPES,
    "POWER": [np.int32, np.int64, np.uint32, np.float32, np.float64],
    "ARCTAN2": FLOAT_TYPES,
}
COMPARE = ["GREATER", "GREATER_EQUAL", "LESS", "LESS_EQUAL", "EQUAL", "NOT_EQUAL"]
LOGICAL = ["LOGICAL_AND", "LOGICAL_OR", "LOGICAL_XOR"]
UNARY_FLOAT = ["COS", "SIN", "TAN", "COSH", "SINH", "TANH", "ARCSIN", "ARCCOS", "ARCTAN", "ARCSINH", "ARCCOSH",
               "ARCTANH", "EXP", "EXP2", "EXPM1", "LOG", "LOG2", "LOG10", "LOG1P", "SQRT", "CEIL", "TRUNC", "FLOOR",
               "RINT"]
UNARY_ANY = ["ABSOLUTE", "SIGN", "ISNAN", "ISINF", "ISFINITE", "INVERT", "LOGICAL_NOT"]
TRANSCENDENTAL = {"COS", "SIN", "TAN", "COSH", "SINH", "TANH", "ARCSIN", "ARCCOS", "ARCTAN", "ARCSINH", "ARCCOSH",
                  "ARCTANH", "EXP", "EXP2", "EXPM1", "LOG", "LOG2", "LOG10", "LOG1P", "ARCTAN2", "POWER"}


def binary_inputs(name, dtype, n=1000, seed=0):
    """The two operand arrays of binary_program (its constant operand is B[3])."""
    dt = np.dtype(dtype)
    lo = 0 if name in ("LEFT_SHIFT", "RIGHT_SHIFT", "POWER") or dt.kind == "u" else None
    hi_b = 5 if name in ("LEFT_SHIFT", "RIGHT_SHIFT", "POWER") else None
    nz = name in ("DIVIDE", "MOD", "REMAINDER")
    if dt.kind == "f":
        A = data(n, dt, seed, 0.05, 4.0)
        B = data(n, dt, seed + 1, 0.05 if nz or name == "POWER" else -2.0, 3.0)
    else:
        # POWER stays inside the type's range: the reference converts pow()'s double result,
        # which is undefined behaviour in C on overflow.
        A = data(n, dt, seed, lo, 20 if name == "POWER" else (None if hi_b is None else 100))
        B = data(n, dt, seed + 1, lo if lo is not None else None, hi_b, nonzero=nz)
    return A, B


def binary_program(name, dtype, n=1000, seed=0):
    dt = np.dtype(dtype)

    def prog(rt):
        A, B = binary_inputs(name, dt, n, seed)
        a = bh.array(rt, A)
        b = bh.array(rt, B)
        out = bh.empty(rt, (n,), dt)
        rt.enqueue(ir.Instr(ir.OPCODES[name], [out.view(), a.view(), b.view()]))
        # the same operation with a constant operand
        out2 = bh.empty(rt, (n,), dt)
        c = B[3].item()
        rt.enqueue(ir.Instr(ir.OPCODES[name], [out2.view(), a.view(), None], ir.Constant(c, ir.bh_type(dt))))
        return [out, out2]
    return prog


def compare_inputs(dtype, n=1000, seed=0):
    """The operands of compare_program: every third element equal."""
    A = data(n, dtype, seed)
    B = data(n, dtype, seed + 1)
    B[::3] = A[::3]
    return A, B


def compare_program(name, dtype, n=1000, seed=0):
    def prog(rt):
        A, B = compare_inputs(dtype, n, seed)
        a, b = bh.array(rt, A), bh.array(rt, B)
        out = bh.empty(rt, (n,), np.bool_)
        rt.enqueue(ir.Instr(ir.OPCODES[name], [out.view(), a.view(), b.view()]))
        return [out]
    return prog


def logical_program(name, n=1000, seed=0):
    def prog(rt):
        a, b = bh.array(rt, data(n, np.bool_, seed)), bh.array(rt, data(n, np.bool_, seed + 1))
        out = bh.empty(rt, (n,), np.bool_)
        rt.enqueue(ir.Instr(ir.OPCODES[name], [out.view(), a.view(), b.view()]))
        return [out]
    return prog


def unary_inputs(name, dtype, n=1000, seed=0):
    """The operand of unary_program: inside each function's domain, with NaNs and infinities for
    the predicates."""
    dt = np.dtype(dtype)
    if dt.kind == "f":
        lo, hi = {"ARCCOSH": (1.0, 5.0), "ARCTANH": (-0.9, 0.9), "ARCSIN": (-1, 1), "ARCCOS": (-1, 1),
                  "LOG": (0.01, 9), "LOG2": (0.01, 9), "LOG10": (0.01, 9), "SQRT": (0, 9),
                  "LOG1P": (-0.5, 9)}.get(name, (-3.0, 3.0))
        A = data(n, dt, seed, lo, hi)
        if name in ("ISNAN", "ISINF", "ISFINITE"):
            A[::7] = np.nan
            A[1::11] = np.inf
    else:
        A = data(n, dt, seed)
    return A


def unary_program(name, dtype, n=1000, seed=0):
    dt = np.dtype(dtype)
    out_dt = np.bool_ if name in ("ISNAN", "ISINF", "ISFINITE") else dt

    def prog(rt):
        a = bh.array(rt, unary_inputs(name, dt, n, seed))
        out = bh.empty(rt, (n,), out_dt)
        rt.enqueue(ir.Instr(ir.OPCODES[name], [out.view(), a.view()]))
        return [out]
    return prog


def identity_inputs(src_dt, dst_dt, n=500, seed=0):
    """The source array of identity_program: values every destination type holds (no negative
    values for unsigned destinations, floats within +-100)."""
    s = np.dtype(src_dt)
    if s.kind == "f":
        return data(n, s, seed, -100.0 if np.dtype(dst_dt).kind in "if" else 0.0, 100.0)
    return data(n, s, seed, 0 if np.dtype(dst_dt).kind == "u" else None)


def identity_program(src_dt, dst_dt, n=500, seed=0):
    def prog(rt):
        a = bh.array(rt, identity_inputs(src_dt, dst_dt, n, seed))
        return [a.astype(dst_dt)]
    return prog


REDUCE_OPS = ["ADD_REDUCE", "MULTIPLY_REDUCE", "MINIMUM_REDUCE", "MAXIMUM_REDUCE", "BITWISE_AND_REDUCE",
              "BITWISE_OR_REDUCE", "BITWISE_XOR_REDUCE", "LOGICAL_AND_REDUCE", "LOGICAL_OR_REDUCE",
              "LOGICAL_XOR_REDUCE"]


def reduce_program(name, dtype, shape, axis, view="plain", seed=0):
    dt = np.dtype(dtype)

    def prog(rt):
        if name == "MULTIPLY_REDUCE" and dt.kind == "f":
            A = data(shape, dt, seed, 0.9, 1.1)
        elif name == "MULTIPLY_REDUCE":
            A = data(shape, dt, seed, 1, 2)
        else:
            A = data(shape, dt, seed)
        a = bh.array(rt, A)
        if view == "transposed":
            a = a.T
        elif view == "sliced":
            a = a[tuple(slice(1, None, 2) if s > 2 else slice(None) for s in a.shape)]
        elif view == "reversed":
            a = a[tuple(slice(None, None, -1) for _ in a.shape)]
        return [bh.reduce(name, a, axis)]
    return prog


def accumulate_program(name, dtype, shape, axis, seed=0):
    def prog(rt):
        A = data(shape, dtype, seed, 0.5, 1.5) if np.dtype(dtype).kind == "f" else data(shape, dtype, seed, 1, 3)
        a = bh.array(rt, A)
        return [bh.accumulate(name, a, axis)]
    return prog


def views_program(seed=0):
    """Strided, negative-stride, broadcast and 3-D views in one fused chain."""
    def prog(rt):
        A = data((6, 7, 8), np.float64, seed)
        B = data((8,), np.float64, seed + 1)
        a, b = bh.array(rt, A), bh.array(rt, B)
        x = a[::-1, 1:6:2, :] * b          # broadcast along the last axis
        y = (x + a[:, 1:6:2, ::-1].transpose((0, 1, 2)))
        z = y.sum(axis=1)
        return [x, y, z]
    return prog


def random_program(shape, start, key):
    def prog(rt):
        r = bh.random123(rt, shape, start, key)
        f = bh.random_sample(rt, shape, start, key, np.float32)
        return [r, f]
    return prog


def gather_scatter_program(n=1000, seed=0):
    def prog(rt):
        rng = np.random.default_rng(seed)
        src = bh.array(rt, rng.random(n))
        idx = bh.array(rt, rng.permutation(n).astype(np.uint64))
        g = bh.gather(src, idx)
        dst = bh.zeros(rt, (n,), np.float64)
        bh.scatter(dst, g, idx)
        return [g, dst]
    return prog


def range_program(n=1000):
    def prog(rt):
        r = bh.arange(rt, n, np.uint64)
        return [r, r[10:500:3] * 2]
    return prog


def fused_chain_program(n, dtype=np.float64, seed=0):
    """A longer elementwise chain with a full reduction and an axis reduction."""
    def prog(rt):
        A, B = data(n, dtype, seed), data(n, dtype, seed + 1)
        a, b = bh.array(rt, A), bh.array(rt, B)
        y = bh.sqrt(a * a + b * b) * bh.exp(-b) + bh.maximum(a, b) * 0.5
        m = (y * 2).reshape(n // 4, 4)
        return [y, y.sum(), y.max(), m.sum(axis=1), m.sum(axis=0)]
    return prog


def empty_program():
    """Zero-length arrays and reductions of them."""
    def prog(rt):
        a = bh.array(rt, np.zeros(0))
        b = a * 2 + 1
        return [b]
    return prog


# ----------------------------------------------------------------------------- complex numbers
# The reference's complex type signatures (core/codegen/opcodes.json): ADD, SUBTRACT, MULTIPLY,
# DIVIDE, POWER; COS ... TANH, EXP, LOG, LOG10, SQRT, SIGN, CONJ (complex -> complex); ABSOLUTE,
# REAL, IMAG (complex -> real); ISNAN, ISINF, ISFINITE, EQUAL, NOT_EQUAL (-> bool); IDENTITY from
# every type; ADD/MULTIPLY reductions and accumulates; GATHER, SCATTER, COND_SCATTER.
COMPLEX_TYPES = [np.complex64, np.complex128]
COMPLEX_BINARY = ["ADD", "SUBTRACT", "MULTIPLY", "DIVIDE", "POWER"]
COMPLEX_UNARY = ["COS", "SIN", "TAN", "COSH", "SINH", "TANH", "EXP", "LOG", "LOG10", "SQRT", "SIGN", "CONJ"]
COMPLEX_TO_REAL = ["ABSOLUTE", "REAL", "IMAG"]
COMPLEX_PREDICATES = ["ISNAN", "ISINF", "ISFINITE"]
COMPLEX_TRANSCENDENTAL = {"COS", "SIN", "TAN", "COSH", "SINH", "TANH", "EXP", "LOG", "LOG10", "SQRT", "POWER",
                          "ABSOLUTE", "DIVIDE"}


def real_dtype(dtype):
    return np.dtype(np.float32) if np.dtype(dtype) == np.complex64 else np.dtype(np.float64)


def cdata(shape, dtype, seed, lo=-2.0, hi=2.0):
    """Seeded complex values with real and imaginary parts uniform in [lo, hi)."""
    rng = np.random.default_rng(seed)
    re = rng.random(shape) * (hi - lo) + lo
    im = rng.random(shape) * (hi - lo) + lo
    return (re + 1j * im).astype(dtype)


def complex_binary_program(name, dtype, n=1000, seed=0):
    def prog(rt):
        A = cdata(n, dtype, seed, 0.1, 2.0)
        B = cdata(n, dtype, seed + 1, 0.1 if name in ("DIVIDE", "POWER") else -2.0, 1.5)
        a, b = bh.array(rt, A), bh.array(rt, B)
        out = bh.empty(rt, (n,), dtype)
        rt.enqueue(ir.Instr(ir.OPCODES[name], [out.view(), a.view(), b.view()]))
        out2 = bh.empty(rt, (n,), dtype)
        rt.enqueue(ir.Instr(ir.OPCODES[name], [out2.view(), a.view(), None],
                            ir.Constant(complex(B[3]), ir.bh_type(np.dtype(dtype)))))
        return [out, out2]
    return prog


def complex_unary_program(name, dtype, n=1000, seed=0):
    dt = np.dtype(dtype)
    out_dt = {**{k: real_dtype(dt) for k in COMPLEX_TO_REAL},
              **{k: np.dtype(np.bool_) for k in COMPLEX_PREDICATES}}.get(name, dt)

    def prog(rt):
        A = cdata(n, dt, seed)
        if name == "SIGN":
            A.real[::5] = 0  # the imaginary part decides there
            A[::25] = 0
        if name in COMPLEX_PREDICATES:
            A.real[::7] = np.nan
            A.imag[3::7] = np.nan  # a NaN imaginary part alone: the reference tests the real part
            A.real[1::11] = np.inf
            A.imag[5::11] = np.inf
        a = bh.array(rt, A)
        out = bh.empty(rt, (n,), out_dt)
        rt.enqueue(ir.Instr(ir.OPCODES[name], [out.view(), a.view()]))
        return [out]
    return prog


def complex_compare_program(name, dtype, n=1000, seed=0):
    def prog(rt):
        A = cdata(n, dtype, seed)
        B = cdata(n, dtype, seed + 1)
        B[::3] = A[::3]
        B.real[1::5] = A.real[1::5]  # equal real parts, different imaginary parts
        a, b = bh.array(rt, A), bh.array(rt, B)
        out = bh.empty(rt, (n,), np.bool_)
        rt.enqueue(ir.Instr(ir.OPCODES[name], [out.view(), a.view(), b.view()]))
        return [out]
    return prog


def complex_identity_program(src_dt, dst_dt, n=500, seed=0):
    def prog(rt):
        s = np.dtype(src_dt)
        if s.kind == "c":
            A = cdata(n, s, seed, -100.0, 100.0)
        elif s.kind == "f":
            A = data(n, s, seed, -100.0, 100.0)
        else:
            A = data(n, s, seed)
        return [bh.array(rt, A).astype(dst_dt)]
    return prog


def complex_reduce_program(name, dtype, shape, axis, seed=0):
    def prog(rt):
        if name == "MULTIPLY_REDUCE":
            # |z| near 1 and small phases, so long products stay finite
            rng = np.random.default_rng(seed)
            A = ((0.95 + 0.1 * rng.random(shape)) * np.exp(0.05j * (rng.random(shape) - 0.5))).astype(dtype)
        else:
            A = cdata(shape, dtype, seed)
        return [bh.reduce(name, bh.array(rt, A), axis)]
    return prog


def complex_accumulate_input(name, dtype, shape, seed=0):
    """Factors of modulus 0.98-1.02 near the real axis for products (no overflow or underflow over
    1e6 of them), values in [-2, 2) + i[-2, 2) for sums."""
    if name == "MULTIPLY_ACCUMULATE":
        rng = np.random.default_rng(seed)
        return ((0.98 + 0.04 * rng.random(shape)) * np.exp(0.05j * (rng.random(shape) - 0.5))).astype(dtype)
    return cdata(shape, dtype, seed)


def complex_accumulate_program(name, dtype, shape, axis, seed=0):
    def prog(rt):
        A = complex_accumulate_input(name, dtype, shape, seed)
        return [bh.accumulate(name, bh.array(rt, A), axis)]
    return prog


def complex_gather_scatter_program(dtype, n=1000, seed=0):
    def prog(rt):
        rng = np.random.default_rng(seed)
        src = bh.array(rt, cdata(n, dtype, seed))
        idx = bh.array(rt, rng.permutation(n).astype(np.uint64))
        g = bh.gather(src, idx)
        dst = bh.zeros(rt, (n,), dtype)
        bh.scatter(dst, g, idx)
        return [g, dst]
    return prog


def complex_chain_program(n, dtype=np.complex128, seed=0):
    """A fused complex chain: twiddle factors exp(i*theta) applied to a signal, a complex sum,
    the power |z|^2 as a real array and its sum."""
    def prog(rt):
        rdt = real_dtype(dtype)
        x = bh.array(rt, cdata(n, dtype, seed))
        theta = bh.array(rt, data(n, rdt, seed + 1, -3.0, 3.0))
        w = bh.exp(theta.astype(dtype) * 1j)
        z = w * x + bh.conj(x) * 0.5
        p = bh.real(z) * bh.real(z) + bh.imag(z) * bh.imag(z)
        return [z, z.sum(), p, p.sum(), bh.absolute(z)]
    return prog


def loop_triangular_numbers(rt, niter=10):
    """a[i+1] += a[i] for niter iterations of one flush-and-repeat, the three views sliding by one
    element per iteration (the reference's test_loop_faculty_function_using_sliding_views).
    Returns the result and NumPy's loop."""
    host = np.arange(1, niter + 2, dtype=np.int64)
    a = bh.array(rt, host)
    rt.flush()
    ins = ir.Instr(ir.OPCODES["ADD"], [ir.View(a.base, 1, (1,), (1,)), ir.View(a.base, 1, (1,), (1,)),
                                       ir.View(a.base, 0, (1,), (1,))])
    for k in range(3):
        ins.slides[k] = ([ir.Slide(0, 1, 0, 1, niter + 1)], {})
    rt.ex.execute(ir.Flush([ins], nrepeats=niter))
    want = host.copy()
    for i in range(niter):
        want[i + 1] += want[i]
    return a.numpy(), want


def loop_diagonal(rt, niter=5):
    """res[i] += b[i, i] for niter iterations, the (1, 1) view of b sliding along both axes (the
    reference's test_loop_one_and_two_dimensional_sliding_views). Returns the result and NumPy's
    loop."""
    B = np.ones((20, niter))
    B[::2, ::2] += 1
    B[1::2, 1::2] += 1
    b = bh.array(rt, B)
    res = bh.zeros(rt, (niter, 1), np.float64)
    rt.flush()
    ins = ir.Instr(ir.OPCODES["ADD"], [ir.View(res.base, 0, (1, 1), (1, 1)), ir.View(res.base, 0, (1, 1), (1, 1)),
                                       ir.View(b.base, 0, (1, 1), (niter, 1))])
    for k in range(2):
        ins.slides[k] = ([ir.Slide(0, 1, 0, 1, niter)], {})
    ins.slides[2] = ([ir.Slide(0, 1, 0, niter, 20), ir.Slide(1, 1, 0, 1, niter)], {})
    rt.ex.execute(ir.Flush([ins], nrepeats=niter))
    want = np.zeros((niter, 1))
    for i in range(niter):
        want[i] += B[i, i]
    return res.numpy(), want
