"""A small NumPy-like array front end that emits Bohrium bytecode.

Each operation appends instructions to a Runtime's queue (like bhxx::BhArray of the reference,
bridge/cxx/include/bhxx/BhArray.hpp). Arrays own their base: when the owning array is garbage
collected a BH_FREE is enqueued, which lets the fuser contract temporaries. Reductions over
several axes are lowered one axis at a time, largest stride first, as the reference's Python
bridge does on GPU stacks (bridge/npbackend/bohrium/ufuncs.pyx:371-440).
"""
from __future__ import annotations

import numbers
from typing import Optional, Sequence

import numpy as np

from . import ir
from .runtime import Runtime

OP = ir.OPCODES


def _contig_strides(shape):
    s, out = 1, []
    for n in reversed(shape):
        out.append(s)
        s *= n
    return tuple(reversed(out))


class BhArray:
    __slots__ = ("rt", "base", "start", "shape", "strides", "_owner", "__weakref__")

    def __init__(self, rt: Runtime, base: ir.Base, start: int, shape, strides, owner=None):
        self.rt = rt
        self.base = base
        self.start = int(start)
        self.shape = tuple(int(s) for s in shape)
        self.strides = tuple(int(s) for s in strides)
        self._owner = owner  # the array owning `base` (None: this array owns it)

    def __del__(self):
        try:
            if self._owner is None and self.base is not None and self.rt is not None:
                self.rt.free(self.base)
        except Exception:
            pass

    # -- properties ------------------------------------------------------------------------
    @property
    def dtype(self):
        return self.base.dtype

    @property
    def ndim(self):
        return len(self.shape)

    @property
    def size(self):
        return int(np.prod(self.shape, dtype=np.int64)) if self.shape else 1

    def view(self) -> ir.View:
        # Zero-dimensional arrays travel as one-element 1-D views, as the reference's bridge sends
        # them (bridge/npbackend/src/bharray.c:41-45).
        if self.ndim == 0:
            return ir.View(self.base, self.start, (1,), (1,))
        return ir.View(self.base, self.start, self.shape, self.strides)

    def _root(self):
        return self if self._owner is None else self._owner

    def __repr__(self):
        return f"BhArray(shape={self.shape}, dtype={self.dtype}, base={self.base})"

    # -- views -----------------------------------------------------------------------------
    def __getitem__(self, key):
        if not isinstance(key, tuple):
            key = (key,)
        if any(k is Ellipsis for k in key):
            i = [j for j, k in enumerate(key) if k is Ellipsis][0]
            fill = self.ndim - (len(key) - 1)
            key = key[:i] + (slice(None),) * fill + key[i + 1:]
        key = key + (slice(None),) * (self.ndim - len(key))
        start = self.start
        shape, strides = [], []
        for k, n, s in zip(key, self.shape, self.strides):
            if isinstance(k, slice):
                a, b, c = k.indices(n)
                cnt = len(range(a, b, c))
                start += a * s
                shape.append(cnt)
                strides.append(s * c)
            elif isinstance(k, numbers.Integral):
                k = int(k)
                if k < 0:
                    k += n
                if not 0 <= k < n:
                    raise IndexError("index out of range")
                start += k * s
            else:
                raise TypeError("unsupported index: only integers and slices")
        return BhArray(self.rt, self.base, start, shape, strides, self._root())

    def __setitem__(self, key, value):
        self[key].assign(value)

    def assign(self, value):
        """self[...] = value (BH_IDENTITY with broadcasting and casting)."""
        if isinstance(value, BhArray):
            src = value._broadcast_to(self.shape)
            self.rt.enqueue(ir.Instr(OP["IDENTITY"], [self.view(), src.view()]))
        else:
            self.rt.enqueue(ir.Instr(OP["IDENTITY"], [self.view(), None], ir.Constant(value, ir.bh_type(self.dtype))))
        return self

    def transpose(self, axes: Optional[Sequence[int]] = None):
        axes = list(reversed(range(self.ndim))) if axes is None else list(axes)
        return BhArray(self.rt, self.base, self.start, [self.shape[a] for a in axes], [self.strides[a] for a in axes],
                       self._root())

    @property
    def T(self):
        return self.transpose()

    def is_contiguous(self):
        return self.strides == _contig_strides(self.shape) or self.size <= 1

    def reshape(self, *shape):
        if len(shape) == 1 and isinstance(shape[0], (tuple, list)):
            shape = tuple(shape[0])
        shape = list(shape)
        if -1 in shape:
            i = shape.index(-1)
            rest = int(np.prod([s for s in shape if s != -1])) or 1
            shape[i] = self.size // rest
        if int(np.prod(shape)) != self.size:
            raise ValueError("reshape: size mismatch")
        src = self if self.is_contiguous() else self.copy()
        return BhArray(self.rt, src.base, src.start, shape, _contig_strides(shape), src._root())

    def flatten(self):
        return self.reshape(-1)

    def _broadcast_to(self, shape):
        shape = tuple(shape)
        if self.shape == shape:
            return self
        nd = len(shape)
        if self.ndim > nd:
            raise ValueError(f"cannot broadcast {self.shape} to {shape}")
        pad = nd - self.ndim
        src_shape = (1,) * pad + self.shape
        src_strides = (0,) * pad + self.strides
        strides = []
        for n_src, s_src, n in zip(src_shape, src_strides, shape):
            if n_src == n:
                strides.append(s_src)
            elif n_src == 1:
                strides.append(0)
            else:
                raise ValueError(f"cannot broadcast {self.shape} to {shape}")
        return BhArray(self.rt, self.base, self.start, shape, strides, self._root())

    # -- conversion ------------------------------------------------------------------------
    def copy(self):
        out = self.rt_empty(self.shape, self.dtype)
        out.assign(self)
        return out

    def astype(self, dtype):
        dtype = np.dtype(dtype)
        if dtype == self.dtype:
            return self
        out = self.rt_empty(self.shape, dtype)
        out.assign(self)
        return out

    def rt_empty(self, shape, dtype):
        return empty(self.rt, shape, dtype)

    def numpy(self) -> np.ndarray:
        """Flush and return a NumPy copy (the reference's copy2numpy)."""
        self.rt.flush(syncs=[self.base])
        host = self.rt.ex.get_data(self.base)
        if self.ndim == 0:
            return host[self.start].copy()
        it = host.itemsize
        return np.lib.stride_tricks.as_strided(host[self.start:], shape=self.shape,
                                               strides=[s * it for s in self.strides]).copy()

    def item(self):
        return self.numpy().reshape(-1)[0].item()

    # -- arithmetic ------------------------------------------------------------------------
    def __add__(self, o): return binary("ADD", self, o)
    def __radd__(self, o): return binary("ADD", o, self)
    def __sub__(self, o): return binary("SUBTRACT", self, o)
    def __rsub__(self, o): return binary("SUBTRACT", o, self)
    def __mul__(self, o): return binary("MULTIPLY", self, o)
    def __rmul__(self, o): return binary("MULTIPLY", o, self)
    def __truediv__(self, o): return true_divide(self, o)
    def __rtruediv__(self, o): return true_divide(o, self)
    def __floordiv__(self, o): return binary("DIVIDE", self, o)
    def __rfloordiv__(self, o): return binary("DIVIDE", o, self)
    def __pow__(self, o): return binary("POWER", self, o)
    def __rpow__(self, o): return binary("POWER", o, self)
    def __mod__(self, o): return binary("REMAINDER", self, o)
    def __rmod__(self, o): return binary("REMAINDER", o, self)
    def __and__(self, o): return binary("BITWISE_AND", self, o)
    def __or__(self, o): return binary("BITWISE_OR", self, o)
    def __xor__(self, o): return binary("BITWISE_XOR", self, o)
    def __lshift__(self, o): return binary("LEFT_SHIFT", self, o)
    def __rshift__(self, o): return binary("RIGHT_SHIFT", self, o)
    def __gt__(self, o): return binary("GREATER", self, o, out_dtype=np.bool_)
    def __ge__(self, o): return binary("GREATER_EQUAL", self, o, out_dtype=np.bool_)
    def __lt__(self, o): return binary("LESS", self, o, out_dtype=np.bool_)
    def __le__(self, o): return binary("LESS_EQUAL", self, o, out_dtype=np.bool_)
    def __eq__(self, o): return binary("EQUAL", self, o, out_dtype=np.bool_)
    def __ne__(self, o): return binary("NOT_EQUAL", self, o, out_dtype=np.bool_)
    def __neg__(self): return binary("MULTIPLY", self, -1)
    def __abs__(self): return absolute(self)
    def __invert__(self): return unary("INVERT", self)
    __hash__ = object.__hash__

    def sum(self, axis=None): return reduce("ADD_REDUCE", self, axis)
    def prod(self, axis=None): return reduce("MULTIPLY_REDUCE", self, axis)
    def max(self, axis=None): return reduce("MAXIMUM_REDUCE", self, axis)
    def min(self, axis=None): return reduce("MINIMUM_REDUCE", self, axis)
    def any(self, axis=None): return reduce("LOGICAL_OR_REDUCE", self.astype(np.bool_), axis)
    def all(self, axis=None): return reduce("LOGICAL_AND_REDUCE", self.astype(np.bool_), axis)

    def mean(self, axis=None):
        s = self.sum(axis)
        n = self.size if axis is None else self.shape[axis]
        return true_divide(s, n)

    def cumsum(self, axis=0): return accumulate("ADD_ACCUMULATE", self, axis)
    def cumprod(self, axis=0): return accumulate("MULTIPLY_ACCUMULATE", self, axis)


# ------------------------------------------------------------------------------ construction
def empty(rt: Runtime, shape, dtype=np.float64) -> BhArray:
    shape = (shape,) if isinstance(shape, numbers.Integral) else tuple(shape)
    n = int(np.prod(shape, dtype=np.int64)) if shape else 1
    base = rt.new_base(dtype, n)
    return BhArray(rt, base, 0, shape, _contig_strides(shape))


def full(rt: Runtime, shape, value, dtype=np.float64) -> BhArray:
    a = empty(rt, shape, dtype)
    a.assign(value)
    return a


def zeros(rt, shape, dtype=np.float64):
    return full(rt, shape, 0, dtype)


def ones(rt, shape, dtype=np.float64):
    return full(rt, shape, 1, dtype)


def array(rt: Runtime, data, dtype=None) -> BhArray:
    data = np.asarray(data, dtype=dtype)
    a = empty(rt, data.shape, data.dtype)
    rt.ex.set_data(a.base, data)
    return a


def arange(rt: Runtime, n: int, dtype=np.int64) -> BhArray:
    idx = empty(rt, (n,), np.uint64)
    rt.enqueue(ir.Instr(OP["RANGE"], [idx.view()]))
    return idx if np.dtype(dtype) == np.uint64 else idx.astype(dtype)


def random123(rt: Runtime, shape, start: int, key: int) -> BhArray:
    """BH_RANDOM: uint64 Philox2x32-10 of counter start+i with the low 32 bits of `key`."""
    out = empty(rt, shape, np.uint64)
    rt.enqueue(ir.Instr(OP["RANDOM"], [out.view(), None], ir.Constant((start, key), ir.R123)))
    return out


def random_sample(rt: Runtime, shape, start: int = 0, key: int = 42, dtype=np.float64) -> BhArray:
    """Uniform [0, 1): float(uint64) / float(UINT64_MAX) (bridge/npbackend/bohrium/random123.pyx:258-267)."""
    r = random123(rt, shape, start, key)
    f = r.astype(dtype)
    del r
    return binary("DIVIDE", f, dtype(np.iinfo(np.uint64).max) if callable(dtype) else np.dtype(dtype).type(
        np.iinfo(np.uint64).max))


# --------------------------------------------------------------------------------- operations
def _result_type(a, b):
    ta = a.dtype if isinstance(a, BhArray) else None
    tb = b.dtype if isinstance(b, BhArray) else None
    if ta is not None and tb is not None:
        return np.result_type(ta, tb)
    t = ta if ta is not None else tb
    s = b if ta is not None else a
    if isinstance(s, (bool, np.bool_)):
        return t
    if isinstance(s, numbers.Integral):
        return t
    if isinstance(s, numbers.Real):
        return t if np.issubdtype(t, np.inexact) else np.dtype(np.float64)
    if isinstance(s, numbers.Complex):
        if np.issubdtype(t, np.complexfloating):
            return t
        return np.dtype(np.complex64) if t == np.float32 else np.dtype(np.complex128)
    return np.result_type(t, np.asarray(s).dtype)


def _operand(x, dtype, shape):
    if isinstance(x, BhArray):
        if x.dtype != dtype:
            x = x.astype(dtype)
        return x._broadcast_to(shape), None
    return None, ir.Constant(np.asarray(x).astype(dtype).item() if dtype != np.bool_ else bool(x), ir.bh_type(dtype))


def binary(name: str, a, b, out_dtype=None, out: Optional[BhArray] = None) -> BhArray:
    rt = a.rt if isinstance(a, BhArray) else b.rt
    dtype = _result_type(a, b)
    shape = np.broadcast_shapes(a.shape if isinstance(a, BhArray) else (), b.shape if isinstance(b, BhArray) else ())
    if out is None:
        out = empty(rt, shape, out_dtype if out_dtype is not None else dtype)
    va, ca = _operand(a, dtype, shape)
    vb, cb = _operand(b, dtype, shape)
    if ca is not None and cb is not None:
        raise ValueError("binary(): two constants")
    const = ca if ca is not None else cb
    rt.enqueue(ir.Instr(OP[name], [out.view(), va.view() if va is not None else None,
                                   vb.view() if vb is not None else None], const))
    return out


def unary(name: str, a: BhArray, out_dtype=None, out: Optional[BhArray] = None) -> BhArray:
    if out is None:
        out = empty(a.rt, a.shape, out_dtype if out_dtype is not None else a.dtype)
    a.rt.enqueue(ir.Instr(OP[name], [out.view(), a._broadcast_to(out.shape).view()]))
    return out


def true_divide(a, b):
    def f(x):
        if isinstance(x, BhArray) and not np.issubdtype(x.dtype, np.inexact):
            return x.astype(np.float64)
        return x
    return binary("DIVIDE", f(a), f(b))


def reduce(name: str, a: BhArray, axis=None) -> BhArray:
    if name in ("ADD_REDUCE", "MULTIPLY_REDUCE") and a.dtype == np.bool_:
        a = a.astype(np.uint64)
    if axis is None:
        axes = list(range(a.ndim))
    elif isinstance(axis, numbers.Integral):
        axes = [axis]
    else:
        axes = list(axis)
    axes = [x + a.ndim if x < 0 else x for x in axes]
    if len(axes) == 1:
        ax = axes[0]
        shape = tuple(s for i, s in enumerate(a.shape) if i != ax)
        out = empty(a.rt, shape, a.dtype)
        a.rt.enqueue(ir.Instr(OP[name], [out.view(), a.view(), None], ir.Constant(ax, ir.INT64)))
        return out
    # Largest stride first (column-major order, as the reference bridge does for GPU stacks) where
    # the order can change the result (floating-point sums and products); reductions whose result
    # does not depend on the order (max, min, logical and bitwise ones, integer sums and
    # products) go smallest stride first, so the first one sweeps the contiguous axis.
    order_free = name not in ("ADD_REDUCE", "MULTIPLY_REDUCE") or a.dtype.kind in "biu"
    order = sorted(axes, key=lambda i: abs(a.strides[i]), reverse=not order_free)
    first = order[0]
    tmp = reduce(name, a, first)
    rest = [i if i < first else i - 1 for i in order[1:]]
    return reduce(name, tmp, rest)


def accumulate(name: str, a: BhArray, axis=0) -> BhArray:
    out = empty(a.rt, a.shape, a.dtype)
    a.rt.enqueue(ir.Instr(OP[name], [out.view(), a.view(), None], ir.Constant(axis, ir.INT64)))
    return out


def gather(src: BhArray, index: BhArray) -> BhArray:
    """out[i] = src.flat[index[i]] (BH_GATHER; `src` is read as a flat array from its start)."""
    out = empty(src.rt, index.shape, src.dtype)
    src.rt.enqueue(ir.Instr(OP["GATHER"], [out.view(), src.view(), index.view()]))
    return out


def scatter(dst: BhArray, values: BhArray, index: BhArray) -> None:
    """dst.flat[index[i]] = values[i] (BH_SCATTER)."""
    dst.rt.enqueue(ir.Instr(OP["SCATTER"], [dst.view(), values.view(), index.view()]))


def _make_unary(name, float_only=False):
    def f(a, out=None):
        if float_only and not np.issubdtype(a.dtype, np.inexact):
            a = a.astype(np.float64)
        return unary(name, a, out=out)
    f.__name__ = name.lower()
    return f


def _real_dtype(dt):
    return np.dtype(np.float32) if dt == np.complex64 else np.dtype(np.float64)


def _complex_part(name):
    def f(a, out=None):
        if not np.issubdtype(a.dtype, np.complexfloating):
            raise TypeError(f"{name.lower()}(): complex array expected")
        return unary(name, a, out_dtype=_real_dtype(a.dtype), out=out)
    f.__name__ = name.lower()
    return f


sqrt = _make_unary("SQRT", True)
exp = _make_unary("EXP", True)
log = _make_unary("LOG", True)
sin = _make_unary("SIN", True)
cos = _make_unary("COS", True)
tanh = _make_unary("TANH", True)
floor = _make_unary("FLOOR", True)
sign = _make_unary("SIGN")
tan = _make_unary("TAN", True)
sinh = _make_unary("SINH", True)
cosh = _make_unary("COSH", True)
log10 = _make_unary("LOG10", True)
real = _complex_part("REAL")
imag = _complex_part("IMAG")


def absolute(a, out=None):
    """|a| (BH_ABSOLUTE); the modulus, a real array, for complex input."""
    if np.issubdtype(a.dtype, np.complexfloating):
        return unary("ABSOLUTE", a, out_dtype=_real_dtype(a.dtype), out=out)
    return unary("ABSOLUTE", a, out=out)


def conj(a, out=None):
    """Complex conjugate (BH_CONJ)."""
    if not np.issubdtype(a.dtype, np.complexfloating):
        raise TypeError("conj(): complex array expected")
    return unary("CONJ", a, out=out)


def maximum(a, b):
    return binary("MAXIMUM", a, b)


def minimum(a, b):
    return binary("MINIMUM", a, b)


def where(cond: BhArray, a, b):
    """a if cond else b, written with arithmetic on the 0/1 mask (no select opcode exists)."""
    m = cond.astype(_result_type(a, b))
    return m * a + (1 - m) * b


# ------------------------------------------------------------------------------ extension methods
_EXT_BASE = ir.MAX_OPCODE_ID + 1


def extmethod_opcode(rt: Runtime, name: str) -> int:
    """The opcode of extension method `name`, registered with the runtime's stack on first use
    (bhc_extmethod of the reference's C bridge). The table lives with the executor (the stack),
    which keeps its registrations for its whole life."""
    table = rt.ex.__dict__.setdefault("_extmethods", {})
    if name not in table:
        opcode = _EXT_BASE + len(table)
        rt.ex.extmethod(name, opcode)
        table[name] = opcode
    return table[name]


def matmul(a: BhArray, b: BhArray, trans_a: bool = False) -> BhArray:
    """C = A @ B (or A^T @ B) of contiguous 2-D float32/float64 arrays through the stack's BLAS
    extension methods `blas_gemm` / `blas_gemmt` (operands C, A, B as in the reference's
    extmethods/blas)."""
    m = a.shape[1] if trans_a else a.shape[0]
    out = empty(a.rt, (m, b.shape[1]), a.dtype)
    op = extmethod_opcode(a.rt, "blas_gemmt" if trans_a else "blas_gemm")
    a.rt.enqueue(ir.Instr(op, [out.view(), a.view(), b.view()]))
    return out


def is_behaving(a: BhArray) -> bool:
    """A behaving array is C-contiguous, starts at the first element of its base and covers all
    of it, so a user kernel can index it without offsets or strides (the reference's
    `_bh.is_array_behaving`, used by bridge/npbackend/bohrium/user_kernel.py:62-71)."""
    return a.start == 0 and a.is_contiguous() and a.size == a.base.nelem


def make_behaving(a: BhArray, dtype=None) -> BhArray:
    """`a` (converted to `dtype`), copied if it is not behaving
    (bridge/npbackend/bohrium/user_kernel.py:120-150)."""
    if dtype is not None:
        a = a.astype(dtype)
    return a if is_behaving(a) else a.copy()


def _param_string(param) -> str:
    """{"global_work_size": (20, 5), ...} -> "global_work_size: 20 5; ..." (as the reference's
    front end builds it, bridge/npbackend/bohrium/user_kernel.py:76-83)."""
    parts = []
    for key, value in (param or {}).items():
        if isinstance(value, (list, tuple)):
            value = " ".join(str(v) for v in value)
        parts.append(f"{key}: {value}")
    return "; ".join(parts)


def user_kernel(kernel_source: str, operand_list: Sequence[BhArray], compiler_command: Optional[str] = None,
                tag: str = "openmp", param=None, only_behaving_operands: bool = True) -> None:
    """Compile and run the function `execute` of `kernel_source` with the arrays of `operand_list`
    as its arguments (bohrium.user_kernel.execute, bridge/npbackend/bohrium/user_kernel.py:21-89).

    Pending bytecode is flushed first. With tag "cuda" the stack's CUDA engine compiles the source
    with NVRTC: `execute` must be an `extern "C" __global__` function taking one pointer per
    operand, and `param` gives "global_work_size" and "local_work_size" (up to three dimensions,
    the global size a multiple of the local size). Raises RuntimeError with the engine's message
    when compilation or the launch fails, and TypeError for an operand that is not behaving
    unless `only_behaving_operands` is False."""
    ops = list(operand_list)
    if not ops:
        raise ValueError("user_kernel: operand_list is empty")
    for op in ops:
        if not isinstance(op, BhArray):
            raise TypeError("All operands in `operand_list` must be Bohrium arrays")
        if only_behaving_operands and not is_behaving(op):
            raise TypeError("Operand is not behaving set `only_behaving_operands=False` or use `make_behaving()`")
    rt = ops[0].rt
    rt.flush()
    msg = rt.ex.user_kernel(kernel_source, [op.base for op in ops], compiler_command or "", tag,
                            _param_string(param))
    if msg:
        raise RuntimeError(msg)
