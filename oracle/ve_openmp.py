"""CPU oracle engine: the reference's ve/openmp restated -- test infrastructure.

Every flushed BhIR is fused with oracle/jitk.py and each kernel is written as C99 with OpenMP
pragmas, compiled with `gcc -x c -fPIC -shared -std=gnu99 -O3 -march=native -fopenmp` and run on
the host cores, as ve/openmp/engine_openmp.cpp:122-248, 251-482 and ve/openmp/openmp_util.hpp:
27-94 of the reference do: `#pragma omp parallel for` on rank-0 loops, `reduction(op:var)` for
reductions whose output lives in a register, `atomic`/`critical` otherwise, serial loops for
accumulates. Operation semantics follow core/jitk/instruction.cpp:58-544.

`OracleExecutor` implements the executor interface of bohrium_b200.runtime (register, release,
set_data, get_data, execute), so a bohrium_b200.Runtime can drive it exactly like the GPU stack.
"""
from __future__ import annotations

import ctypes
import hashlib
import os
import subprocess
import tempfile
import time
from typing import Optional

import numpy as np

from bohrium_b200 import ir
from . import jitk
from .jitk import I, IB, Loop, OP, V

HERE = os.path.dirname(os.path.abspath(__file__))
CC = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
CFLAGS = ["-x", "c", "-fPIC", "-shared", "-std=gnu99", "-O3", "-march=native", "-fopenmp"]

_CTYPE = {np.dtype(np.bool_): "bool", np.dtype(np.int8): "int8_t", np.dtype(np.int16): "int16_t",
          np.dtype(np.int32): "int32_t", np.dtype(np.int64): "int64_t", np.dtype(np.uint8): "uint8_t",
          np.dtype(np.uint16): "uint16_t", np.dtype(np.uint32): "uint32_t", np.dtype(np.uint64): "uint64_t",
          np.dtype(np.float32): "float", np.dtype(np.float64): "double",
          np.dtype(np.complex64): "float complex", np.dtype(np.complex128): "double complex"}

_RED = {"ADD_REDUCE": "+", "MULTIPLY_REDUCE": "*", "BITWISE_AND_REDUCE": "&", "BITWISE_OR_REDUCE": "|",
        "BITWISE_XOR_REDUCE": "^", "MAXIMUM_REDUCE": "max", "MINIMUM_REDUCE": "min"}
_ATOMIC = {"ADD_REDUCE", "MULTIPLY_REDUCE", "BITWISE_AND_REDUCE", "BITWISE_OR_REDUCE", "BITWISE_XOR_REDUCE"}


def ctype(dt) -> str:
    dt = np.dtype(dt)
    if dt not in _CTYPE:
        raise NotImplementedError(f"oracle: element type {dt} not supported")
    return _CTYPE[dt]


def _isfloat(dt):
    return np.issubdtype(np.dtype(dt), np.floating)


def _iscomplex(dt):
    return dt is not None and np.issubdtype(np.dtype(dt), np.complexfloating)


def _is_signed(dt):
    return np.issubdtype(np.dtype(dt), np.signedinteger)


def _is_unsigned(dt):
    return np.issubdtype(np.dtype(dt), np.unsignedinteger)


def _reduce_expr(name, acc, x):
    return {"ADD_REDUCE": f"{acc} + {x}", "MULTIPLY_REDUCE": f"{acc} * {x}",
            "MINIMUM_REDUCE": f"{acc} < {x} ? {acc} : {x}", "MAXIMUM_REDUCE": f"{acc} > {x} ? {acc} : {x}",
            "LOGICAL_AND_REDUCE": f"{acc} && {x}", "LOGICAL_OR_REDUCE": f"{acc} || {x}",
            "LOGICAL_XOR_REDUCE": f"!{acc} != !{x}", "BITWISE_AND_REDUCE": f"{acc} & {x}",
            "BITWISE_OR_REDUCE": f"{acc} | {x}", "BITWISE_XOR_REDUCE": f"{acc} ^ {x}"}[name]


def op_statement(ins: I, ops, atomic=False) -> str:
    """One C statement for `ins` (core/jitk/instruction.cpp:58-544)."""
    name = ir.OPNAMES[ins.opcode]
    t0 = ins.ops[0].base.dtype if ins.ops and ins.ops[0] is not None else None
    t1 = None
    if len(ins.ops) > 1:
        if ins.ops[1] is not None:
            t1 = ins.ops[1].base.dtype
        else:
            t1 = np.dtype(np.uint64) if ins.const[1] == ir.R123 else np.dtype(ir.np_dtype(ins.const[1]))
    o = ops[0]
    if name in ir.REDUCTIONS:
        if atomic:
            sym = {"ADD_REDUCE": "+=", "MULTIPLY_REDUCE": "*=", "BITWISE_AND_REDUCE": "&=",
                   "BITWISE_OR_REDUCE": "|=", "BITWISE_XOR_REDUCE": "^="}[name]
            return f"{o} {sym} {ops[1]};"
        return f"{o} = {_reduce_expr(name, o, ops[1])};"
    bin_ = {"ADD": "+", "SUBTRACT": "-", "MULTIPLY": "*", "GREATER": ">", "GREATER_EQUAL": ">=", "LESS": "<",
            "LESS_EQUAL": "<=", "EQUAL": "==", "NOT_EQUAL": "!=", "LOGICAL_AND": "&&", "LOGICAL_OR": "||",
            "BITWISE_AND": "&", "BITWISE_OR": "|", "BITWISE_XOR": "^", "LEFT_SHIFT": "<<", "RIGHT_SHIFT": ">>"}
    if name in bin_:
        return f"{o} = {ops[1]} {bin_[name]} {ops[2]};"
    fn = {"COS": "cos", "SIN": "sin", "TAN": "tan", "COSH": "cosh", "SINH": "sinh", "TANH": "tanh", "ARCSIN": "asin",
          "ARCCOS": "acos", "ARCTAN": "atan", "ARCSINH": "asinh", "ARCCOSH": "acosh", "ARCTANH": "atanh",
          "EXP": "exp", "EXP2": "exp2", "EXPM1": "expm1", "LOG": "log", "LOG2": "log2", "LOG10": "log10",
          "LOG1P": "log1p", "SQRT": "sqrt", "CEIL": "ceil", "TRUNC": "trunc", "FLOOR": "floor", "RINT": "rint"}
    if name in fn and not (name == "LOG10" and _iscomplex(t0)):
        return f"{o} = {fn[name]}({ops[1]});"
    a = ops[1] if len(ops) > 1 else None
    b = ops[2] if len(ops) > 2 else None
    if name == "DIVIDE":
        if _is_signed(t0):
            return (f"{o} = (({a} > 0) != ({b} > 0) && ({a} % {b}) != 0) ? ({a} / {b} - 1) : ({a} / {b});")
        return f"{o} = {a} / {b};"
    if name == "POWER":
        if not _isfloat(t0) and not _iscomplex(t0):
            return f"{o} = pow((double) {a}, (double) {b});"
        return f"{o} = pow({a}, {b});"
    if name == "ABSOLUTE":
        if t1 == np.bool_ or _is_unsigned(t1):
            return f"{o} = {a};"
        if _isfloat(t1) or _iscomplex(t1):  # <tgmath.h>: fabs of a complex value is cabs
            return f"{o} = fabs({a});"
        if t1 == np.int64:
            return f"{o} = llabs({a});"
        return f"{o} = abs((int){a});"
    if name == "LOGICAL_XOR":
        return f"{o} = !{a} != !{b};"
    if name == "LOGICAL_NOT":
        return f"{o} = !{a};"
    if name == "MAXIMUM":
        return f"{o} = {a} > {b} ? {a} : {b};"
    if name == "MINIMUM":
        return f"{o} = {a} < {b} ? {a} : {b};"
    if name == "INVERT":
        return f"{o} = !{a};" if t0 == np.bool_ else f"{o} = ~{a};"
    if name == "ARCTAN2":
        return f"{o} = atan2({a}, {b});"
    if name == "MOD":
        return f"{o} = fmod({a}, {b});" if _isfloat(t0) else f"{o} = {a} % {b};"
    if name == "REMAINDER":
        if _isfloat(t0):
            return f"{o} = {a} - floor({a} / {b}) * {b};"
        if _is_unsigned(t0):
            return f"{o} = {a} % {b};"
        return f"{o} = (({a} > 0) == ({b} > 0) || ({a} % {b}) == 0) ? ({a} % {b}) : ({a} % {b}) + {b};"
    if name in ("ISNAN", "ISINF", "ISFINITE"):
        if _iscomplex(t1):  # the real part only (instruction.cpp:212-258)
            return f"{o} = {name.lower()}(creal({a}));"
        if _isfloat(t1):
            return f"{o} = {name.lower()}({a});"
        return f"{o} = {'true' if name == 'ISFINITE' else 'false'};"
    if name in ("IDENTITY", "RANGE", "RANDOM", "GATHER", "SCATTER"):
        return f"{o} = {a};"
    if name == "COND_SCATTER":
        return f"if ({ops[2]}) {{ {o} = {a}; }}"
    if name == "SIGN":
        if _iscomplex(t0):  # csgn: sgn(Re z), or sgn(Im z) where Re z == 0 (instruction.cpp:493-527)
            rt = "float" if t0 == np.complex64 else "double"
            return (f"{{ {rt} re_ = creal({a}), im_ = cimag({a}); "
                    f"{o} = (re_ == 0 ? ((im_ > 0) - (0 > im_)) : ((re_ > 0) - (0 > re_))); }}")
        return f"{o} = (({a} > 0) - (0 > {a}));"
    if name == "REAL":
        return f"{o} = creal({a});"
    if name == "IMAG":
        return f"{o} = cimag({a});"
    if name == "CONJ":
        return f"{o} = conj({a});"
    if name == "LOG10" and _iscomplex(t0):
        # C99 has no complex log10; the reference divides by log(10.0f), a float under <tgmath.h>
        # (instruction.cpp:459-475).
        return f"{o} = clog({a}) / log(10.0f);"
    if name == "ADD_ACCUMULATE":
        return f"{o} = {a} + {b};"
    if name == "MULTIPLY_ACCUMULATE":
        return f"{o} = {a} * {b};"
    raise NotImplementedError(f"oracle: opcode {name} not supported")


def _ignore_one_key(v: V):
    """View identity ignoring size-1 dimensions (the reference's IgnoreOneDim_less)."""
    return (v.base.id, v.start, tuple((s, st) for s, st in zip(v.shape, v.stride) if s > 1))


class _Kernel:
    """C source and argument layout of one fused kernel."""

    def __init__(self, kernel: Loop):
        self.kernel = kernel
        instrs = kernel.all_instr()
        self.base_ids, self.bases = {}, []
        always = set()
        for ins in instrs:
            nm = ir.OPNAMES[ins.opcode]
            if nm in ir.ACCUMULATES:
                always.add(ins.ops[0].base.id)
            elif nm == "GATHER":
                always.add(ins.ops[1].base.id)
            elif nm in ("SCATTER", "COND_SCATTER"):
                always.add(ins.ops[0].base.id)
            for v in ins.views():
                if v.base.id not in self.base_ids:
                    self.base_ids[v.base.id] = len(self.bases)
                    self.bases.append(v.base)
        self.temps = {b for b in kernel.all_temps() if b not in always}
        self.always = always
        self.params = [b for b in self.bases if b.id not in self.temps]
        self.param_idx = {b.id: k for k, b in enumerate(self.params)}
        self.meta: list = []
        self.view_off = {}
        for ins in instrs:
            for v in ins.views():
                k = v.key()
                if k not in self.view_off:
                    self.view_off[k] = len(self.meta)
                    self.meta.append(v.start)
                    self.meta.extend(v.stride)
        self.loop_off = {}
        self._collect_loops(kernel)
        self.consts, self.const_idx = [], {}
        for ins in instrs:
            if None in ins.ops and ir.OPNAMES[ins.opcode] not in ir.REDUCTIONS | ir.ACCUMULATES:
                self.const_idx[id(ins)] = len(self.consts)
                self.consts.append(ins)
        self.lines: list = []
        self._write()
        self.source = "\n".join(self.lines) + "\n"

    def _collect_loops(self, loop: Loop):
        for it in loop.items:
            if isinstance(it, Loop):
                self.loop_off[id(it)] = len(self.meta)
                self.meta.append(it.size)
                self._collect_loops(it)

    # -- expressions -----------------------------------------------------------------------
    def index(self, v: V, hidden=jitk.MAXDIM, prev_axis=-1):
        off = self.view_off[v.key()]
        parts = [f"m[{off}]"]
        if not v.is_scalar():
            for d in range(v.ndim):
                t = d + 1 if d >= hidden else d
                it = f"(i{t} == 0 ? 0 : i{t} - 1)" if t == prev_axis else f"i{t}"
                parts.append(f"{it} * m[{off + 1 + d}]")
        return "(" + " + ".join(parts) + ")"

    def aref(self, v: V, hidden=jitk.MAXDIM, prev_axis=-1):
        return f"a{self.param_idx[v.base.id]}[{self.index(v, hidden, prev_axis)}]"

    def name(self, v: V, scope, hidden=jitk.MAXDIM):
        if v.base.id in self.temps and scope.is_tmp(v.base.id):
            return f"t{self.base_ids[v.base.id]}"
        r = scope.repl(v)
        if r is not None:
            return r
        return self.aref(v, hidden)

    def const(self, ins: I):
        t = ctype(ir.np_dtype(ins.const[1]))
        return f"(*(const {t}*)(c + {16 * self.const_idx[id(ins)]}))"

    # -- writing ---------------------------------------------------------------------------
    def _write(self):
        L = self.lines
        L += ["#include <stdint.h>", "#include <stdlib.h>", "#include <stdbool.h>", "#include <complex.h>",
              "#include <tgmath.h>",
              "#include <math.h>", '#include "kernel_deps.h"', "",
              "void kernel(void **data, const int64_t *m, const unsigned char *c) {"]
        for k, b in enumerate(self.params):
            L.append(f"    {ctype(b.dtype)} *a{k} = ({ctype(b.dtype)} *)data[{k}];")
        self.atomic, self.critical = set(), set()
        self._body(self.kernel, _Scope(None), 4)
        L.append("}")

    def _body(self, loop: Loop, scope, ind):
        L = self.lines
        sp = " " * ind
        for bid in sorted(loop.local_temps(), key=lambda x: self.base_ids.get(x, 0)):
            if bid in self.temps and not scope.is_tmp(bid):
                scope.tmps.add(bid)
                b = self.bases[self.base_ids[bid]]
                L.append(f"{sp}{ctype(b.dtype)} t{self.base_ids[bid]};")
        replaced = []
        for sub in loop.subloops():
            for ins in sub.local_instr():
                if ir.OPNAMES[ins.opcode] in ir.REDUCTIONS and ins.sweep_axis() == ins.ops[1].ndim - 1:
                    v = ins.ops[0]
                    if scope.is_tmp(v.base.id) or scope.repl(v) is not None or v.base.id in self.always:
                        continue
                    nm = f"s{self.base_ids[v.base.id]}_{len(replaced)}_r{loop.rank + 1}"
                    scope.rep[_ignore_one_key(v)] = nm
                    replaced.append((v, ins))
                    L.append(f"{sp}{ctype(v.base.dtype)} {nm};")
        for it in loop.items:
            if isinstance(it, IB):
                self._instr(it.instr, scope, ind)
            else:
                if it.is_system_only():
                    continue
                self._loop_head(it, scope, ind)
                inner = _Scope(scope)
                self._body(it, inner, ind + 4)
                L.append(f"{sp}}}")
        for v, ins in replaced:
            if scope.is_tmp(v.base.id):
                continue
            L.append(f"{sp}{self.aref(v, ins.sweep_axis())} = {scope.rep[_ignore_one_key(v)]};")
            del scope.rep[_ignore_one_key(v)]

    def _loop_head(self, loop: Loop, scope, ind):
        sp = " " * ind
        size = f"m[{self.loop_off[id(loop)]}]"
        if loop.rank == 0 and loop.size > 1 and all(ir.OPNAMES[s.opcode] in ir.REDUCTIONS for s in loop.sweeps):
            clauses = ["parallel for"]
            for s in sorted(loop.sweeps, key=lambda s: self.view_off.get(s.ops[0].key(), 0)):
                nm = ir.OPNAMES[s.opcode]
                v = s.ops[0]
                local = scope.repl(v) is not None or scope.is_tmp(v.base.id)
                if nm in _RED and local:
                    clauses.append(f"reduction({_RED[nm]}:{self.name(v, scope)})")
                elif nm in _ATOMIC and not _iscomplex(v.base.dtype):
                    # gcc rejects `omp atomic` on complex lvalues, which the reference would emit
                    # (openmp_util.hpp:82-94); complex outputs take the critical section instead.
                    self.atomic.add(id(s))
                else:
                    self.critical.add(id(s))
            self.lines.append(f"{sp}#pragma omp " + " ".join(clauses))
        self.lines.append(f"{sp}for (int64_t i{loop.rank} = 0; i{loop.rank} < {size}; ++i{loop.rank}) {{")

    def _instr(self, ins: I, scope, ind):
        if ins.is_system() or not ins.ops:
            return
        sp = " " * ind
        nm = ir.OPNAMES[ins.opcode]
        if nm == "RANGE":
            ops = [self.name(ins.ops[0], scope), f"(uint64_t){self.index(ins.ops[0])}"]
        elif nm == "RANDOM":
            k = 16 * self.const_idx[id(ins)]
            ops = [self.name(ins.ops[0], scope),
                   f"bh_random123(*(const uint64_t*)(c + {k}), *(const uint64_t*)(c + {k + 8}), "
                   f"(uint64_t){self.index(ins.ops[0])})"]
        elif nm == "GATHER":
            src = ins.ops[1]
            ops = [self.name(ins.ops[0], scope),
                   f"a{self.param_idx[src.base.id]}[m[{self.view_off[src.key()]}] + (int64_t){self.name(ins.ops[2], scope)}]"]
        elif nm in ("SCATTER", "COND_SCATTER"):
            dst = ins.ops[0]
            ops = [f"a{self.param_idx[dst.base.id]}[m[{self.view_off[dst.key()]}] + (int64_t){self.name(ins.ops[2], scope)}]",
                   self.name(ins.ops[1], scope)]
            if nm == "COND_SCATTER":
                ops.append(self.name(ins.ops[3], scope))
        elif nm in ir.ACCUMULATES:
            ops = [self.name(ins.ops[0], scope), self.aref(ins.ops[0], prev_axis=ins.sweep_axis()),
                   self.name(ins.ops[1], scope)]
        elif nm in ir.REDUCTIONS:
            v = ins.ops[0]
            if ins.ops[1].ndim > 1 and scope.repl(v) is None and not scope.is_tmp(v.base.id):
                out = self.aref(v, ins.sweep_axis())
            else:
                out = self.name(v, scope)
            ops = [out, self.name(ins.ops[1], scope)]
        else:
            ops = [self.const(ins) if v is None else self.name(v, scope) for v in ins.ops]
        atomic = id(ins) in self.atomic
        if atomic:
            self.lines.append(f"{sp}#pragma omp atomic")
        elif id(ins) in self.critical:
            self.lines.append(f"{sp}#pragma omp critical")
        self.lines.append(sp + op_statement(ins, ops, atomic))

    def const_bytes(self) -> bytes:
        buf = bytearray(16 * max(len(self.consts), 1))
        for k, ins in enumerate(self.consts):
            value, t = ins.const
            if t == ir.R123:
                buf[16 * k:16 * k + 8] = int(value[0]).to_bytes(8, "little")
                buf[16 * k + 8:16 * k + 16] = int(value[1]).to_bytes(8, "little")
            else:
                b = np.array([value], dtype=ir.np_dtype(t)).tobytes()
                buf[16 * k:16 * k + len(b)] = b
        return bytes(buf)


class _Scope:
    def __init__(self, parent):
        self.parent, self.tmps, self.rep = parent, set(), {}

    def is_tmp(self, bid):
        return bid in self.tmps or (self.parent is not None and self.parent.is_tmp(bid))

    def repl(self, v: V) -> Optional[str]:
        k = _ignore_one_key(v)
        if k in self.rep:
            return self.rep[k]
        return self.parent.repl(v) if self.parent is not None else None


_compiled: dict = {}
_workdir = None


def _compile(source: str):
    global _workdir
    h = hashlib.sha1((" ".join(CFLAGS) + source).encode()).hexdigest()[:20]
    if h in _compiled:
        return _compiled[h]
    if _workdir is None:
        _workdir = tempfile.mkdtemp(prefix="bh_oracle_")
    src = os.path.join(_workdir, h + ".c")
    so = os.path.join(_workdir, h + ".so")
    with open(src, "w") as f:
        f.write(source)
    r = subprocess.run([CC] + CFLAGS + ["-I" + HERE, src, "-o", so, "-lm"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle: gcc failed:\n" + r.stderr + "\n" + source)
    lib = ctypes.CDLL(so)
    fn = lib.kernel
    fn.restype = None
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    _compiled[h] = fn
    return fn


def _compile_user(source: str):
    """A user kernel's source with its launcher, compiled like the oracle's own kernels; returns
    the launcher `_bh_launcher(void *data_list[])`."""
    global _workdir
    h = "u" + hashlib.sha1((" ".join(CFLAGS) + source).encode()).hexdigest()[:20]
    if h in _compiled:
        return _compiled[h]
    if _workdir is None:
        _workdir = tempfile.mkdtemp(prefix="bh_oracle_")
    src = os.path.join(_workdir, h + ".c")
    so = os.path.join(_workdir, h + ".so")
    with open(src, "w") as f:
        f.write(source)
    r = subprocess.run([CC] + CFLAGS + [src, "-o", so, "-lm"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("[UserKernel] compilation failed:\n" + r.stderr)
    fn = ctypes.CDLL(so)._bh_launcher
    fn.restype = None
    fn.argtypes = [ctypes.c_void_p]
    _compiled[h] = fn
    return fn


def set_threads(n: int) -> None:
    try:
        lib = ctypes.CDLL("libgomp.so.1")
        lib.omp_set_num_threads(int(n))
    except OSError:
        os.environ["OMP_NUM_THREADS"] = str(n)


class OracleExecutor:
    """Runs flushes on the host cores with the restated ve/openmp engine."""

    def __init__(self, threads: Optional[int] = None, fuser=("greedy", "collapse_redundant_axes")):
        self.store: dict = {}
        self.fuser = tuple(fuser)
        self.threads = threads or os.cpu_count() or 1
        set_threads(self.threads)
        self.exec_seconds = 0.0
        self.kernels_run = 0
        self._slide_state: dict = {}

    # executor interface ------------------------------------------------------------------
    def register(self, base: ir.Base) -> None:
        base.handle = -1 - base.id  # any non-zero value: the oracle keys storage by base id

    def release(self, base: ir.Base) -> None:
        self.store.pop(base.id, None)

    def set_data(self, base: ir.Base, data) -> None:
        self.store[base.id] = np.ascontiguousarray(np.asarray(data, dtype=base.dtype).reshape(-1)).copy()

    def get_data(self, base: ir.Base) -> np.ndarray:
        a = self.store.get(base.id)
        return np.zeros(base.nelem, base.dtype) if a is None else a.copy()

    def peek(self, base: ir.Base) -> np.ndarray:
        return self.get_data(base)

    def message(self, msg: str) -> str:
        return ""

    def _array(self, base: ir.Base) -> np.ndarray:
        a = self.store.get(base.id)
        if a is None:
            a = np.zeros(max(base.nelem, 1), dtype=base.dtype)
            self.store[base.id] = a
        return a

    def user_kernel(self, kernel: str, bases, compile_cmd: str, tag: str, param: str) -> str:
        """ComponentImpl::userKernel of ve/openmp (ve/openmp/engine_openmp.cpp:484-530): the
        source plus a launcher that casts each operand's data to its C type and calls
        `execute(a0, a1, ...)`, compiled and run on the host. Only tag "openmp"; the oracle's own
        compiler flags replace `compile_cmd`. Returns "" or the error text."""
        if tag != "openmp":
            return f'[UserKernel] the oracle runs tag "openmp" only, not "{tag}"'
        lines = [kernel, "void _bh_launcher(void *data_list[]) {"]
        for i, b in enumerate(bases):
            lines.append(f"    {ctype(b.dtype)} *a{i} = data_list[{i}];")
        lines.append("    execute(" + ", ".join(f"a{i}" for i in range(len(bases))) + ");")
        lines.append("}")
        try:
            fn = _compile_user("\n".join(lines) + "\n")
        except RuntimeError as e:
            return str(e)
        arrays = [self._array(b) for b in bases]
        ptrs = (ctypes.c_void_p * max(len(arrays), 1))(*[a.ctypes.data for a in arrays])
        fn(ptrs)
        return ""

    # execution ---------------------------------------------------------------------------
    def execute(self, flush: ir.Flush) -> None:
        instrs = list(flush.instrs)
        for rep in range(flush.nrepeats):
            self._execute_once(instrs)
            if flush.condition is not None:
                if not bool(self._array(flush.condition)[0]):
                    break
            instrs = self._slide(instrs)

    def _convert(self, instrs):
        out = []
        for ins in instrs:
            ops = [None if v is None else V(v.base, v.start, list(v.shape), list(v.stride)) for v in ins.operands]
            const = None
            if ins.constant is not None:
                const = (ins.constant.value, ins.constant.dtype)
            out.append(I(ins.opcode, ops, const))
        return out

    def _execute_once(self, flush_instrs):
        instrs = self._convert(flush_instrs)
        instrs, frees = jitk.remove_non_computed(instrs)
        for b in frees:
            self.store.pop(b.id, None)
        constructed = set(self.store)
        for ins in instrs:
            ins.constructor = False
            for k, v in enumerate(ins.ops):
                if v is None:
                    continue
                if k == 0 and v.base.id not in constructed:
                    ins.constructor = True
                constructed.add(v.base.id)
        for kernel in jitk.kernel_list(instrs, self.fuser):
            if not kernel.is_system_only():
                self._run(kernel)
            for bid, b in kernel.all_frees().items():
                self.store.pop(bid, None)

    def _run(self, kernel: Loop):
        k = _Kernel(kernel)
        fn = _compile(k.source)
        arrays = [self._array(b) for b in k.params]
        ptrs = (ctypes.c_void_p * max(len(arrays), 1))(*[a.ctypes.data for a in arrays])
        meta = np.array(k.meta if k.meta else [0], dtype=np.int64)
        consts = k.const_bytes()
        t0 = time.perf_counter()
        fn(ptrs, meta.ctypes.data, consts)
        self.exec_seconds += time.perf_counter() - t0
        self.kernels_run += 1

    def _slide(self, instrs):
        """Slide views between repeats (include/bohrium/jitk/engines/dyn_view.hpp:21-67)."""
        out = []
        for idx, ins in enumerate(instrs):
            if not ins.slides:
                out.append(ins)
                continue
            ops = list(ins.operands)
            for o, (dims, resets) in ins.slides.items():
                v = ops[o]
                st = self._slide_state.setdefault((id(ins), o), {"it": 0, "since": {d: 0 for d in resets}})
                start, shape = v.start, list(v.shape)
                for d in dims:
                    if d.step_delay == 1 or st["it"] % d.step_delay == d.step_delay - 1:
                        if d.stride:
                            change = d.offset_change * d.stride
                            max_rel = d.stride * d.shape
                            rel = start % (d.stride * d.shape) + change
                            if rel < 0:
                                change += max_rel
                            elif rel >= max_rel:
                                change -= max_rel
                            start += change
                            if d.rank in resets:
                                st["since"][d.rank] += change
                                reset_at = resets[d.rank]
                                if st["it"] > 0 and (st["it"] // d.step_delay) % reset_at == reset_at - 1:
                                    start -= st["since"][d.rank]
                                    st["since"][d.rank] = 0
                                    shape[d.rank] -= reset_at * d.shape_change
                        shape[d.rank] = max(shape[d.rank] + d.shape_change, 0)
                st["it"] += 1
                ops[o] = ir.View(v.base, start, tuple(shape), v.stride)
            new = ir.Instr(ins.opcode, ops, ins.constant, ins.slides)
            self._slide_state[(id(new), 0)] = self._slide_state.get((id(ins), 0), {"it": 0, "since": {}})
            for o in ins.slides:
                self._slide_state[(id(new), o)] = self._slide_state.pop((id(ins), o))
            out.append(new)
        return out
