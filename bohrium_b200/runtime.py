"""Runtime: owns a component stack and the list of pending instructions.

Mirrors bhxx::Runtime (bridge/cxx/src/Runtime.cpp:28-140 of the reference): instructions are
enqueued, `flush()` hands them to the stack as one BhIR, `sync` makes a base's host copy valid.
The stack is reached through an *executor*: `NativeExecutor` drives the native libraries through
the C ABI of include/bh_b200.h. Other executors (e.g. the CPU oracle used by the tests) implement
the same five methods.
"""
from __future__ import annotations

import ctypes
import os
import weakref
from typing import Optional

import numpy as np

from . import ir

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(PKG, "lib")
DEFAULT_CONFIG = os.path.join(PKG, "config.ini")

_lib = None


def load_library():
    """Load libbh_core.so (the C bridge). Raises if the native build is missing."""
    global _lib
    if _lib is not None:
        return _lib
    path = os.path.join(LIB_DIR, "libbh_core.so")
    if not os.path.exists(path):
        raise RuntimeError(f"native library missing: {path} (run `python -m bohrium_b200.build`)")
    lib = ctypes.CDLL(path, mode=ctypes.RTLD_GLOBAL)
    P, I64, U64, I = ctypes.c_void_p, ctypes.c_int64, ctypes.c_uint64, ctypes.c_int
    sig = {
        "bhb_last_error": (ctypes.c_char_p, []),
        "bhb_runtime_create": (P, [ctypes.c_char_p, ctypes.c_char_p]),
        "bhb_runtime_destroy": (None, [P]),
        "bhb_base_create": (P, [I, I64]),
        "bhb_base_destroy": (None, [P]),
        "bhb_base_dtype": (I, [P]),
        "bhb_base_nelem": (I64, [P]),
        "bhb_base_data": (P, [P]),
        "bhb_data_get": (P, [P, P, I, I, I]),
        "bhb_data_set": (I, [P, P, I, P]),
        "bhb_host_alloc": (P, [P, I64]),
        "bhb_data_copy_in": (I, [P, P, P, I64]),
        "bhb_ir_create": (P, [P, I64, P, I64, U64, P, P, I64]),
        "bhb_ir_destroy": (None, [P]),
        "bhb_ir_execute": (I, [P, P]),
        "bhb_execute": (I, [P, P, I64, P, I64, U64, P, P, I64]),
        "bhb_message": (ctypes.c_char_p, [P, ctypes.c_char_p]),
        "bhb_extmethod": (I, [P, ctypes.c_char_p, I64]),
        "bhb_get_device_context": (P, [P]),
        "bhb_set_device_context": (I, [P, P]),
        "bhb_last_execute_ms": (ctypes.c_double, [P]),
        "bhb_user_kernel": (ctypes.c_char_p, [P, ctypes.c_char_p, I64, P, ctypes.c_char_p, ctypes.c_char_p,
                                              ctypes.c_char_p]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _err(lib) -> str:
    return (lib.bhb_last_error() or b"").decode(errors="replace")


class NativeExecutor:
    """Executes flushes on a native component stack (by default the `cuda` stack)."""

    def __init__(self, config: Optional[str] = None, stack: Optional[str] = None):
        self.lib = load_library()
        cfg = config or os.environ.get("BH_CONFIG") or DEFAULT_CONFIG
        self.rt = self.lib.bhb_runtime_create(cfg.encode(), (stack or os.environ.get("BH_STACK", "")).encode())
        if not self.rt:
            raise RuntimeError("bhb_runtime_create: " + _err(self.lib))
        self._pinned = {}

    def close(self):
        if self.rt:
            self.lib.bhb_runtime_destroy(self.rt)
            self.rt = None

    # -- bases -----------------------------------------------------------------------------
    def register(self, base: ir.Base) -> None:
        h = self.lib.bhb_base_create(ir.bh_type(base.dtype), base.nelem)
        if not h:
            raise RuntimeError("bhb_base_create: " + _err(self.lib))
        base.handle = h

    def release(self, base: ir.Base) -> None:
        if base.handle:
            self.lib.bhb_base_destroy(base.handle)
            base.handle = 0

    def set_data(self, base: ir.Base, data: np.ndarray) -> None:
        data = np.ascontiguousarray(data, dtype=base.dtype).reshape(-1)
        if data.size != base.nelem:
            raise ValueError("set_data: size mismatch")
        if self.lib.bhb_data_copy_in(self.rt, base.handle, data.ctypes.data, data.nbytes) != 0:
            raise RuntimeError("bhb_data_copy_in: " + _err(self.lib))

    def set_pinned(self, base: ir.Base, data: np.ndarray) -> np.ndarray:
        """Give `base` page-locked host storage filled with `data`; returns a numpy view of it."""
        p = self.lib.bhb_host_alloc(self.rt, max(base.nbytes, 1))
        if not p:
            raise RuntimeError("bhb_host_alloc: " + _err(self.lib))
        arr = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_uint8)), shape=(base.nbytes,))
        view = arr.view(base.dtype)
        view[:] = np.asarray(data, dtype=base.dtype).reshape(-1)
        if self.lib.bhb_data_set(self.rt, base.handle, 1, p) != 0:
            raise RuntimeError("bhb_data_set: " + _err(self.lib))
        return view

    def get_data(self, base: ir.Base) -> np.ndarray:
        """Host copy of the base (the stack releases its device copy, as getMemoryPointer does)."""
        p = self.lib.bhb_data_get(self.rt, base.handle, 1, 1, 0)
        if not p and base.nbytes:
            raise RuntimeError("bhb_data_get: " + _err(self.lib))
        if base.nbytes == 0:
            return np.zeros(0, dtype=base.dtype)
        buf = (ctypes.c_uint8 * base.nbytes).from_address(p)
        return np.frombuffer(buf, dtype=base.dtype).copy()

    def peek(self, base: ir.Base) -> np.ndarray:
        """Host copy after a sync that keeps the device copy valid (lazy host sync)."""
        self.execute(ir.Flush([], syncs=[base]))
        p = self.lib.bhb_base_data(base.handle)
        if base.nbytes == 0:
            return np.zeros(0, dtype=base.dtype)
        buf = (ctypes.c_uint8 * base.nbytes).from_address(p)
        return np.frombuffer(buf, dtype=base.dtype).copy()

    # -- execution -------------------------------------------------------------------------
    def compile(self, flush: ir.Flush):
        """Decode a flush once into a re-executable native BhIR handle."""
        words = ir.encode(flush.instrs)
        slides = ir.encode_slides(flush.instrs)
        syncs = (ctypes.c_void_p * max(len(flush.syncs), 1))(*[b.handle for b in flush.syncs])
        cond = flush.condition.handle if flush.condition is not None else None
        h = self.lib.bhb_ir_create(words.ctypes.data, len(words), syncs, len(flush.syncs), flush.nrepeats, cond,
                                   slides.ctypes.data, len(slides))
        if not h:
            raise RuntimeError("bhb_ir_create: " + _err(self.lib))
        return NativeIR(self, h, (words, slides), flush.released)

    def execute(self, flush: ir.Flush) -> None:
        words = ir.encode(flush.instrs)
        slides = ir.encode_slides(flush.instrs)
        syncs = (ctypes.c_void_p * max(len(flush.syncs), 1))(*[b.handle for b in flush.syncs])
        cond = flush.condition.handle if flush.condition is not None else None
        r = self.lib.bhb_execute(self.rt, words.ctypes.data, len(words), syncs, len(flush.syncs), flush.nrepeats,
                                 cond, slides.ctypes.data, len(slides))
        if r != 0:
            raise RuntimeError("bhb_execute: " + _err(self.lib))

    def message(self, msg: str) -> str:
        r = self.lib.bhb_message(self.rt, msg.encode())
        if r is None:
            raise RuntimeError("bhb_message: " + _err(self.lib))
        return r.decode()

    def extmethod(self, name: str, opcode: int) -> None:
        if self.lib.bhb_extmethod(self.rt, name.encode(), opcode) != 0:
            raise RuntimeError("bhb_extmethod: " + _err(self.lib))

    def last_execute_ms(self) -> float:
        return float(self.lib.bhb_last_execute_ms(self.rt))

    def user_kernel(self, kernel: str, bases, compile_cmd: str, tag: str, param: str) -> str:
        """ComponentImpl::userKernel through bhb_user_kernel: the component's message ("" on
        success, else the error text)."""
        handles = (ctypes.c_void_p * max(len(bases), 1))(*[b.handle for b in bases])
        r = self.lib.bhb_user_kernel(self.rt, kernel.encode(), len(bases), handles, compile_cmd.encode(),
                                     tag.encode(), param.encode())
        if r is None:
            raise RuntimeError("bhb_user_kernel: " + _err(self.lib))
        return r.decode()


class NativeIR:
    """A decoded flush that can be executed repeatedly (bhb_ir_execute)."""

    def __init__(self, ex: NativeExecutor, handle, keep, released=()):
        self.ex, self.handle, self._keep = ex, handle, keep
        self._released = list(released)  # bases freed by the flush: released with the handle

    def execute(self):
        if self.ex.lib.bhb_ir_execute(self.ex.rt, self.handle) != 0:
            raise RuntimeError("bhb_ir_execute: " + _err(self.ex.lib))

    def __del__(self):
        try:
            if self.handle:
                self.ex.lib.bhb_ir_destroy(self.handle)
                self.handle = None
            for b in self._released:
                self.ex.release(b)
        except Exception:
            pass


class Runtime:
    """Instruction queue in front of an executor (bhxx::Runtime)."""

    def __init__(self, executor=None, auto_flush: int = 0):
        self.ex = executor if executor is not None else NativeExecutor()
        self.instrs: list = []
        self.auto_flush = auto_flush  # flush when this many instructions are queued (0: never)
        self._released: list = []

    # -- bases -----------------------------------------------------------------------------
    def new_base(self, dtype, nelem: int) -> ir.Base:
        b = ir.Base(dtype, nelem)
        self.ex.register(b)
        weakref.finalize(b, lambda: None)
        return b

    def enqueue(self, ins: ir.Instr) -> None:
        self.instrs.append(ins)
        if self.auto_flush and len(self.instrs) >= self.auto_flush:
            self.flush()

    def free(self, base: ir.Base) -> None:
        """Enqueue BH_FREE of `base`; its native handle is released after the flush."""
        self.enqueue(ir.Instr(ir.OPCODES["FREE"], [ir.View.whole(base)]))
        self._released.append(base)

    def flush(self, syncs=(), nrepeats: int = 1, condition: Optional[ir.Base] = None) -> None:
        instrs, self.instrs = self.instrs, []
        released, self._released = self._released, []
        self.ex.execute(ir.Flush(instrs, list(syncs), nrepeats, condition))
        for b in released:
            self.ex.release(b)

    def take(self) -> ir.Flush:
        """Remove and return the pending instructions as a Flush (not executed). The bases its
        BH_FREEs free go with it (Flush.released): a compiled flush releases them when it is
        destroyed, so a later flush of this runtime cannot release bases it still uses."""
        instrs, self.instrs = self.instrs, []
        released, self._released = self._released, []
        return ir.Flush(instrs, released=released)
