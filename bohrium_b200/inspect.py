"""Device-free inspection of the engine: fusion plan, launch schedules and NVRTC compilation.

`dry_run(flush)` calls bh_ve_cuda_dry_run() of libbh_ve_cuda.so, which runs the same fuser and
code generator as the engine and compiles every generated kernel for sm_100a with NVRTC, without
touching a GPU. `DryRunExecutor` is an executor that records flushes instead of running them.
"""
from __future__ import annotations

import ctypes
import json
import os

import numpy as np

from . import ir
from .runtime import LIB_DIR, load_library

_ve = None


def _ve_lib():
    global _ve
    if _ve is None:
        load_library()
        path = os.path.join(LIB_DIR, "libbh_ve_cuda.so")
        if not os.path.exists(path):
            raise RuntimeError(f"native library missing: {path}")
        _ve = ctypes.CDLL(path)
        _ve.bh_ve_cuda_dry_run.restype = ctypes.c_char_p
        _ve.bh_ve_cuda_dry_run.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p]
    return _ve


def dry_run(flush: ir.Flush, compile: bool = True, fuser_list: str | None = None) -> dict:
    lib = load_library()
    words = ir.encode(flush.instrs)
    slides = ir.encode_slides(flush.instrs)
    syncs = (ctypes.c_void_p * max(len(flush.syncs), 1))(*[b.handle for b in flush.syncs])
    h = lib.bhb_ir_create(words.ctypes.data, len(words), syncs, len(flush.syncs), flush.nrepeats, None,
                          slides.ctypes.data, len(slides))
    if not h:
        raise RuntimeError("bhb_ir_create: " + lib.bhb_last_error().decode())
    try:
        r = _ve_lib().bh_ve_cuda_dry_run(h, 1 if compile else 0, fuser_list.encode() if fuser_list else None)
        if r is None:
            raise RuntimeError("dry run: " + lib.bhb_last_error().decode())
        return json.loads(r.decode())
    finally:
        lib.bhb_ir_destroy(h)


class DryRunExecutor:
    """Executor that keeps base handles (no device) and records the flushes it is given."""

    def __init__(self):
        self.lib = load_library()
        self.flushes: list = []
        self.data: dict = {}

    def register(self, base: ir.Base) -> None:
        base.handle = self.lib.bhb_base_create(ir.bh_type(base.dtype), base.nelem)

    def release(self, base: ir.Base) -> None:
        pass

    def set_data(self, base: ir.Base, data) -> None:
        self.data[base.id] = np.asarray(data, dtype=base.dtype).reshape(-1).copy()

    def get_data(self, base: ir.Base):
        raise RuntimeError("DryRunExecutor has no device")

    def execute(self, flush: ir.Flush) -> None:
        self.flushes.append(flush)

    def message(self, msg: str) -> str:
        return ""


def filter_text(flush: ir.Flush, filters=("bcexp", "bccon")) -> tuple[list, str]:
    """Apply the bytecode filters of the filter components to `flush` (decoded natively) and
    return (rewrites per filter, the text listing of the result, see bhb_ir_text)."""
    lib = load_library()
    lib.bhb_ir_filter.restype = ctypes.c_int
    lib.bhb_ir_filter.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
    lib.bhb_ir_text.restype = ctypes.c_char_p
    lib.bhb_ir_text.argtypes = [ctypes.c_void_p]
    words = ir.encode(flush.instrs)
    slides = ir.encode_slides(flush.instrs)
    syncs = (ctypes.c_void_p * max(len(flush.syncs), 1))(*[b.handle for b in flush.syncs])
    h = lib.bhb_ir_create(words.ctypes.data, len(words), syncs, len(flush.syncs), flush.nrepeats, None,
                          slides.ctypes.data, len(slides))
    if not h:
        raise RuntimeError("bhb_ir_create: " + lib.bhb_last_error().decode())
    try:
        counts = []
        for f in filters:
            n = lib.bhb_ir_filter(h, f.encode())
            if n < 0:
                raise RuntimeError("bhb_ir_filter: " + lib.bhb_last_error().decode())
            counts.append(n)
        return counts, lib.bhb_ir_text(h).decode()
    finally:
        lib.bhb_ir_destroy(h)
