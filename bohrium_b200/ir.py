"""Python model of Bohrium bytecode (BhIR) and its flat int64 wire encoding.

The model mirrors the reference's C++ types (include/bohrium/bh_instruction.hpp, bh_view.hpp,
bh_base.hpp, bh_ir.hpp): a flush is a list of instructions whose operands are views (base, start,
shape, stride, in elements) or the instruction's constant. The encoding is the one read by
bhb_ir_create() in include/bh_b200.h.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

# Opcode ids: the wire values of the Bohrium bytecode (include/bohrium/bh_opcode.h).
OPCODES = {
    "ADD": 1, "SUBTRACT": 2, "MULTIPLY": 3, "DIVIDE": 4, "POWER": 5, "ABSOLUTE": 6, "GREATER": 7,
    "GREATER_EQUAL": 8, "LESS": 9, "LESS_EQUAL": 10, "EQUAL": 11, "NOT_EQUAL": 12, "LOGICAL_AND": 13,
    "LOGICAL_OR": 14, "LOGICAL_XOR": 15, "LOGICAL_NOT": 16, "MAXIMUM": 17, "MINIMUM": 18, "BITWISE_AND": 19,
    "BITWISE_OR": 20, "BITWISE_XOR": 21, "INVERT": 22, "LEFT_SHIFT": 23, "RIGHT_SHIFT": 24, "COS": 25, "SIN": 26,
    "TAN": 27, "COSH": 28, "SINH": 29, "TANH": 30, "ARCSIN": 31, "ARCCOS": 32, "ARCTAN": 33, "ARCSINH": 34,
    "ARCCOSH": 35, "ARCTANH": 36, "ARCTAN2": 37, "EXP": 38, "EXP2": 39, "EXPM1": 40, "LOG": 41, "LOG2": 42,
    "LOG10": 43, "LOG1P": 44, "SQRT": 45, "CEIL": 46, "TRUNC": 47, "FLOOR": 48, "RINT": 49, "MOD": 50,
    "ISNAN": 51, "ISINF": 52, "IDENTITY": 53, "FREE": 55, "NONE": 57, "TALLY": 58, "ADD_REDUCE": 59,
    "MULTIPLY_REDUCE": 60, "MINIMUM_REDUCE": 61, "MAXIMUM_REDUCE": 62, "LOGICAL_AND_REDUCE": 63,
    "BITWISE_AND_REDUCE": 64, "LOGICAL_OR_REDUCE": 65, "BITWISE_OR_REDUCE": 66, "LOGICAL_XOR_REDUCE": 67,
    "BITWISE_XOR_REDUCE": 68, "RANDOM": 71, "RANGE": 72, "REAL": 73, "IMAG": 74, "ADD_ACCUMULATE": 75,
    "MULTIPLY_ACCUMULATE": 76, "SIGN": 77, "GATHER": 79, "SCATTER": 80, "REMAINDER": 81, "COND_SCATTER": 82,
    "ISFINITE": 83, "CONJ": 84,
}
OPNAMES = {v: k for k, v in OPCODES.items()}
MAX_OPCODE_ID = 84
NOP = {k: 3 for k in OPCODES}
NOP.update({k: 2 for k in [
    "ABSOLUTE", "LOGICAL_NOT", "INVERT", "COS", "SIN", "TAN", "COSH", "SINH", "TANH", "ARCSIN", "ARCCOS", "ARCTAN",
    "ARCSINH", "ARCCOSH", "ARCTANH", "EXP", "EXP2", "EXPM1", "LOG", "LOG2", "LOG10", "LOG1P", "SQRT", "CEIL", "TRUNC",
    "FLOOR", "RINT", "ISNAN", "ISINF", "IDENTITY", "RANDOM", "REAL", "IMAG", "SIGN", "ISFINITE", "CONJ"]})
NOP.update({"FREE": 1, "NONE": 0, "TALLY": 0, "RANGE": 1, "COND_SCATTER": 4})
REDUCTIONS = {k for k in OPCODES if k.endswith("_REDUCE")}
ACCUMULATES = {"ADD_ACCUMULATE", "MULTIPLY_ACCUMULATE"}

# bh_type enum (include/bohrium/bh_type.hpp)
BOOL, INT8, INT16, INT32, INT64, UINT8, UINT16, UINT32, UINT64, FLOAT32, FLOAT64, COMPLEX64, COMPLEX128, R123 = range(14)
_NP2BH = {np.dtype(np.bool_): BOOL, np.dtype(np.int8): INT8, np.dtype(np.int16): INT16, np.dtype(np.int32): INT32,
          np.dtype(np.int64): INT64, np.dtype(np.uint8): UINT8, np.dtype(np.uint16): UINT16,
          np.dtype(np.uint32): UINT32, np.dtype(np.uint64): UINT64, np.dtype(np.float32): FLOAT32,
          np.dtype(np.float64): FLOAT64, np.dtype(np.complex64): COMPLEX64, np.dtype(np.complex128): COMPLEX128}
_BH2NP = {v: k for k, v in _NP2BH.items()}


def bh_type(dtype) -> int:
    return _NP2BH[np.dtype(dtype)]


def np_dtype(t: int) -> np.dtype:
    return _BH2NP[t]


_base_ids = itertools.count()


class Base:
    """A base array: element type and count. `handle` is set by the executor that owns it."""

    def __init__(self, dtype, nelem: int):
        self.dtype = np.dtype(dtype)
        self.nelem = int(nelem)
        self.id = next(_base_ids)
        self.handle = 0

    @property
    def nbytes(self) -> int:
        return self.nelem * self.dtype.itemsize

    def __repr__(self):
        return f"a{self.id}<{self.dtype},{self.nelem}>"


@dataclass(frozen=True)
class View:
    base: Base
    start: int
    shape: tuple
    stride: tuple

    @property
    def ndim(self):
        return len(self.shape)

    @staticmethod
    def whole(base: Base) -> "View":
        return View(base, 0, (base.nelem,), (1,))


@dataclass
class Constant:
    value: object
    dtype: int  # bh_type

    def words(self) -> tuple:
        raw = bytearray(16)
        if self.dtype == R123:
            start, key = self.value
            raw[0:8] = int(start).to_bytes(8, "little", signed=False)
            raw[8:16] = int(key).to_bytes(8, "little", signed=False)
        else:
            arr = np.array([self.value], dtype=np_dtype(self.dtype))
            b = arr.tobytes()
            raw[: len(b)] = b
        w = np.frombuffer(bytes(raw), dtype=np.int64)
        return int(w[0]), int(w[1])


@dataclass
class Slide:
    """One sliding dimension of an operand (bh_slide_dim)."""
    rank: int
    offset_change: int
    shape_change: int
    stride: int
    shape: int
    step_delay: int = 1


@dataclass
class Instr:
    opcode: int
    operands: list  # View or None (the constant)
    constant: Optional[Constant] = None
    slides: dict = field(default_factory=dict)  # operand index -> (list[Slide], {dim: reset_max})

    @property
    def name(self):
        return OPNAMES.get(self.opcode, f"EXT{self.opcode}")


@dataclass
class Flush:
    instrs: list
    syncs: list = field(default_factory=list)  # Base
    nrepeats: int = 1
    condition: Optional[Base] = None
    # Bases that the flush's BH_FREEs free: their handles must outlive every execution of the
    # flush (a compiled flush keeps them until it is destroyed).
    released: list = field(default_factory=list)


def encode(instrs: Sequence[Instr]) -> np.ndarray:
    """Encode instructions into the int64 words read by bhb_ir_create()."""
    words: list = []
    for ins in instrs:
        if ins.constant is not None:
            c0, c1 = ins.constant.words()
            words += [ins.opcode, len(ins.operands), ins.constant.dtype, c0, c1]
        else:
            words += [ins.opcode, len(ins.operands), -1, 0, 0]
        for op in ins.operands:
            if op is None:
                words.append(0)
            else:
                if op.base.handle == 0:
                    raise RuntimeError(f"base {op.base} has no native handle")
                words += [op.base.handle, op.start, len(op.shape)]
                words += list(op.shape)
                words += list(op.stride)
    return np.array(words, dtype=np.int64)


def encode_slides(instrs: Sequence[Instr]) -> np.ndarray:
    words: list = []
    for i, ins in enumerate(instrs):
        for o, (dims, resets) in ins.slides.items():
            words += [i, o, len(dims)]
            for d in dims:
                words += [d.rank, d.offset_change, d.shape_change, d.stride, d.shape, d.step_delay]
            words.append(len(resets))
            for dim, reset_max in resets.items():
                words += [dim, reset_max]
    return np.array(words, dtype=np.int64)


def pprint(instrs: Sequence[Instr]) -> str:
    lines = []
    for ins in instrs:
        ops = []
        for op in ins.operands:
            if op is None:
                ops.append(f"C({ins.constant.value})")
            else:
                ops.append(f"{op.base}[{op.start}:{op.shape}:{op.stride}]")
        lines.append(f"{ins.name} " + " ".join(ops))
    return "\n".join(lines)
