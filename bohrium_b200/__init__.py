"""B200-native Bohrium vector engine.

The native stack (bohrium_b200/lib/*.so) is a drop-in for the reference's `cuda` vector engine
behind its component interface; this package adds a Python front end that emits Bohrium bytecode
(`array`), a runtime that hands flushes to the stack through the C ABI (`runtime`), and a
device-free inspection of the engine's lowering (`dry_run`).
"""
from . import ir
from .runtime import NativeExecutor, Runtime, load_library
from .array import (BhArray, empty, full, zeros, ones, array, arange, random123, random_sample, binary, unary,
                    reduce, accumulate, gather, scatter, sqrt, exp, log, sin, cos, tanh, absolute, floor, sign,
                    maximum, minimum, where, true_divide, matmul, extmethod_opcode, tan, sinh, cosh, log10, real,
                    imag, conj, user_kernel, make_behaving, is_behaving)
from .inspect import DryRunExecutor, dry_run

__all__ = ["ir", "NativeExecutor", "Runtime", "load_library", "BhArray", "empty", "full", "zeros", "ones", "array",
           "arange", "random123", "random_sample", "binary", "unary", "reduce", "accumulate", "gather", "scatter",
           "sqrt", "exp", "log", "sin", "cos", "tanh", "absolute", "floor", "sign", "maximum", "minimum", "where",
           "true_divide", "matmul", "extmethod_opcode", "tan", "sinh", "cosh", "log10", "real", "imag", "conj",
           "user_kernel", "make_behaving", "is_behaving", "DryRunExecutor", "dry_run"]
