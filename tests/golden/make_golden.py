"""Generate the golden vectors under tests/golden/ (run in the build container, where the
reference tree exists; the vectors are committed so the tests never need the reference).

random123.json: BH_RANDOM outputs computed by the reference's own vendored Random123
(thirdparty/Random123-1.09/include/Random123/philox.h, built by `make -C oracle` into
oracle/_ref/libref_random123.so) for several (start, key) pairs, including counters that carry
into the high 32-bit word and keys whose high 32 bits must be ignored.

integer_semantics.json: NumPy results of floor division, remainder and shifts on signed and
unsigned integers -- NumPy is the witness of the reference's test-suite (test/python/run.py:42-59)
and the reference's generated code restates NumPy's rules (core/jitk/instruction.cpp:146-165,
411-432).
"""
import ctypes
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def random123_vectors():
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_random123.so"))
    lib.ref_random123_fill.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p]
    cases = []
    for start, key, n in [(0, 42, 64), (0, 0, 16), (1, 1, 16), (2**32 - 8, 7, 16), (2**40 + 3, 2**33 + 5, 16),
                          (123456789, 0xFFFFFFFF, 16), (2**64 - 4, 99, 8)]:
        out = np.zeros(n, dtype=np.uint64)
        lib.ref_random123_fill(start, key, n, out.ctypes.data)
        cases.append({"start": start, "key": key, "values": [int(v) for v in out]})
    return {"source": "reference thirdparty/Random123-1.09 philox2x32_R(10 rounds) via oracle/_ref", "cases": cases}


def integer_vectors():
    rng = np.random.default_rng(7)
    out = {}
    for dt in ["int8", "int16", "int32", "int64", "uint8", "uint32", "uint64"]:
        t = np.dtype(dt)
        info = np.iinfo(t)
        lo, hi = max(info.min, -1000), min(info.max, 1000)
        a = rng.integers(lo, hi + 1, 64).astype(t)
        b = rng.integers(lo, hi + 1, 64).astype(t)
        b[b == 0] = 3
        if t.kind == "i":
            b[b == -1] = 5
        out[dt] = {"a": a.tolist(), "b": b.tolist(), "floor_divide": (a // b).tolist(),
                   "remainder": np.remainder(a, b).tolist()}
    return {"source": "numpy " + np.__version__, "cases": out}


if __name__ == "__main__":
    with open(os.path.join(HERE, "random123.json"), "w") as f:
        json.dump(random123_vectors(), f, indent=1)
    with open(os.path.join(HERE, "integer_semantics.json"), "w") as f:
        json.dump(integer_vectors(), f)
    print("written")
