"""The bytecode filters of the bcexp and bccon components (filter/bcexp/expander.cpp:42-87,
filter/bccon/contracter.cpp:46-52 of the reference), applied to decoded BhIRs on the CPU: which
instructions they rewrite, and into what."""
import numpy as np

import bohrium_b200 as bh
from bohrium_b200 import ir
from bohrium_b200.inspect import filter_text

OP = ir.OPCODES


def _flush(prog):
    ex = bh.DryRunExecutor()
    rt = bh.Runtime(ex)
    outs = prog(rt)
    flush = rt.take()
    flush.syncs = [o.base for o in outs]
    return flush


def _ops(text):
    return [int(line.split()[0]) for line in text.splitlines() if line.strip()]


def test_powk_unfolds_integer_powers():
    for k, want in [(0, [OP["IDENTITY"]]), (1, [OP["IDENTITY"]]), (2, [OP["MULTIPLY"]]),
                    (3, [OP["MULTIPLY"]] * 2), (8, [OP["MULTIPLY"]] * 3), (11, [OP["MULTIPLY"]] * 6)]:
        def prog(rt, k=k):
            x = bh.empty(rt, (100,), np.int64)
            return [bh.binary("POWER", x, np.int64(k))]
        counts, text = filter_text(_flush(prog), ("bcexp",))
        assert counts == [1], (k, text)
        ops = [o for o in _ops(text) if o != OP["FREE"]]
        assert ops == want, (k, text)


def test_powk_keeps_float_exponents_and_in_place_powers():
    def prog(rt):
        x = bh.empty(rt, (100,), np.float64)
        return [bh.binary("POWER", x, np.float64(2.5))]
    counts, text = filter_text(_flush(prog), ("bcexp",))
    assert counts == [0] and OP["POWER"] in _ops(text)


def test_sign_expansion():
    def prog(rt):
        x = bh.empty(rt, (10,), np.float32)
        return [bh.sign(x)]
    counts, text = filter_text(_flush(prog), ("bcexp+sign",))
    assert counts == [1]
    ops = _ops(text)
    assert OP["SIGN"] not in ops and ops.count(OP["FREE"]) >= 4
    assert OP["GREATER"] in ops and OP["LESS"] in ops and OP["SUBTRACT"] in ops


def test_stupidmath_only_rewrites_identities():
    def prog(rt):
        x = bh.empty(rt, (10,), np.int32)
        return [x * np.int32(1), x + np.int32(0), x - np.int32(0), np.int32(0) - x, np.int32(1) // x]
    counts, text = filter_text(_flush(prog), ("bccon",))
    ops = _ops(text)
    assert ops.count(OP["IDENTITY"]) == 3, text
    assert OP["SUBTRACT"] in ops  # 0 - x is not x


def test_collect_folds_integer_constant_chains():
    def prog(rt):
        x = bh.empty(rt, (10,), np.int64)
        return [((x + np.int64(3)) - np.int64(5)) + np.int64(7)]
    counts, text = filter_text(_flush(prog), ("bccon",))
    lines = [l for l in text.splitlines() if int(l.split()[0]) not in (OP["FREE"],)]
    assert len(lines) == 1 and lines[0].startswith(str(OP["ADD"])) and lines[0].endswith("= 5"), text


def test_collect_leaves_float_chains_alone():
    def prog(rt):
        x = bh.empty(rt, (10,), np.float64)
        return [(x + 3.0) + 7.0]
    counts, text = filter_text(_flush(prog), ("bccon",))
    assert counts == [0]


def test_muladd_combines_integer_products():
    def prog(rt):
        x = bh.empty(rt, (10,), np.int32)
        return [x * np.int32(2) + x * np.int32(3)]
    counts, text = filter_text(_flush(prog), ("bccon",))
    lines = [l for l in text.splitlines() if int(l.split()[0]) != OP["FREE"]]
    assert len(lines) == 1 and lines[0].startswith(str(OP["MULTIPLY"])) and lines[0].endswith("= 5"), text


def test_reduce1d_splits_long_1d_reductions():
    """expand_reduce1d.cpp:31-80: with the GPU stack's thread limit 32000, a 1-D reduction of
    2^20 elements becomes a [32, 32768] axis-0 reduction into a temporary plus the reduction of
    the temporary (fold = largest divisor of n up to n/32000); short or prime-length ones stay."""
    def prog(rt, n=1 << 20, name="ADD_REDUCE"):
        x = bh.empty(rt, (n,), np.float64)
        return [bh.reduce(name, x, 0)]
    counts, text = filter_text(_flush(prog), ("bcexp+reduce1d=32000",))
    assert counts == [1], text
    lines = [line for line in text.splitlines() if line.strip()]
    reds = [line for line in lines if int(line.split()[0]) == OP["ADD_REDUCE"]]
    assert len(reds) == 2, text
    assert "[0;32,32768;32768,1]" in reds[0], reds[0]
    assert "[0;32768;1]" in reds[1], reds[1]
    assert any(int(line.split()[0]) == OP["FREE"] for line in lines)
    # 16000 <= n: split; below, or without a divisor in [2, n/L]: unchanged
    for n, want in [(20_000, 0), (64_000, 1), (1_000_003, 0), (96_000, 1)]:
        counts, _ = filter_text(_flush(lambda rt, n=n: prog(rt, n, "MAXIMUM_REDUCE")), ("bcexp+reduce1d=32000",))
        assert counts == [want], n
    counts, _ = filter_text(_flush(prog), ("bcexp",))
    assert counts == [0]
