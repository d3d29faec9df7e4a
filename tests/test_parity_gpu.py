"""Parity of the CUDA engine with the CPU oracle (the restated ve/openmp) on the same bytecode.

Integer, boolean and random outputs must be bit-exact. Elementwise floating-point results may
differ by a few ulps (CUDA's vs glibc's math functions, FMA contraction on the CPU), reductions by
the change of summation order: 1e-5 relative for float32 and 1e-12 for float64.
"""
import numpy as np
import pytest

import bohrium_b200 as bh
from tests import programs as P
from tests.harness import assert_close, float_tol, reduce_tol, run

pytestmark = pytest.mark.gpu


def both(gpu_rt, oracle_rt, prog):
    return run(gpu_rt, prog), run(oracle_rt, prog)


@pytest.mark.parametrize("name", sorted(P.BINARY))
def test_binary_opcodes(gpu_rt, oracle_rt, name):
    for dt in P.BINARY[name]:
        g, o = both(gpu_rt, oracle_rt, P.binary_program(name, dt, n=777))
        # a - floor(a/b)*b cancels: the CPU's FMA contraction of the product moves the result by
        # an ulp of `a`, so remainders get an absolute tolerance at that scale.
        rtol, atol = float_tol(dt, name in P.TRANSCENDENTAL or name in ("REMAINDER", "MOD"))
        for k in range(2):
            assert_close(g[k], o[k], rtol, atol, f"{name} {np.dtype(dt)}")


@pytest.mark.parametrize("name", P.COMPARE)
def test_comparisons(gpu_rt, oracle_rt, name):
    for dt in P.INT_TYPES + P.FLOAT_TYPES:
        g, o = both(gpu_rt, oracle_rt, P.compare_program(name, dt, n=500))
        assert_close(g[0], o[0], 0, 0, f"{name} {np.dtype(dt)}")


@pytest.mark.parametrize("name", P.LOGICAL)
def test_logical(gpu_rt, oracle_rt, name):
    g, o = both(gpu_rt, oracle_rt, P.logical_program(name, n=500))
    assert_close(g[0], o[0], 0, 0, name)


@pytest.mark.parametrize("name", P.UNARY_FLOAT)
def test_unary_float(gpu_rt, oracle_rt, name):
    for dt in P.FLOAT_TYPES:
        g, o = both(gpu_rt, oracle_rt, P.unary_program(name, dt, n=1000))
        rtol, atol = float_tol(dt, name in P.TRANSCENDENTAL)
        assert_close(g[0], o[0], rtol, atol, f"{name} {np.dtype(dt)}")


@pytest.mark.parametrize("name", P.UNARY_ANY)
def test_unary_any(gpu_rt, oracle_rt, name):
    types = {"INVERT": P.INT_TYPES + [np.bool_], "LOGICAL_NOT": [np.bool_]}.get(
        name, P.INT_TYPES + P.FLOAT_TYPES)
    for dt in types:
        g, o = both(gpu_rt, oracle_rt, P.unary_program(name, dt, n=500))
        assert_close(g[0], o[0], 0, 0, f"{name} {np.dtype(dt)}")


def test_type_conversions(gpu_rt, oracle_rt):
    types = [np.bool_, np.int8, np.int32, np.int64, np.uint8, np.uint64, np.float32, np.float64]
    for s in types:
        for d in types:
            if s == d:
                continue
            g, o = both(gpu_rt, oracle_rt, P.identity_program(s, d))
            assert_close(g[0], o[0], 0, 0, f"{np.dtype(s)}->{np.dtype(d)}")


@pytest.mark.parametrize("name", P.REDUCE_OPS)
@pytest.mark.parametrize("shape,axis", [((1000,), 0), ((37, 53), 0), ((37, 53), 1), ((37, 53), None),
                                        ((5, 6, 7), 1), ((5, 6, 7), 2), ((3, 4, 5, 6), 0)])
def test_reductions(gpu_rt, oracle_rt, name, shape, axis):
    if name.startswith("LOGICAL"):
        types = [np.bool_]
    elif name.startswith("BITWISE"):
        types = [np.int32, np.uint64, np.bool_]
    else:
        types = [np.int64, np.float32, np.float64]
    for dt in types:
        g, o = both(gpu_rt, oracle_rt, P.reduce_program(name, dt, shape, axis))
        assert_close(g[0], o[0], reduce_tol(dt), 0, f"{name} {np.dtype(dt)} {shape} axis={axis}")


@pytest.mark.parametrize("view", ["transposed", "sliced", "reversed"])
@pytest.mark.parametrize("axis", [0, 1, None])
def test_reductions_of_views(gpu_rt, oracle_rt, view, axis):
    g, o = both(gpu_rt, oracle_rt, P.reduce_program("ADD_REDUCE", np.float64, (40, 30), axis, view))
    assert_close(g[0], o[0], 1e-12, 0, f"{view} axis={axis}")


def test_large_and_ragged_reductions(gpu_rt, oracle_rt):
    # lengths around the tile size (2048) and the grid size, and a long one
    for n in [1, 2, 255, 2047, 2048, 2049, 300001, 3_000_017]:
        g, o = both(gpu_rt, oracle_rt, P.reduce_program("ADD_REDUCE", np.float64, (n,), None))
        assert_close(g[0], o[0], 1e-12, 0, f"sum n={n}")
        g, o = both(gpu_rt, oracle_rt, P.reduce_program("MAXIMUM_REDUCE", np.int32, (n,), None))
        assert_close(g[0], o[0], 0, 0, f"max n={n}")


@pytest.mark.parametrize("name", ["ADD_ACCUMULATE", "MULTIPLY_ACCUMULATE"])
@pytest.mark.parametrize("shape,axis", [((1000,), 0), ((20, 30), 0), ((20, 30), 1), ((4, 5, 6), 2)])
def test_accumulate(gpu_rt, oracle_rt, name, shape, axis):
    for dt in [np.int64, np.float64]:
        g, o = both(gpu_rt, oracle_rt, P.accumulate_program(name, dt, shape, axis))
        assert_close(g[0], o[0], 1e-12, 0, f"{name} {np.dtype(dt)} {shape} {axis}")


def test_views_and_broadcast(gpu_rt, oracle_rt):
    g, o = both(gpu_rt, oracle_rt, P.views_program())
    for k in range(3):
        assert_close(g[k], o[k], 1e-14, 1e-15, f"views[{k}]")


@pytest.mark.parametrize("shape,start,key", [((1000,), 0, 42), ((33, 17), 12345, 7), ((5000,), 2**32 - 100, 2**40)])
def test_random_is_bit_exact(gpu_rt, oracle_rt, shape, start, key):
    g, o = both(gpu_rt, oracle_rt, P.random_program(shape, start, key))
    assert_close(g[0], o[0], 0, 0, "random123")
    assert_close(g[1], o[1], 0, 0, "random_sample float32")


def test_random_matches_reference_golden(gpu_rt):
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "random123.json")) as f:
        cases = json.load(f)["cases"]
    for case in cases:
        r = bh.random123(gpu_rt, (len(case["values"]),), case["start"], case["key"]).numpy()
        assert r.tolist() == case["values"]


def test_gather_scatter_range(gpu_rt, oracle_rt):
    g, o = both(gpu_rt, oracle_rt, P.gather_scatter_program(2000))
    assert_close(g[0], o[0], 0, 0, "gather")
    assert_close(g[1], o[1], 0, 0, "scatter")
    g, o = both(gpu_rt, oracle_rt, P.range_program(3000))
    assert_close(g[0], o[0], 0, 0, "range")
    assert_close(g[1], o[1], 0, 0, "range view")


@pytest.mark.parametrize("n", [4, 1024, 4096 * 3 + 4, 1 << 20])
def test_fused_chain(gpu_rt, oracle_rt, n):
    g, o = both(gpu_rt, oracle_rt, P.fused_chain_program(n))
    rtol = float_tol(np.float64, True)
    assert_close(g[0], o[0], *rtol, "map")
    for k in range(1, 5):
        assert_close(g[k], o[k], 1e-12, 1e-12, f"reduction[{k}]")


def test_empty_arrays(gpu_rt, oracle_rt):
    g, o = both(gpu_rt, oracle_rt, P.empty_program())
    assert g[0].shape == o[0].shape == (0,)


def test_repeat_with_condition_and_slides(gpu_rt, oracle_rt):
    """flush-and-repeat with a sliding view and a repeat condition (test/python/tests/test_loop.py)."""
    from bohrium_b200 import ir
    results = []
    for rt in (gpu_rt, oracle_rt):
        A = np.arange(20, dtype=np.float64)
        a = bh.array(rt, A)
        acc = bh.zeros(rt, (1,), np.float64)
        cond = bh.ones(rt, (1,), np.bool_)
        rt.flush()
        add = ir.Instr(ir.OPCODES["ADD"], [acc.view(), acc.view(), ir.View(a.base, 0, (1,), (1,))])
        add.slides[2] = ([ir.Slide(0, 1, 0, 1, 20)], {})
        # keep going while acc < 50
        less = ir.Instr(ir.OPCODES["LESS"], [cond.view(), acc.view(), None], ir.Constant(50.0, ir.FLOAT64))
        rt.ex.execute(ir.Flush([add, less], nrepeats=20, condition=cond.base))
        results.append(acc.numpy()[0])
    assert results[0] == results[1] == float(sum(range(11)))


@pytest.mark.parametrize("shape,axis", [((100_000, 3), 0), ((4096, 50), 0), ((3, 70_000), 1), ((2000, 2000), 0),
                                        ((16, 9000, 4), 1)])
def test_split_reductions(gpu_rt, oracle_rt, shape, axis):
    """Axis reductions with few outputs and a long swept axis (the split-reduction schedule),
    including a fused consumer of the reduction (mean = sum / n)."""
    def prog(rt):
        A = P.data(shape, np.float64, 11)
        a = bh.array(rt, A)
        m = a.max(axis)
        s = a.sum(axis)
        mean = s / float(shape[axis])
        return [m, s, mean]
    g, o = both(gpu_rt, oracle_rt, prog)
    assert_close(g[0], o[0], 0, 0, "max")
    assert_close(g[1], o[1], 1e-12, 1e-12, "sum")
    assert_close(g[2], o[2], 1e-12, 1e-12, "mean")


def test_grouped_launches_are_bit_identical(gpu_executor):
    """Independent kernels of one flush run as one grouped launch; the results equal the plain
    one-launch-per-kernel results bit for bit."""
    from bohrium_b200 import workloads as W
    rt = bh.Runtime(gpu_executor)
    lengths = W.batching_lengths(64, 256, 20000, 9)
    xs = [bh.array(rt, np.random.default_rng(i).random(int(n), dtype=np.float32)) for i, n in enumerate(lengths)]
    rt.flush()
    outs = []
    for x in xs:
        y = W.batching_chain(x)
        outs += [y, y.sum(), y.max()]
    ir = gpu_executor.compile(rt.take())
    results = {}
    try:
        for mode in ["off", "grouped"]:
            gpu_executor.message(f"CUDA: batch {mode}")
            l0 = int(gpu_executor.message("CUDA: launches"))
            ir.execute()
            ir.execute()
            launches = int(gpu_executor.message("CUDA: launches")) - l0
            results[mode] = [gpu_executor.peek(o.base) for o in outs]
            if mode == "grouped":
                assert launches <= 4, launches
            else:
                assert launches == 2 * 64, launches
    finally:
        gpu_executor.message("CUDA: batch off")
    for p, q in zip(results["off"], results["grouped"]):
        assert np.array_equal(p, q)


def test_replayed_flushes_keep_their_own_constants(gpu_executor, oracle_rt):
    """Compiled flushes of the same structure but different constants (and Random123 keys) share
    one plan; replaying each one must still use its own constants."""
    rt = bh.Runtime(gpu_executor)
    host = np.random.default_rng(3).random(10000)
    x = bh.array(rt, host)
    rt.flush()
    irs, outs = [], []
    for k in range(3):
        r = bh.random123(rt, (10000,), 5, 100 + k)
        y = (x * float(k + 2) + float(k)).sum()
        outs.append((y, r))
        irs.append(gpu_executor.compile(rt.take()))
    for _ in range(3):  # first run builds the plan, later runs replay it
        for ir in irs:
            ir.execute()
    for k, (y, r) in enumerate(outs):
        want_r = bh.random123(oracle_rt, (10000,), 5, 100 + k).numpy()
        assert np.array_equal(gpu_executor.peek(r.base), want_r), k
        want = float(np.sum(host * float(k + 2) + float(k)))
        got = float(gpu_executor.peek(y.base)[0])
        assert abs(got - want) <= 1e-12 * abs(want), (k, got, want)


@pytest.mark.parametrize("rows,cols,dtype,op", [
    (300, 1000, np.float64, "sum"), (512, 4096, np.float32, "max"), (200, 37, np.float32, "sum"),
    (1000, 3000, np.int32, "sum"), (149, 70001, np.float64, "min"), (4096, 64, np.float32, "prod"),
])
def test_row_reductions_lane_schedule(gpu_rt, oracle_rt, rows, cols, dtype, op):
    """Reductions over the contiguous axis of many rows (LANE_REDUCE), fused with the map before
    and the instruction after, against the oracle."""
    rng = np.random.default_rng(rows + cols)
    host = rng.random((rows, cols))
    if op == "prod":
        host = 1.0 + (host - 0.5) * 1e-3
    host = (host * 100).astype(dtype) if np.dtype(dtype).kind == "i" else host.astype(dtype)

    def prog(rt):
        x = bh.array(rt, host)
        y = getattr(x * dtype(2) + dtype(1), op)(axis=1)
        return [y, y * dtype(3)]

    g, o = both(gpu_rt, oracle_rt, prog)
    rtol = reduce_tol(dtype)
    for a, b, what in zip(g, o, ["reduce", "after"]):
        assert_close(a, b, rtol, rtol, what)


def _stencil_prog(host, rows, cols, dtype, op, offsets):
    """dst[2:2+rows, 1:1+cols] = sum_k (k + 1) * x[2 + dr_k + i, 1 + dc_k + j]; returns the
    reduction `op` of that sum over axis 1 and dst (the shape of the heat stencil)."""
    def prog(rt):
        x = bh.array(rt, host)
        dst = bh.zeros(rt, host.shape, dtype)
        acc = None
        for k, (dr, dc) in enumerate(offsets):
            term = x[2 + dr:2 + dr + rows, 1 + dc:1 + dc + cols] * dtype(k + 1)
            acc = term if acc is None else acc + term
        dst[2:2 + rows, 1:1 + cols] = acc
        return [getattr(acc - x[2:2 + rows, 1:1 + cols], op)(axis=1), dst]
    return prog


@pytest.mark.parametrize("rows,cols,dtype,op,offsets", [
    (1000, 1500, np.float64, "sum", [(0, 0), (-1, 0), (1, 0), (0, -1), (0, 1)]),
    (700, 4000, np.float32, "max", [(-2, 0), (-1, 0), (0, 0), (1, 0), (2, 0)]),
    (513, 300, np.float32, "sum", [(0, 0), (2, 0), (0, 1)]),
    (2000, 4094, np.float32, "max", [(0, 0), (-1, 0), (1, 0), (0, -1), (0, 1)]),
    (300, 4096, np.float64, "min", [(-1, -1), (0, 0), (1, 1), (-1, 1), (1, -1)]),
    (160, 257, np.float64, "sum", [(1, 0), (-1, 0)]),
])
def test_stencil_rows_lane_schedule(gpu_rt, oracle_rt, rows, cols, dtype, op, offsets):
    """Row reductions of stencils (shifted views of one array, the heat step's shape) on the
    LANE_REDUCE schedule with its inputs preloaded, against the oracle."""
    host = np.random.default_rng(rows + cols).random((rows + 4, cols + 2)).astype(dtype)
    g, o = both(gpu_rt, oracle_rt, _stencil_prog(host, rows, cols, dtype, op, offsets))
    rtol = reduce_tol(dtype)
    assert_close(g[0], o[0], rtol, rtol, "reduce")
    assert_close(g[1], o[1], *float_tol(dtype), "stencil")


@pytest.mark.parametrize("dtype,op", [(np.int32, "sum"), (np.int64, "max"), (np.complex64, "sum"),
                                      (np.complex128, "sum")])
def test_stencil_rows_other_element_types(gpu_rt, oracle_rt, dtype, op):
    """The staged stencil rows with integer and complex elements (4, 8 and 16-byte elements: the
    16-byte ones take the plain lane code), against the oracle."""
    rng = np.random.default_rng(5)
    shape = (604, 1004)  # a row of 1004 elements: 16-byte multiples for 4 and 8-byte elements
    if np.dtype(dtype).kind == "c":
        host = (rng.random(shape) + 1j * rng.random(shape)).astype(dtype)
    else:
        host = rng.integers(-1000, 1000, shape).astype(dtype)
    offsets = [(0, 0), (-1, 0), (1, 0), (0, -1), (0, 1)]
    g, o = both(gpu_rt, oracle_rt, _stencil_prog(host, 600, 1002, dtype, op, offsets))
    tol = 0 if np.dtype(dtype).kind == "i" else (1e-5 if np.dtype(dtype) == np.complex64 else 1e-12)
    assert_close(g[0], o[0], tol, tol, "reduce")
    assert_close(g[1], o[1], tol, tol, "stencil")


def test_stencil_rows_grouped_launch_is_bit_identical(gpu_executor):
    """Two independent stencils in one flush share a kernel and level, so batch mode "grouped"
    runs them as one grouped launch; results equal the plain launches' bit for bit."""
    rt = bh.Runtime(gpu_executor)
    offsets = [(0, 0), (-1, 0), (1, 0), (0, -1), (0, 1)]
    hosts = [np.random.default_rng(s).random((604, 1002)).astype(np.float32) for s in (1, 2)]
    res = {}
    try:
        for mode in ["off", "grouped"]:
            gpu_executor.message(f"CUDA: batch {mode}")
            outs = []
            for h in hosts:
                outs += _stencil_prog(h, 600, 1000, np.float32, "sum", offsets)(rt)
            res[mode] = [o.numpy().tobytes() for o in outs]
    finally:
        gpu_executor.message("CUDA: batch off")
    assert res["off"] == res["grouped"]


def test_matrix_full_reductions_grouped_and_graph(gpu_executor, oracle_rt):
    """Full reductions of matrices (a row or column reduction, then a small 1-D reduction of its
    results). Equal shapes in one flush share kernels and levels, so batch modes "grouped" and
    "graph" run them as grouped launches. Every mode gives the same bits, on every execution,
    within the reduction tolerance of the oracle."""
    shapes = [(3000, 257), (4096, 300), (5000, 40), (700, 1500)]
    hosts = [np.random.default_rng(k).random(s) for k, s in enumerate(shapes)]

    keep = []  # the inputs stay alive, so the compiled flush does not free them

    def prog(rt):
        outs = []
        for h in hosts * 2:  # pairs of equal shapes: the same kernel twice in one level
            x = bh.array(rt, h)
            keep.append(x)
            outs += [(x * 2.0 + 1.0).sum(), (x - 0.5).max()]
        return outs
    want = run(oracle_rt, prog)
    rt = bh.Runtime(gpu_executor)
    res = {}
    try:
        for mode in ["off", "grouped", "graph"]:
            gpu_executor.message(f"CUDA: batch {mode}")
            outs = prog(rt)
            ir = gpu_executor.compile(rt.take())
            runs = []
            for _ in range(3):
                ir.execute()
                runs.append([gpu_executor.peek(o.base).tobytes() for o in outs])
            assert runs[0] == runs[1] == runs[2], mode
            res[mode] = runs[0]
            got = [gpu_executor.peek(o.base) for o in outs]
            for g, w in zip(got, want):
                assert_close(g.reshape(w.shape), w, 1e-12, 1e-12, mode)
    finally:
        gpu_executor.message("CUDA: batch off")
    assert res["off"] == res["grouped"] == res["graph"]


def test_graph_replay_is_bit_identical(gpu_executor):
    """Batch mode "graph": a re-executed flush is captured into a CUDA graph (grouped launches,
    arrays created and freed inside the flush parked) and replayed; results equal the plain
    one-launch-per-kernel results bit for bit, on every replay."""
    from bohrium_b200 import workloads as W
    rt = bh.Runtime(gpu_executor)
    lengths = W.batching_lengths(48, 256, 30000, 11)
    hosts = [np.random.default_rng(i).random(int(n), dtype=np.float32) for i, n in enumerate(lengths)]
    xs = [bh.array(rt, h) for h in hosts]
    rt.flush()
    outs = []
    for x in xs:
        y = W.batching_chain(x)
        t = y * np.float32(2)          # a temporary that the flush creates and frees
        outs += [y, t.sum(), y.max(), (t - y).min()]
    ir = gpu_executor.compile(rt.take())
    results = {}
    try:
        for mode in ["off", "graph"]:
            gpu_executor.message(f"CUDA: batch {mode}")
            r0 = _stat(gpu_executor, "graph_replays")
            runs = []
            for _ in range(4):
                ir.execute()
                runs.append([gpu_executor.peek(o.base).tobytes() for o in outs])
            results[mode] = runs
            if mode == "graph":
                assert _stat(gpu_executor, "graph_replays") - r0 >= 2
    finally:
        gpu_executor.message("CUDA: batch off")
    for run in results["off"] + results["graph"]:
        assert run == results["off"][0]


def _stat(ex, key):
    for line in ex.message("statistic").splitlines():
        if line.startswith(key + ":"):
            return float(line.split(":")[1])
    return 0.0


def test_autotuned_variants_are_bit_identical(monkeypatch):
    """The first launches of a large kernel rotate through register-capped variants (autotuning);
    every launch gives the same bits. A fresh engine without a kernel cache directory, so no
    earlier process's tuning choice applies."""
    from bohrium_b200 import workloads as W
    monkeypatch.setenv("BH_CUDA_CACHE_DIR", "NONE")
    gpu_executor = bh.NativeExecutor(stack="cuda")
    rt = bh.Runtime(gpu_executor)
    n = 3 << 20
    S, K, T = W.black_scholes_inputs(n, 5)
    s, k, t = (bh.array(rt, x) for x in (S, K, T))
    rt.flush()
    # A heavy float64 kernel of its own (no other test compiles this source, so it is untuned).
    m = (bh.sqrt(s) * bh.log(k) / (t + 1.5) - bh.exp(-t) * 0.25).sum()
    ir = gpu_executor.compile(rt.take())
    t0 = _stat(gpu_executor, "tune_launches")
    seen = set()
    for _ in range(10):
        ir.execute()
        seen.add(gpu_executor.peek(m.base).tobytes())
    assert len(seen) == 1
    assert _stat(gpu_executor, "tune_launches") > t0
    want = float(np.sum(np.sqrt(S) * np.log(K) / (T + 1.5) - np.exp(-T) * 0.25))
    got = float(np.frombuffer(seen.pop(), dtype=np.float64)[0])
    assert abs(got - want) <= 1e-11 * abs(want)  # NumPy's exp/log differ from CUDA's by ulps
    del ir, m, s, k, t
    gpu_executor.close()


@pytest.mark.parametrize("n,dtype", [(1_000_003, np.float32), (16_000_000, np.float64), (45_000_001, np.float32)])
def test_grid_reduce_order_is_canonical(gpu_rt, n, dtype):
    """GRID_REDUCE sums in one fixed order whatever the number of tiles a work item takes (1, 2 or
    4 at these sizes): the GPU result equals the exact order model bit for bit."""
    from tests.harness import grid_reduce_sum
    x = np.random.default_rng(n).standard_normal(n).astype(dtype)
    got = bh.array(gpu_rt, x).sum().numpy()
    want = grid_reduce_sum(x)
    assert np.asarray(got).tobytes() == np.asarray(want).tobytes(), (got, want)


@pytest.mark.parametrize("n,dtype,name", [(1_000_003, np.float64, "ADD_ACCUMULATE"), (4_000_000, np.int64, "ADD_ACCUMULATE"),
                                          (2049, np.float32, "ADD_ACCUMULATE"), (300_001, np.float64, "MULTIPLY_ACCUMULATE"),
                                          (5_000_000, np.int32, "ADD_ACCUMULATE")])
def test_scan1d(gpu_rt, oracle_rt, n, dtype, name):
    """1-D cumulative sums/products with the instructions around them fused (SCAN1D: chunk totals,
    carries, re-scan), against the oracle's sequential scan."""
    rng = np.random.default_rng(n)
    if name == "MULTIPLY_ACCUMULATE":
        host = (1.0 + (rng.random(n) - 0.5) * 1e-5).astype(dtype)
    elif np.dtype(dtype).kind == "i":
        host = rng.integers(-50, 50, n).astype(dtype)
    else:
        host = rng.random(n).astype(dtype)

    def prog(rt):
        x = bh.array(rt, host)
        c = bh.accumulate(name, x * dtype(1) + dtype(0), 0)
        return [c, c * dtype(2)]

    g, o = both(gpu_rt, oracle_rt, prog)
    if np.dtype(dtype) == np.float32:
        # The oracle adds sequentially, the engine in SCAN1D's fixed order (bit-exact against its
        # order model in test_scan1d_order_is_canonical); each is held to its own rounding-error
        # bound around the exact prefix sums, and the engine to 1e-5 relative of them.
        from tests.harness import U32, assert_cumsum_within_bound, scan1d_depth
        for a, b, scale, what in zip(g, o, (1, 2), ("scan", "after")):
            assert_cumsum_within_bound(np.asarray(a) / scale, host, scan1d_depth(n), U32, what + " engine")
            assert_cumsum_within_bound(np.asarray(b) / scale, host, np.arange(1, n + 1), U32, what + " oracle")
            exact = np.cumsum(host.astype(np.float64)) * scale
            np.testing.assert_allclose(np.asarray(a, dtype=np.float64), exact, rtol=1e-5, atol=0, err_msg=what)
        return
    tol = 0 if np.dtype(dtype).kind == "i" else 1e-11
    for a, b, what in zip(g, o, ["scan", "after"]):
        assert_close(a, b, tol, tol, what)


@pytest.mark.parametrize("n,dtype", [(5, np.float64), (2049, np.float32), (1_000_003, np.float64),
                                     (4_500_001, np.float32), (9_000_001, np.float64)])
def test_scan1d_order_is_canonical(gpu_rt, n, dtype):
    """SCAN1D adds in one fixed order (per-thread runs of 8, block scans, carries over the chunk
    totals, more than one group of 2048 totals from 4.2M elements, each group's carry from the
    previous group's): the GPU cumulative sum of a fused input equals the exact order model bit
    for bit."""
    from tests.harness import scan1d_cumsum
    x = np.random.default_rng(n).standard_normal(n).astype(dtype)

    def prog(rt):
        return [bh.accumulate("ADD_ACCUMULATE", bh.array(rt, x) * dtype(1) + dtype(0), 0)]
    (got,) = run(gpu_rt, prog)
    want = scan1d_cumsum(x)
    assert np.asarray(got).tobytes() == want.tobytes()


@pytest.mark.parametrize("n,dtype", [(1, np.float64), (32, np.float32), (33, np.float64), (4097, np.float32)])
def test_small_maps_after_a_reduction_match_the_oracle(gpu_rt, oracle_rt, n, dtype):
    """A map of at most 32 elements that reads a reduction's result runs in the reduction kernel's
    tail (one CTA); a larger one keeps its own launch. Both against the oracle."""
    a_host = np.random.default_rng(n).random(1 << 20).astype(dtype)
    b_host = np.random.default_rng(n + 1).random(n).astype(dtype)

    def prog(rt):
        a, b = bh.array(rt, a_host), bh.array(rt, b_host)
        s = a.sum()
        return [s, b * s + dtype(1), bh.sqrt(b) - s / dtype(n)]
    g, o = both(gpu_rt, oracle_rt, prog)
    rtol = reduce_tol(dtype)
    assert_close(g[0], o[0], rtol, rtol, "sum")
    for x, y in zip(g[1:], o[1:]):
        assert_close(x, y, rtol, rtol, "map")


@pytest.mark.parametrize("name", ["ADD_ACCUMULATE", "MULTIPLY_ACCUMULATE"])
def test_scan1d_windows_equal_the_whole_length_units(gpu_rt, monkeypatch, name):
    """With scan_windows on, units A and C run one group of chunks at a time (C repeating unit
    B's scan of its group); by default the three units run over the whole length. Both give the same bits, for sums and products, over three groups and a
    partial one."""
    n = 3 * 2048 * 2048 + 12345
    rng = np.random.default_rng(17)
    x = (1.0 + 1e-7 * rng.standard_normal(n)) if name == "MULTIPLY_ACCUMULATE" else rng.standard_normal(n)

    def prog(rt):
        a = bh.array(rt, x)
        c = bh.accumulate(name, a * 1.0 + 0.0, 0)
        return [c, c * 2.0]
    whole = run(gpu_rt, prog)
    monkeypatch.setenv("BH_CUDA_SCAN_WINDOWS", "true")
    ex = bh.NativeExecutor(stack="cuda")
    try:
        windowed = run(bh.Runtime(ex), prog)
    finally:
        ex.close()
    for a, b in zip(windowed, whole):
        assert np.asarray(a).tobytes() == np.asarray(b).tobytes()
    if name == "ADD_ACCUMULATE":
        from tests.harness import scan1d_cumsum
        assert np.asarray(windowed[0]).tobytes() == scan1d_cumsum(x).tobytes()


@pytest.mark.parametrize("dtype", [np.float64, np.int64])
def test_scan1d_reads_values_from_before_the_accumulate(gpu_rt, oracle_rt, dtype):
    """Instructions after the accumulate that read a kept array computed before it, or the
    accumulate's own input array, against the oracle; float64 also bit for bit against the order
    model."""
    from tests.harness import scan1d_cumsum
    n = 1_000_003
    rng = np.random.default_rng(7)
    host = rng.standard_normal(n) if dtype == np.float64 else rng.integers(-50, 50, n)
    host = host.astype(dtype)

    def kept(rt):
        x = bh.array(rt, host)
        t = x * dtype(2) + dtype(1)
        c = bh.accumulate("ADD_ACCUMULATE", t, 0)
        return [t, c, c - t]

    def recomputed(rt):
        x = bh.array(rt, host)
        c = bh.accumulate("ADD_ACCUMULATE", x * dtype(2) + dtype(1), 0)
        # c - 2x: the product is exact, so its multiply-add contraction rounds once like NumPy's.
        return [c, c - x * dtype(2)]

    tol = 0 if dtype == np.int64 else 1e-11
    g, o = both(gpu_rt, oracle_rt, kept)
    for a, b, what in zip(g, o, ["kept", "scan", "after kept"]):
        assert_close(a, b, tol, tol, what)
    g2, o2 = both(gpu_rt, oracle_rt, recomputed)
    for a, b, what in zip(g2, o2, ["scan", "after recomputed"]):
        assert_close(a, b, tol, tol, what)
    if dtype == np.float64:
        t = host * 2.0 + 1.0
        c = scan1d_cumsum(t)
        assert g[1].tobytes() == c.tobytes() and g[2].tobytes() == (c - t).tobytes()
        assert g2[0].tobytes() == c.tobytes() and g2[1].tobytes() == (c - host * 2.0).tobytes()


@pytest.mark.parametrize("m,k,n,dtype,trans", [(64, 48, 80, np.float64, False), (300, 200, 100, np.float32, False),
                                               (128, 256, 64, np.float64, True)])
def test_blas_extmethods_on_cublas(gpu_rt, m, k, n, dtype, trans):
    """blas_gemm / blas_gemmt extension methods run on cuBLAS on the engine's device buffers, between
    regular bytecode before and after (NumPy is the witness, as in the reference's tests)."""
    rng = np.random.default_rng(m + n)
    A = rng.standard_normal((k, m) if trans else (m, k)).astype(dtype)
    B = rng.standard_normal((k, n)).astype(dtype)
    a = bh.array(gpu_rt, A) * dtype(2)
    b = bh.array(gpu_rt, B)
    c = bh.matmul(a, b, trans_a=trans) + dtype(1)
    got = c.numpy()
    want = (2 * (A.T if trans else A)).astype(np.float64) @ B.astype(np.float64) + 1
    rtol = 1e-4 if dtype == np.float32 else 1e-11
    np.testing.assert_allclose(got, want, rtol=rtol, atol=rtol * np.abs(want).max())
