"""Device-free checks of the engine's lowering: fusion plan, schedules, NVRTC compilation."""
import numpy as np
import pytest

import bohrium_b200 as bh
from bohrium_b200 import workloads as W
from tests import programs as P


def plan(prog, compile=True, fuser_list=None):
    ex = bh.DryRunExecutor()
    rt = bh.Runtime(ex)
    outs = prog(rt)
    flush = rt.take()
    flush.syncs = [o.base for o in outs]
    res = bh.dry_run(flush, compile=compile, fuser_list=fuser_list)
    units = [u for k in res["kernels"] for u in k["units"]]
    for u in units:
        assert u["compile_error"] == "", u["compile_error"][:3000]
    return res, units


def test_plain_chain_is_one_grid_reduction():
    def prog(rt):
        a, b, c = (bh.empty(rt, (1 << 20,), np.float64) for _ in range(3))
        return [W.plain_chain(rt, a, b, c)]
    res, units = plan(prog)
    assert [u["sched"] for u in units] == ["grid_reduce"]
    # the whole chain is contracted: only the three inputs and the scalar are read/written
    assert units[0]["bytes"] == 3 * 8 * (1 << 20) + 8


def test_black_scholes_iteration_is_one_kernel():
    """The whole iteration is one GRID_REDUCE launch: the mean (the sum divided by n, a
    one-element map) runs in its tail, in the CTA that finishes last."""
    def prog(rt):
        S, K, T = (bh.empty(rt, (10000,), np.float64) for _ in range(3))
        return [W.black_scholes_iteration(rt, S, K, T, 0)]
    res, units = plan(prog)
    scheds = [u["sched"] for u in units]
    assert scheds == ["grid_reduce"] and units[0]["tail"], scheds
    assert [k["folded_into"] for k in res["kernels"] if k["folded_into"] >= 0] == [0]


def test_small_maps_run_in_the_producers_tail_and_large_ones_do_not():
    """A map of at most 32 elements that reads a reduction's result runs in the reduction kernel's
    tail; a larger one keeps its own launch. Maps of every size share one kernel source."""
    def prog(n):
        def p(rt):
            a = bh.empty(rt, (1 << 20,), np.float32)
            b = bh.empty(rt, (n,), np.float32)
            return [b * a.sum() + 1.0]
        return p
    _, small = plan(prog(32))
    _, large = plan(prog(33))
    assert [u["sched"] for u in small] == ["grid_reduce"] and small[0]["tail"], [u["sched"] for u in small]
    assert [u["sched"] for u in large] == ["grid_reduce", "flat"], [u["sched"] for u in large]


def test_heat_step_fuses_stencil_write_and_split_partial_max():
    def prog(rt):
        a = bh.empty(rt, (64, 64), np.float32)
        b = bh.empty(rt, (64, 64), np.float32)
        return [W.heat_step(a, b), b]
    res, units = plan(prog)
    scheds = [u["sched"] for u in units]
    # the max over the 62 row maxima runs in the tail of the stencil kernel
    assert scheds == ["split_reduce"] and units[0]["tail"], scheds
    assert [k["folded_into"] for k in res["kernels"] if k["folded_into"] >= 0] == [0]


def test_small_order_free_second_level_reduction_runs_in_the_tail():
    """A 2-D max (or integer sum) is a row reduction followed by a small reduction of the row
    results: at most four tiles of those run in the first kernel's tail. Floating-point sums keep
    their own kernel (a different fold order would change the result), and so do larger arrays."""
    cases = [((4096, 300), np.float64, "max", True), ((8192, 300), np.float32, "min", True),
             ((4096, 300), np.int64, "sum", True), ((4096, 300), np.float64, "sum", False),
             ((8193, 300), np.float64, "max", False)]
    for shape, dt, op, folded in cases:
        def prog(rt, shape=shape, dt=dt, op=op):
            x = bh.empty(rt, shape, dt)
            return [getattr(getattr(x + dt(1), op)(axis=1), op)()]
        res, units = plan(prog)
        tails = [u["tail"] for u in units]
        assert any(tails) == folded, (shape, dt, op, [u["sched"] for u in units], tails)


def test_batching_systems_lower_to_one_unit_each():
    def prog(rt):
        outs = []
        for n in [300, 1000, 4097]:
            x = bh.empty(rt, (n,), np.float32)
            y = W.batching_chain(x)
            outs += [y, y.sum(), y.max()]
        return outs
    res, units = plan(prog)
    assert [u["sched"] for u in units] == ["grid_reduce"] * 3
    # one compiled kernel serves every length
    assert len({u["name"] for u in units}) == 1


@pytest.mark.parametrize("name", ["ADD", "DIVIDE", "REMAINDER", "POWER", "RIGHT_SHIFT", "MAXIMUM"])
@pytest.mark.parametrize("dtype", [np.int8, np.int64, np.uint32, np.float32])
def test_binary_opcodes_compile(name, dtype):
    if np.dtype(dtype) not in [np.dtype(t) for t in P.BINARY[name]]:
        pytest.skip("signature not defined")
    plan(P.binary_program(name, dtype, n=64))


@pytest.mark.parametrize("name", P.UNARY_FLOAT + ["ABSOLUTE", "SIGN", "ISNAN"])
def test_unary_opcodes_compile(name):
    plan(P.unary_program(name, np.float64, n=64))


@pytest.mark.parametrize("name", P.REDUCE_OPS)
def test_reductions_compile(name):
    dt = np.bool_ if name.startswith("LOGICAL") else (np.int32 if "BITWISE" in name else np.float32)
    plan(P.reduce_program(name, dt, (33, 65), None))


def test_views_random_gather_scatter_compile():
    for prog in [P.views_program(), P.random_program((100,), 1, 2), P.gather_scatter_program(100),
                 P.range_program(100), P.fused_chain_program(1024),
                 P.accumulate_program("ADD_ACCUMULATE", np.float64, (8, 9), 1),
                 P.accumulate_program("MULTIPLY_ACCUMULATE", np.int64, (40,), 0)]:
        plan(prog)


def test_outer_axis_reduction_runs_on_gpu_without_swap():
    """Without push_reductions_inwards an axis-0 reduction sweeps rank 0; it must still lower to a
    GPU schedule (the reference offloads such blocks to the CPU)."""
    prog = P.reduce_program("ADD_REDUCE", np.float64, (100, 7, 5), 0)
    res, units = plan(prog, fuser_list="greedy,collapse_redundant_axes")
    assert "outer_reduce" in [u["sched"] for u in units]


def test_bounds_are_parameters_not_constants():
    """Loop sizes, offsets and strides are kernel parameters: shapes share compiled kernels."""
    names = set()
    for n in [1000, 2000, 12345]:
        def prog(rt, n=n):
            a = bh.empty(rt, (n,), np.float32)
            return [bh.sqrt(a) + 1]
        _, units = plan(prog, compile=False)
        names.add(units[0]["name"])
    assert len(names) == 1


def test_row_reductions_of_contiguous_rows_use_lanes():
    """A reduction over the contiguous axis with enough rows lowers to LANE_REDUCE (C lanes of one
    CTA per row); few rows keep SPLIT_REDUCE; a reduction over the strided axis never uses lanes."""
    def prog_rows(rt):
        x = bh.empty(rt, (300, 1000), np.float64)
        return [(x * 2.0 + 1.0).sum(axis=1) * 3.0]
    res, units = plan(prog_rows)
    assert [u["sched"] for u in units] == ["lane_reduce"], [u["sched"] for u in units]

    def prog_few(rt):
        x = bh.empty(rt, (20, 100000), np.float32)
        return [x.max(axis=1)]
    res, units = plan(prog_few)
    assert "lane_reduce" not in [u["sched"] for u in units]

    def prog_cols(rt):
        x = bh.empty(rt, (1000, 300), np.float64)
        return [x.sum(axis=0)]
    res, units = plan(prog_cols)
    assert "lane_reduce" not in [u["sched"] for u in units]


def test_one_dimensional_accumulate_lowers_to_scan_units_or_one_pass(monkeypatch):
    """By default a 1-D accumulate is the three units (chunk totals, carries, re-scan) over the
    whole length; with scan_windows on it is units A and C (the
    re-scan repeating unit B's scan of the group's totals) per group of 2048 chunks; with
    scan_single_pass on it is one unit (look-back with bounded waits and a fallback)."""
    def prog(rt):
        a = bh.empty(rt, (100000,), np.float64)
        return [bh.accumulate("ADD_ACCUMULATE", a * 2.0 + 1.0, 0) * 3.0]
    res, units = plan(prog)
    assert [u["sched"] for u in units] == ["scan1d", "scan1d", "scan1d"], [u["sched"] for u in units]
    assert all("chunk_carry" not in u["source"] for u in units)
    assert all("const bh_i64 c = p.first + w;" in u["source"] for u in units)
    monkeypatch.setenv("BH_CUDA_SCAN_WINDOWS", "true")
    res, units = plan(prog)
    assert [u["sched"] for u in units] == ["scan1d", "scan1d"], [u["sched"] for u in units]
    assert "chunk_carry" in units[1]["source"] and "chunk_carry" not in units[0]["source"]
    monkeypatch.delenv("BH_CUDA_SCAN_WINDOWS")
    monkeypatch.setenv("BH_CUDA_SCAN_SINGLE_PASS", "true")
    res, units = plan(prog)
    assert [u["sched"] for u in units] == ["scan1d"], [u["sched"] for u in units]
    src = units[0]["source"]
    assert "bh_await" in src and "p.spin_cap" in src and "atomicExch(ctr + 2, 1u)" in src


@pytest.mark.parametrize("dtype", [np.float64, np.int8, np.complex128])
def test_scan_units_stage_elements_at_coalesced_positions(dtype):
    """The chunk-total and re-scan units compute the accumulate's input at element k*256 + t of the
    chunk in thread t and stage it in shared memory, from which thread t folds elements
    8t..8t+7; instructions after the accumulate run at the coalesced positions again. Kept arrays
    and the input array read after the accumulate compile for 1-, 8- and 16-byte elements."""
    def kept(rt):
        x = bh.empty(rt, (1_000_003,), dtype)
        t = x * dtype(2) + dtype(1)
        c = bh.accumulate("ADD_ACCUMULATE", t, 0)
        return [t, c, c - t]

    def recomputed(rt):
        x = bh.empty(rt, (1_000_003,), dtype)
        c = bh.accumulate("ADD_ACCUMULATE", x * dtype(2) + dtype(1), 0)
        return [c, c - x * dtype(3)]

    for prog in (kept, recomputed):
        import os
        os.environ["BH_CUDA_SCAN_SINGLE_PASS"] = "true"
        try:
            _, units = plan(prog)  # one pass: both stagings in the one unit
        finally:
            del os.environ["BH_CUDA_SCAN_SINGLE_PASS"]
        assert [u["sched"] for u in units] == ["scan1d"]
        src = units[0]["source"]
        assert "const int q = k * 256 + (int)threadIdx.x;" in src
        assert "stage[q + (q >> 3)] = x;" in src and "= stage[q + (q >> 3)];" in src
        _, units = plan(prog)
        assert [u["sched"] for u in units] == ["scan1d"] * 3
        for phase in (0, 2):
            src = units[phase]["source"]
            assert "const int q = k * 256 + (int)threadIdx.x;" in src
            assert "stage[q + (q >> 3)] = x;" in src
        assert "= stage[q + (q >> 3)];" in units[2]["source"]


def test_scan_units_prefetch_their_inputs_through_a_tma_ring(monkeypatch):
    """Units A and C read their unit-stride read-only inputs (the accumulate's own input, or the
    array a fused input is computed from) from a two-slot shared-memory ring filled by TMA bulk
    copies one chunk ahead; unit B has none. With scan_prefetch off, no unit has the ring."""
    def direct(rt):
        y = bh.empty(rt, (1_000_000,), np.float64)
        return [bh.accumulate("ADD_ACCUMULATE", y, 0)]

    def fused(rt):
        x = bh.empty(rt, (1_000_000,), np.float32)
        return [bh.accumulate("ADD_ACCUMULATE", x * np.float32(2), 0)]
    for prog in (direct, fused):
        _, units = plan(prog)
        assert [u["sched"] for u in units] == ["scan1d"] * 3, [u["sched"] for u in units]
        for k, u in enumerate(units):
            ring = "bh_pf_issue" in u["source"] and "bh_bulk_row(ring" in u["source"]
            assert ring == (k != 1), (prog.__name__, k, ring)
    monkeypatch.setenv("BH_CUDA_SCAN_PREFETCH", "false")
    for prog in (direct, fused):
        _, units = plan(prog)
        assert all("bh_pf_issue" not in u["source"] for u in units)


def test_scan_windows_are_groups_of_chunks_sharing_two_kernels(monkeypatch):
    """A scan over 2.5 groups of chunks (2048 chunks of 2048 elements each) is units A and C for
    each group in turn: the same two compiled kernels, with the group's first chunk and chunk
    count as parameters; a window's algorithmic bytes are its share of the scan's."""
    n = 2048 * 2048 * 2 + 2048 * 1024 + 5

    def prog(rt):
        a = bh.empty(rt, (n,), np.float64)
        return [bh.accumulate("ADD_ACCUMULATE", a, 0)]
    monkeypatch.setenv("BH_CUDA_SCAN_WINDOWS", "true")
    _, units = plan(prog, compile=False)
    assert [u["sched"] for u in units] == ["scan1d"] * 6
    names = [u["name"] for u in units]
    assert names[0] == names[2] == names[4] and names[1] == names[3] == names[5] and names[0] != names[1]
    monkeypatch.setenv("BH_CUDA_SCAN_WINDOWS", "false")
    _, whole = plan(prog, compile=False)
    assert [u["work"] for u in whole] == [5121, 3, 5121]
    assert sum(u["bytes"] for u in units) == pytest.approx(whole[2]["bytes"], rel=1e-6)
    assert [u["work"] for u in units] == [2048, 2048, 2048, 2048, 1025, 1025]


def test_complex_programs_compile_for_every_schedule():
    """Complex64/complex128 kernels compile with NVRTC: every elementwise opcode of the complex
    type signatures, and reductions/accumulates on the GRID_REDUCE, SPLIT_REDUCE, LANE_REDUCE and
    SCAN1D schedules (16-byte partials, shuffles and scan totals for complex128)."""
    seen = set()
    for dt in P.COMPLEX_TYPES:
        progs = [P.complex_binary_program(n, dt) for n in P.COMPLEX_BINARY]
        progs += [P.complex_unary_program(n, dt) for n in P.COMPLEX_UNARY + P.COMPLEX_TO_REAL + P.COMPLEX_PREDICATES]
        progs += [P.complex_compare_program("EQUAL", dt), P.complex_gather_scatter_program(dt)]
        progs += [P.complex_reduce_program(n, dt, shape, ax) for n in ("ADD_REDUCE", "MULTIPLY_REDUCE")
                  for shape, ax in [((1 << 20,), 0), ((4096, 64), 0), ((4096, 4096), 1), ((40, 30), 1)]]
        progs += [P.complex_accumulate_program("ADD_ACCUMULATE", dt, (1 << 20,), 0)]
        for prog in progs:
            _, units = plan(prog)
            seen.update(u["sched"] for u in units)
    _, units = plan(P.complex_chain_program(1 << 20))
    assert [u["sched"] for u in units] == ["grid_reduce"]
    assert {"flat", "grid_reduce", "split_reduce", "lane_reduce", "scan1d"} <= seen, seen



def test_heat_step_stages_stencil_rows_in_shared_memory():
    """The heat step's five shifted views of one grid form a stencil group: the lane kernel stages
    grid rows in a ring of shared-memory buffers with asynchronous copies (one row ahead) and asks
    for the ring as dynamic shared memory, with a launch-time check that falls back to the plain
    lane code."""
    def prog(rt):
        a, b = bh.empty(rt, (4096, 4096), np.float32), bh.empty(rt, (4096, 4096), np.float32)
        return [W.heat_step(a, b)]
    res, units = plan(prog)
    lane = [u for u in units if u["sched"] == "lane_reduce"]
    assert len(lane) == 1
    src = lane[0]["source"]
    assert "bh_work_staged(p, lo, hi)" in src and "bh_stage_ok(p, lo, hi)" in src
    assert "// bh_dynamic_shared_bytes: 65600" in src  # 4 rows of 4,100 floats
    assert "cp.async.cg.shared.global" in src


def _fma_count(units):
    """Fused multiply-adds per element: the FLAT and GRID_REDUCE bodies are written twice (full
    tiles without bounds checks, the last one with them)."""
    import re
    n = sum(len(re.findall(r"\bfmaf?\(", u["source"])) for u in units)
    assert n % 2 == 0, n
    return n // 2


def test_black_scholes_multiply_adds_are_contracted_on_the_bytecode():
    """Every product whose only use is one add or subtract, after which it is freed, becomes one
    fused multiply-add before fusion: 17 per option in a Black-Scholes iteration (the erf
    polynomials, the drift term, d2 and the call price)."""
    def prog(rt):
        S, K, T = (bh.empty(rt, (10000,), np.float64) for _ in range(3))
        return [W.black_scholes_iteration(rt, S, K, T, 0)]
    res, units = plan(prog)
    assert _fma_count(units) == 17


@pytest.mark.parametrize("case", ["plain", "synced", "reused", "written_between", "float_only"])
def test_multiply_add_contraction_conditions(case):
    """Contraction needs a float product read once by the next instruction that touches it (an
    add or subtract), freed after that, not synced, with its inputs not written in between."""
    dt = np.int32 if case == "float_only" else np.float32

    def prog(rt):
        a = bh.empty(rt, (4096,), dt)
        b = bh.empty(rt, (4096,), dt)
        t = a * b
        outs = []
        if case == "written_between":
            bh.binary("ADD", a, dt(1), out=a)
        r = t + b
        if case == "reused":
            outs.append(t * dt(3))
        if case == "synced":
            outs.append(t)
        del t
        return [r] + outs
    res, units = plan(prog)
    assert _fma_count(units) == (1 if case == "plain" else 0), case


@pytest.mark.parametrize("dt", [np.float32, np.float64, np.int32])
def test_transposed_views_lower_to_tma_tiles(dt):
    """A 2-D map reading through transposed views is a TILE2D unit: TMA boxes of 128 bytes x 64
    rows per transposed view, 64 elements x TR rows for the row-wise view beside them, the tensor
    maps first in the parameter struct."""
    def prog(rt):
        a = bh.empty(rt, (300, 500), dt)
        b = bh.empty(rt, (500, 300), dt)
        c = bh.empty(rt, (500, 300), dt)
        return [a + b.T * dt(2) + c.T]
    res, units = plan(prog)
    assert [u["sched"] for u in units] == ["tile2d"]
    src = units[0]["source"]
    assert src.count("cp.async.bulk.tensor.2d") == 1 and src.count("bh_tma_2d(stage") == 3
    assert "bh_tmap tm0;" in src and "bh_tmap tm1;" in src and "bh_tmap tm2;" in src
    assert src.count("+ tc * 64), (int)(p.ty") == 1  # the row-wise view's box moves along its rows
    assert src.index("bh_tmap tm0;") < src.index("a0;")
    assert "bh_mbar_wait" in src and "(1 << 20)" in src  # bounded waits


def test_untransposed_and_complex_maps_stay_flat():
    def prog(rt):
        a = bh.empty(rt, (300, 500), np.float32)
        z = bh.empty(rt, (500, 300), np.complex64)
        return [a + a, z.T * z.T]
    res, units = plan(prog)
    assert [u["sched"] for u in units] == ["flat", "flat"]


def test_generated_tma_copies_land_in_the_issuing_cta_only():
    """Every TMA copy the engine generates (TILE2D tiles, staged stencil rows, the scan's prefetch
    ring) reads this GPU's own memory into the issuing CTA's shared memory: no source copies to
    several CTAs of a cluster, and none is launched with a cluster shape."""
    def transpose(rt):
        a, b = bh.empty(rt, (1024, 1024), np.float32), bh.empty(rt, (1024, 1024), np.float32)
        return [a + b.T]

    def heat(rt):
        a, b = bh.empty(rt, (512, 512), np.float32), bh.empty(rt, (512, 512), np.float32)
        return [W.heat_step(a, b), b]

    def scan(rt):
        x = bh.empty(rt, (1_000_000,), np.float64)
        return [bh.accumulate("ADD_ACCUMULATE", x * 2.0, 0)]
    sources = []
    for prog in (transpose, heat, scan):
        _, units = plan(prog)
        sources += [u["source"] for u in units]
    assert any("cp.async.bulk.tensor" in src for src in sources)
    assert any("cp.async.bulk.shared" in src for src in sources)
    to_cluster = "multi" + "cast"  # the qualifier of a copy to several CTAs
    for src in sources:
        assert to_cluster not in src and "__cluster_dims__" not in src


def test_small_light_grid_reductions_hold_one_variant_per_launch_mode():
    """A light grid reduction over at most 64 tiles takes 1 tile per work item in a plain launch
    and 4 in a grouped one: its source holds the device code for both (bh_work for plain
    launches, bh_batch_work for grouped ones). Heavy or large reductions have one variant."""
    from bohrium_b200 import workloads as W

    def small(rt):
        x = bh.empty(rt, (30000,), np.float32)
        y = W.batching_chain(x)
        return [y, y.sum(), y.max()]

    def large(rt):
        x = bh.empty(rt, (1 << 24,), np.float32)
        y = W.batching_chain(x)
        return [y, y.sum(), y.max()]
    _, units = plan(small)
    src = units[0]["source"]
    assert "namespace bh_kp" in src and "namespace bh_kg" in src
    assert "const bh_i64 tile0 = w * 1;" in src and "const bh_i64 tile0 = w * 4;" in src
    assert "void bh_batch_work(const P &p, bh_i64 w) { bh_kg::bh_work(p, w); }" in src
    assert units[0]["work"] == 15  # plain work items: one tile each
    _, units = plan(large)
    assert "namespace bh_kg" not in units[0]["source"]
