"""TILE2D: 2-D maps that read arrays through transposed views, with the views' tiles brought into
shared memory by TMA (cp.async.bulk.tensor.2d). Results against the oracle (the restated
ve/openmp) -- bit-exact, since these are single additions and products of the same operands --
and the TMA path against the same tiles with plain loads (grouped launches, unaligned views)."""
import numpy as np
import pytest

import bohrium_b200 as bh
from tests.harness import assert_close, run

pytestmark = pytest.mark.gpu


def _stats(ex):
    out = {}
    for line in ex.message("statistic").splitlines():
        if ":" in line and not line.startswith(" "):
            k, v = line.split(":", 1)
            try:
                out[k.strip()] = float(v)
            except ValueError:
                pass
    return out


def _data(shape, dt, seed):
    rng = np.random.default_rng(seed)
    if np.dtype(dt).kind == "f":
        return rng.standard_normal(shape).astype(dt)
    return rng.integers(-1000, 1000, shape).astype(dt)


@pytest.mark.parametrize("dt", [np.float32, np.float64, np.int32, np.int64])
@pytest.mark.parametrize("shape", [(1000, 776), (4096, 4096), (96, 4100), (33, 64)])
def test_transpose_add_matches_oracle(gpu_executor, gpu_rt, oracle_rt, dt, shape):
    A, B = _data(shape, dt, 1), _data(shape[::-1], dt, 2)

    def prog(rt):
        a, b = bh.array(rt, A), bh.array(rt, B)
        return [a + b.T, a * dt(3) - b.T]
    t0 = _stats(gpu_executor).get("tma_units", 0)
    g, o = run(gpu_rt, prog), run(oracle_rt, prog)
    for k, (x, y) in enumerate(zip(g, o)):
        assert np.asarray(x).tobytes() == np.asarray(y).tobytes(), k
    assert_close(g[0], A + B.T, 0, 0, "vs numpy")
    # TMA needs rows of B on 16-byte boundaries; (33, 64) has rows of 33 elements: plain loads.
    tma = (shape[0] * np.dtype(dt).itemsize) % 16 == 0
    assert (_stats(gpu_executor)["tma_units"] > t0) == tma


def test_two_transposed_views_and_fallbacks(gpu_executor, gpu_rt, oracle_rt):
    """Two staged views in one kernel; a view whose start is not on a 16-byte boundary (plain
    loads); grouped launches (plain loads): all bit-identical to the oracle."""
    n = 1536
    A, B, C = (_data((n, n), np.float32, s) for s in (3, 4, 5))

    def prog(rt):
        a, b, c = (bh.array(rt, x) for x in (A, B, C))
        out = [a.T * np.float32(2) + b.T + c]
        sub = b[1:, 3:]  # start column 3: not 16-byte aligned
        out.append(a[: n - 3, : n - 1] + sub.T)
        return out
    want = run(oracle_rt, prog)
    for mode in ("off", "grouped"):
        gpu_executor.message(f"CUDA: batch {mode}")
        try:
            got = run(gpu_rt, prog)
        finally:
            gpu_executor.message("CUDA: batch off")
        for k, (x, y) in enumerate(zip(got, want)):
            assert np.asarray(x).tobytes() == np.asarray(y).tobytes(), (mode, k)
