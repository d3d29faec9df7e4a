"""The exact order models of tests/harness.py on the CPU: integer inputs, where every order gives
the same result, pin their structure (tiles, chunks, groups of chunk totals, carries); float
inputs stay within the rounding error of a long sum; and a scalar transcription of the SCAN1D
unit steps (thread folds, shuffle scan, warp offsets, carries) agrees bit for bit on small cases.
The GPU tests compare the engine with the same models bit for bit."""
import numpy as np
import pytest

from tests.harness import grid_reduce_sum, scan1d_cumsum


def _scalar_block_scan(vals, zero):
    """One CTA's block scan written out per thread: returns (exclusive prefixes, total)."""
    x = list(vals)
    for d in (1, 2, 4, 8, 16):
        prev = list(x)
        for t in range(256):
            if t % 32 >= d:
                x[t] = prev[t - d] + prev[t]
    ex = [zero if t % 32 == 0 else x[t - 1] for t in range(256)]
    run, wo = zero, []
    for w in range(8):
        wo.append(run)
        run = run + x[32 * w + 31]
    return [wo[t // 32] + ex[t] for t in range(256)], run


def _scalar_scan1d(x):
    dt = x.dtype.type
    zero = dt(0)
    n = x.size
    nch = -(-n // 2048)
    totals, prefixes = [], []
    for c in range(nch):
        sums = []
        for t in range(256):
            s = zero
            for k in range(8):
                i = 2048 * c + 8 * t + k
                if i < n:
                    s = s + x[i]
            sums.append(s)
        e, tot = _scalar_block_scan(sums, zero)
        totals.append(tot)
        prefixes.append(e)
    carries = [zero] * nch
    run = zero
    for base in range(0, nch, 2048):
        v = [[zero] * 8 for _ in range(256)]
        sums = []
        for t in range(256):
            s = zero
            for k in range(8):
                j = base + 8 * t + k
                v[t][k] = s
                if j < nch:
                    s = s + totals[j]
            sums.append(s)
        e, tot = _scalar_block_scan(sums, zero)
        for t in range(256):
            for k in range(8):
                j = base + 8 * t + k
                if j < nch:
                    carries[j] = run + (e[t] + v[t][k])
        run = run + tot
    out = np.empty(n, dtype=x.dtype)
    for c in range(nch):
        for t in range(256):
            r = zero
            for k in range(8):
                i = 2048 * c + 8 * t + k
                if i < n:
                    r = r + x[i]
                    out[i] = carries[c] + (prefixes[c][t] + r)
    return out


@pytest.mark.parametrize("n", [1, 7, 2047, 2048, 2049, 6000])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_scan_model_matches_scalar_transcription(n, dtype):
    x = np.random.default_rng(n).standard_normal(n).astype(dtype)
    assert scan1d_cumsum(x).tobytes() == _scalar_scan1d(x).tobytes()


@pytest.mark.parametrize("n", [1, 2049, 300_001, 4_194_304, 4_194_305, 9_000_001])
def test_scan_model_is_a_cumulative_sum(n):
    """Integers: exact at every length, across one and several groups of 2048 chunk totals."""
    x = np.random.default_rng(n).integers(-1000, 1000, n).astype(np.int64)
    assert np.array_equal(scan1d_cumsum(x), np.cumsum(x))
    f = np.random.default_rng(n).random(n)
    want = np.cumsum(f.astype(np.longdouble))
    assert np.max(np.abs(scan1d_cumsum(f) - want)) <= 1e-12 * max(1.0, float(want[-1]))


@pytest.mark.parametrize("n", [1, 2048, 2049, 1_000_003, 3_000_017])
def test_grid_reduce_model_is_a_sum(n):
    x = np.random.default_rng(n).integers(-1000, 1000, n).astype(np.int64)
    assert grid_reduce_sum(x) == x.sum()
    f = np.random.default_rng(n).random(n)
    assert abs(float(grid_reduce_sum(f)) - float(np.sum(f.astype(np.longdouble)))) <= 1e-12 * n


@pytest.mark.parametrize("n", [5, 2049, 300_001, 4_500_001])
def test_scan1d_model_within_its_depth_bound(n):
    """The SCAN1D order model stays inside the rounding-error bound that the GPU tests hold the
    engine to (gamma of `scan1d_depth` times the prefix sums of |x|), and sequential float32 sums
    inside the bound of their position."""
    from tests.harness import U32, assert_cumsum_within_bound, scan1d_depth
    x = np.random.default_rng(n).standard_normal(n).astype(np.float32)
    assert_cumsum_within_bound(scan1d_cumsum(x), x, scan1d_depth(n), U32, "model")
    assert_cumsum_within_bound(np.cumsum(x), x, np.arange(1, n + 1), U32, "sequential")


def _scalar_block_tree(vals, dt):
    """One CTA's tree written out per thread: xor butterfly in each warp (lane l adds lane l^m),
    warp sums in shared memory, the same butterfly over them in warp 0 (lanes >= 8 give 0)."""
    v = [dt.type(x) for x in vals]
    for m in (16, 8, 4, 2, 1):
        v = [dt.type(v[i] + v[(i & ~31) | ((i & 31) ^ m)]) for i in range(256)]
    w = [v[32 * k] for k in range(8)] + [dt.type(0)] * 24
    for m in (16, 8, 4, 2, 1):
        w = [dt.type(w[i] + w[i ^ m]) for i in range(32)]
    return w[0]


@pytest.mark.parametrize("n", [1, 2047, 2049, 5000, 600_001])
def test_grid_reduce_model_matches_a_scalar_transcription(n):
    """The GRID_REDUCE order model against the kernel's steps written out thread by thread:
    thread t of a tile adds its elements 4t..4t+3 and 1024+4t..1024+4t+3 in order (the two
    128-bit words it loads), then the CTA tree; the tile partials are folded and reduced the same
    way by one CTA. Bit for bit."""
    dt = np.dtype(np.float32)
    x = np.random.default_rng(n).standard_normal(n).astype(dt)
    ntiles = -(-n // 2048)
    parts = []
    for tile in range(ntiles if n < 100_000 else 0):
        sums = []
        for t in range(256):
            acc = dt.type(0)
            for j in range(8):
                i = tile * 2048 + (j >> 2) * 1024 + 4 * t + (j & 3)
                if i >= n:
                    break
                acc = dt.type(acc + x[i])
            sums.append(acc)
        parts.append(_scalar_block_tree(sums, dt))
    if n >= 100_000:  # the thread folds vectorised, the trees still written out
        pad = np.zeros(ntiles * 2048, dt)
        pad[:n] = x
        t4 = pad.reshape(ntiles, 2, 256, 4)
        acc = np.zeros((ntiles, 256), dt)
        for j in range(8):
            acc = acc + t4[:, j >> 2, :, j & 3]
        parts = [_scalar_block_tree(acc[k], dt) for k in range(ntiles)]
    fold = [dt.type(0)] * 256
    for t in range(256):
        for k in range(t, ntiles, 256):
            fold[t] = dt.type(fold[t] + parts[k])
    want = _scalar_block_tree(fold, dt)
    assert grid_reduce_sum(x).tobytes() == np.asarray(want, dtype=dt).tobytes()


def _single_pass_scan(x):
    """The single-pass SCAN1D's arithmetic chunk by chunk, as its look-back forms it: each chunk's
    exclusive prefix within its thread (v), the thread sums and warp totals that the closing chunks
    publish (32-lane shuffle scan), the warp offsets, and the group carries chained group by group.
    The chunk totals and in-chunk scans are unit A/C's (the model's own helpers)."""
    from tests.harness import _block_scan
    dt = x.dtype
    zero = dt.type(0)
    n = x.size
    nch = -(-n // 2048)
    pad = np.zeros(nch * 2048, dtype=dt)
    pad[:n] = x
    xs = pad.reshape(nch, 256, 8)
    valid = (np.arange(nch * 2048) < n).reshape(nch, 256, 8)
    s = np.full((nch, 256), zero, dtype=dt)
    for k in range(8):
        s = np.where(valid[:, :, k], s + xs[:, :, k], s)
    e, totals = _block_scan(s)
    tsum, wtot, gcarry = {}, {}, {0: zero}
    carry = np.empty(nch, dtype=dt)
    for c in range(nch):  # in ticket order: everything a chunk waits for is published before it
        g, q = divmod(c, 2048)
        k, t = q & 7, q >> 3
        l, w = t & 31, t >> 5
        v = zero
        for i in range(k):
            v = dt.type(v + totals[c - k + i])
        sT = dt.type(v + totals[c])
        if k == 7:
            tsum[c >> 3] = sT
        lanes = [tsum[(c >> 3) - l + i] if i < l else (sT if i == l and k == 7 else zero) for i in range(32)]
        for d in (1, 2, 4, 8, 16):
            lanes = [dt.type(lanes[i - d] + lanes[i]) if i >= d else lanes[i] for i in range(32)]
        ex = lanes[l - 1] if l > 0 else zero
        if k == 7 and l == 31:
            wtot[c >> 8] = lanes[31]
        wo = zero
        for i in range(w):
            wo = dt.type(wo + wtot[(c >> 8) - w + i])
        within = dt.type(dt.type(wo + ex) + v)
        carry[c] = dt.type(gcarry[g] + within)
        if q == 2047:
            gt = zero
            for i in range(7):
                gt = dt.type(gt + wtot[(c >> 8) - 7 + i])
            gt = dt.type(gt + lanes[31])
            gcarry[g + 1] = dt.type(gcarry[g] + gt)
    out = np.empty((nch, 256, 8), dtype=dt)
    r = np.full((nch, 256), zero, dtype=dt)
    for k in range(8):
        r = np.where(valid[:, :, k], r + xs[:, :, k], r)
        out[:, :, k] = carry[:, None] + (e + r)
    return out.reshape(-1)[:n]


@pytest.mark.parametrize("n", [5, 2049, 300_001, 4_500_001])
def test_single_pass_lookback_equals_the_order_model(n):
    """The single-pass scan's look-back (thread sums, warp totals, group carries published by the
    chunks that close them) rebuilds exactly the three units' carries: bit for bit the model."""
    x = np.random.default_rng(n + 1).standard_normal(n).astype(np.float32)
    assert _single_pass_scan(x).tobytes() == scan1d_cumsum(x).tobytes()
