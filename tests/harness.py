"""Helpers to run one program on two runtimes and compare the results."""
from __future__ import annotations

import numpy as np


def run(rt, prog):
    outs = prog(rt)
    return [o.numpy() for o in outs]


def assert_close(got, want, rtol, atol=0.0, what=""):
    got = np.asarray(got)
    want = np.asarray(want)
    assert got.shape == want.shape, f"{what}: shape {got.shape} != {want.shape}"
    assert got.dtype == want.dtype, f"{what}: dtype {got.dtype} != {want.dtype}"
    if got.dtype.kind in "biu":
        bad = np.flatnonzero(got.reshape(-1) != want.reshape(-1))
        assert bad.size == 0, f"{what}: {bad.size} integer mismatches, first at {bad[:5]}: " \
                              f"{got.reshape(-1)[bad[:5]]} vs {want.reshape(-1)[bad[:5]]}"
    else:
        np.testing.assert_allclose(got, want, rtol=rtol, atol=atol, equal_nan=True, err_msg=what)


def float_tol(dtype, transcendental=False):
    """Tolerances for elementwise floating-point results of the CUDA engine vs the CPU oracle:
    a few ulps (CUDA's and glibc's math functions, and FMA contraction on the CPU side)."""
    if np.dtype(dtype) == np.float32:
        return (1e-5, 1e-6) if transcendental else (1e-6, 1e-7)
    return (1e-12, 1e-14) if transcendental else (1e-14, 1e-15)


def reduce_tol(dtype):
    """Reductions change summation order: 1e-5 relative for float32, 1e-12 for float64."""
    return 1e-5 if np.dtype(dtype) == np.float32 else 1e-12


def compare(a_results, b_results, tol=None, what=""):
    assert len(a_results) == len(b_results)
    for k, (x, y) in enumerate(zip(a_results, b_results)):
        if tol is None:
            rtol, atol = float_tol(np.asarray(y).dtype)
        else:
            rtol, atol = tol
        assert_close(x, y, rtol, atol, f"{what}[{k}]")


def grid_reduce_sum(x: np.ndarray) -> np.ndarray:
    """Exact model of the summation order of the engine's GRID_REDUCE schedule for an ADD_REDUCE
    of a contiguous 1-D array: tiles of 256 threads x 8 elements (thread t adds elements
    4t, 4t+1, 4t+2, 4t+3, 1024+4t, ..., 1024+4t+3 of its tile in order, starting from 0 -- two
    128-bit words' worth), a halving tree over the 32 lanes of each warp and over the 8 warp sums
    (padded with 0), then the same per-thread fold and trees over the tile partials (thread t adds
    partials t, t+256, ...). Vectorised NumPy in the array's own dtype, so the result is
    bit-exact."""
    dt = x.dtype
    zero = dt.type(0)
    n = x.size
    ntiles = -(-n // 2048)
    pad = np.zeros(ntiles * 2048, dtype=dt)
    pad[:n] = x
    t = pad.reshape(ntiles, 2, 256, 4)
    acc = np.full((ntiles, 256), zero, dtype=dt)
    for j in range(8):
        acc = acc + t[:, j >> 2, :, j & 3]

    def cta_tree(a):  # a: (rows, 256) -> (rows,)
        w = a.reshape(a.shape[0], 8, 32)
        for m in (16, 8, 4, 2, 1):
            w = w[:, :, :m] + w[:, :, m:2 * m]
        ws = np.full((a.shape[0], 32), zero, dtype=dt)
        ws[:, :8] = w[:, :, 0]
        for m in (16, 8, 4, 2, 1):
            ws = ws[:, :m] + ws[:, m:2 * m]
        return ws[:, 0]

    parts = cta_tree(acc)
    fold = np.full(256, zero, dtype=dt)
    for start in range(0, ntiles, 256):
        chunk = np.full(256, zero, dtype=dt)
        c = parts[start:start + 256]
        chunk[:c.size] = c
        fold = np.where(np.arange(256) < c.size, fold + chunk, fold)
    return cta_tree(fold[None, :])[0]


def _block_scan(s: np.ndarray):
    """The engine's block scan of the 256 thread values of each row of `s` (rows, 256): an
    inclusive shuffle-up scan in each warp (x = y + x for lanes >= d, d = 1..16), shifted by one
    lane, plus the warp offsets from a serial scan of the 8 warp totals. Returns the exclusive
    prefixes (rows, 256) and the row totals."""
    dt = s.dtype
    zero = dt.type(0)
    w = s.reshape(s.shape[0], 8, 32).copy()
    lane = np.arange(32)
    for d in (1, 2, 4, 8, 16):
        y = w.copy()
        y[:, :, d:] = w[:, :, :-d]
        w = np.where(lane >= d, y + w, w)
    ex = np.full_like(w, zero)
    ex[:, :, 1:] = w[:, :, :-1]
    run = np.full(s.shape[0], zero, dtype=dt)
    wo = np.empty((s.shape[0], 8), dtype=dt)
    for k in range(8):
        wo[:, k] = run
        run = run + w[:, k, 31]
    return (wo[:, :, None] + ex).reshape(s.shape[0], 256), run


def scan1d_cumsum(x: np.ndarray) -> np.ndarray:
    """Exact model of the addition order of the engine's SCAN1D schedule for an ADD_ACCUMULATE of
    a contiguous 1-D array. Chunks of 2048 elements; thread t of a chunk folds elements 8t..8t+7
    in order from 0, a block scan of the 256 thread sums gives each thread's exclusive prefix e and
    the chunk total. One CTA scans the chunk totals the same way, 2048 at a time with a running
    carry, into the carry of every chunk. Element 8t+k of a chunk is then
    carry + (e + (x[8t] + ... + x[8t+k])). Vectorised NumPy in the array's own dtype, so the
    result is bit-exact."""
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
    carries = np.empty(nch, dtype=dt)
    run = zero
    for base in range(0, nch, 2048):
        cnt = min(2048, nch - base)
        g = np.zeros(2048, dtype=dt)
        g[:cnt] = totals[base:base + cnt]
        gv = g.reshape(256, 8)
        ok = (np.arange(2048) < cnt).reshape(256, 8)
        v = np.empty((256, 8), dtype=dt)
        acc = np.full(256, zero, dtype=dt)
        for k in range(8):
            v[:, k] = acc
            acc = np.where(ok[:, k], acc + gv[:, k], acc)
        ge, gt = _block_scan(acc[None, :])
        carries[base:base + cnt] = (run + (ge[0][:, None] + v)).reshape(-1)[:cnt]
        run = run + gt[0]
    out = np.empty((nch, 256, 8), dtype=dt)
    r = np.full((nch, 256), zero, dtype=dt)
    for k in range(8):
        r = np.where(valid[:, :, k], r + xs[:, :, k], r)
        out[:, :, k] = carries[:, None] + (e + r)
    return out.reshape(-1)[:n]


# ----------------------------------------------------------------------------- error bounds
# Unit roundoffs of float32 and float64.
U32 = 2.0 ** -24
U64 = 2.0 ** -53


def gamma(d, u):
    """gamma_d = d u / (1 - d u): a sum whose every input passes through at most d roundings
    differs from the exact sum by at most gamma_d * sum(|x|), whatever the order of the additions
    (N. J. Higham, Accuracy and Stability of Numerical Algorithms, 2nd ed., sec. 4.2)."""
    d = np.asarray(d, dtype=np.float64)
    return d * u / (1.0 - d * u)


def scan1d_depth(n: int) -> int:
    """Roundings on the way from any input element to any output of the engine's SCAN1D schedule
    (see `scan1d_cumsum`), at most: 8 in the thread's run, 5 in the warp scan and 8 over the warp
    totals of the chunk, the same 8 + 5 + 8 again over the chunk totals of a group, one per group
    carry, and 3 to combine carry, thread prefix and run -- 45 plus the number of groups, taken
    as 48 plus the groups."""
    chunks = -(-n // 2048)
    groups = -(-chunks // 2048)
    return 48 + groups


def assert_cumsum_within_bound(got, x, depth, u, what=""):
    """Every output of a cumulative sum of the 1-D `x` is within gamma_depth(i) * sum_{j<=i} |x_j|
    of the exact prefix sum (float64, or complex128 component by component; exact enough next to
    a float32 bound). `depth` is a number or one per output."""
    x = np.asarray(x)
    got = np.asarray(got)
    parts = [(np.real, "re"), (np.imag, "im")] if np.iscomplexobj(x) else [(lambda a: a, "")]
    for f, nm in parts:
        xv = f(x).astype(np.float64)
        gv = f(got).astype(np.float64)
        exact = np.cumsum(xv)
        bound = gamma(depth, u) * np.cumsum(np.abs(xv))
        over = np.abs(gv - exact) - bound
        assert over.max(initial=-1.0) <= 0.0, f"{what} {nm}: worst excess over the bound {over.max():.3g} " \
                                              f"at {int(np.argmax(over))}"


def assert_cumprod_within_bound(got, x, u, per_mult=3.0, what=""):
    """Every output of a cumulative product of the 1-D `x` is within ((1 + c u)^i - 1) |p_i| of
    the exact prefix product p_i (complex128), whatever the order of the multiplications: each
    product of i factors takes at most i - 1 multiplications by something other than 1, and each
    complex multiplication errs by at most sqrt(5) u relative (Brent, Percival and Zimmermann,
    Math. Comp. 76, 2007); c = 3 also covers a multiply-add contracted product."""
    x = np.asarray(x).astype(np.complex128 if np.iscomplexobj(x) else np.float64)
    got = np.asarray(got).astype(x.dtype)
    exact = np.cumprod(x)
    i = np.arange(1, x.size + 1, dtype=np.float64)
    bound = np.expm1(i * np.log1p(per_mult * u)) * np.abs(exact)
    over = np.abs(got - exact) - bound
    assert over.max(initial=-1.0) <= 0.0, f"{what}: worst excess over the bound {over.max():.3g} at {int(np.argmax(over))}"
