"""Host-side failure handling of the CUDA engine, with no GPU fault involved: damaged kernel cache
files are rejected before they reach the driver and the kernel is recompiled (the reference's
cache contract, ve/cuda/engine_cuda.cpp:104-132, where a cached cubin stands in for a compile);
injected NVRTC and allocation failures surface as a clean error through the C ABI and leave the
engine usable; and bounds-checked kernels compute the same results as the oracle."""
import numpy as np
import pytest

import bohrium_b200 as bh
from bohrium_b200 import workloads as W
from tests.harness import assert_close, float_tol, reduce_tol, run

pytestmark = pytest.mark.gpu


def _prog(rt):
    x = bh.array(rt, np.linspace(0.0, 3.0, 50_000))
    y = bh.sqrt(x) * 1.5 + bh.exp(-x)
    return [y.sum(), y * 2.0]


def _fresh_executor(monkeypatch, **cuda_keys):
    for k, v in cuda_keys.items():
        monkeypatch.setenv("BH_CUDA_" + k.upper(), str(v))
    return bh.NativeExecutor(stack="cuda")


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


def test_damaged_cache_files_are_rejected_and_recompiled(tmp_path, monkeypatch):
    ex = _fresh_executor(monkeypatch, cache_dir=tmp_path)
    try:
        want = run(bh.Runtime(ex), _prog)
    finally:
        ex.close()
    files = sorted(tmp_path.glob("*.cubin"))
    assert files, "the engine wrote no cache files"
    for k, f in enumerate(files):
        data = f.read_bytes()
        assert data[:8] == b"BHCUBIN1"
        if k % 3 == 0:
            f.write_bytes(data[: len(data) // 2])               # truncated
        elif k % 3 == 1:
            f.write_bytes(bytes(range(256)) * 8)                # not a cache file at all
        else:
            b = bytearray(data)
            b[len(b) // 2] ^= 0x5A                              # one damaged byte of the cubin
            f.write_bytes(bytes(b))
    ex = _fresh_executor(monkeypatch, cache_dir=tmp_path)
    try:
        got = run(bh.Runtime(ex), _prog)
        st = _stats(ex)
    finally:
        ex.close()
    assert st["disk_cache_rejected"] >= len(files), st
    for g, w in zip(got, want):
        assert np.asarray(g).tobytes() == np.asarray(w).tobytes()
    for f in tmp_path.glob("*.cubin"):
        assert f.read_bytes()[:8] == b"BHCUBIN1"  # rewritten intact


@pytest.mark.parametrize("what,msg", [("nvrtc", "injected failure"), ("alloc", "out of memory")])
def test_injected_failures_are_clean_errors(monkeypatch, what, msg):
    ex = _fresh_executor(monkeypatch, cache_dir="NONE")
    try:
        rt = bh.Runtime(ex)
        ex.message(f"CUDA: inject {what} 1")
        with pytest.raises(RuntimeError, match=msg):
            run(rt, _prog)
        ex.message(f"CUDA: inject {what} 0")
        got = run(rt, _prog)
    finally:
        ex.close()
    x = np.linspace(0.0, 3.0, 50_000)
    y = np.sqrt(x) * 1.5 + np.exp(-x)
    assert abs(float(got[0]) - y.sum()) <= 1e-12 * abs(y.sum())
    assert_close(got[1], y * 2.0, *float_tol(np.float64, True))


def test_bounds_checked_kernels_match_the_oracle(monkeypatch, oracle_rt):
    """bounds_check = true: every generated kernel checks its indices and records the first bad
    one (none here); results equal the oracle's within the usual tolerances."""
    ex = _fresh_executor(monkeypatch, bounds_check="true", cache_dir="NONE")
    try:
        gpu = bh.Runtime(ex)
        A, B, C = W.plain_chain_inputs(1 << 16, 3)
        G = W.heat_grid(98, 5)
        M = np.random.default_rng(7).random((123, 77))

        def prog(rt):
            a, b, c = (bh.array(rt, x) for x in (A, B, C))
            out = [W.plain_chain(rt, a, b, c)]
            s, d = bh.array(rt, G), bh.array(rt, G)
            out.append(W.heat_step(s, d))
            out.append(d)
            m = bh.array(rt, M)
            out += [m.sum(axis=0), m.sum(axis=1), bh.accumulate("ADD_ACCUMULATE", m[3], 0), m.T * 2.0]
            return out
        g, o = run(gpu, prog), run(oracle_rt, prog)
    finally:
        ex.close()
    tols = [reduce_tol(np.float64), 1e-6, 1e-5, reduce_tol(np.float64), reduce_tol(np.float64), 1e-12, 1e-15]
    for k, (a, b, t) in enumerate(zip(g, o, tols)):
        assert_close(a, b, t, t * 1e-2, f"output {k}")
