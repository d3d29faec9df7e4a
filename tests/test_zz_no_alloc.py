"""The allocation-free sum entry point (bh_ve_cuda_sum_f64_noalloc of libbh_ve_cuda.so).

It is compared with the existing path for the same operation: an ADD_REDUCE of a float64 array
flushed through the C bridge (bhb_ir_execute) to the `cuda` engine, whose GRID_REDUCE kernel
uses the same tile shape and order. Two calls in a row with different inputs check that the
shared static scratch (tile partials plus a completion counter) is reused correctly. Device
buffers for the new entry point come from torch, which is plumbing here only.
"""
import ctypes
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "bohrium_b200", "lib")
MAX_N = 8192 * 2048


def _noalloc():
    from bohrium_b200.runtime import load_library
    core = load_library()
    ve = ctypes.CDLL(os.path.join(LIB, "libbh_ve_cuda.so"))
    f = ve.bh_ve_cuda_sum_f64_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
    return core, f


def _engine_sum(rt, host: np.ndarray) -> float:
    import bohrium_b200 as bh
    return float(bh.array(rt, host).sum().numpy())


@pytest.mark.gpu
def test_noalloc_sum_matches_engine_on_two_calls(gpu_rt):
    import torch
    core, f = _noalloc()
    rng = np.random.default_rng(7)
    # A ragged size (last tile partial) first, then a different size and data in the second call.
    for n in (1_000_003, 3 * 2048 * 97 + 5):
        host = rng.standard_normal(n)
        expect = _engine_sum(gpu_rt, host)
        x = torch.from_numpy(host).to("cuda")
        out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        held0 = torch.cuda.memory_allocated()
        assert f(x.data_ptr(), n, out.data_ptr(), None) == 0, core.bhb_last_error()
        torch.cuda.synchronize()
        # Nothing was allocated on the device, by the entry point or on its behalf.
        assert torch.cuda.mem_get_info()[0] == free0 and torch.cuda.memory_allocated() == held0
        got = float(out.item())
        # The same tiles, order and trees as the engine's GRID_REDUCE: bit for bit its result.
        assert got == expect, (n, got, expect)
        assert abs(got - float(np.sum(host))) <= 1e-9 * np.sum(np.abs(host))


@pytest.mark.gpu
def test_noalloc_sum_edge_sizes_and_limit(gpu_rt):
    import torch
    core, f = _noalloc()
    rng = np.random.default_rng(11)
    for n in (1, 2048, MAX_N):
        host = rng.random(n)
        expect = _engine_sum(gpu_rt, host)
        x = torch.from_numpy(host).to("cuda")
        out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        assert f(x.data_ptr(), n, out.data_ptr(), None) == 0, core.bhb_last_error()
        torch.cuda.synchronize()
        got = float(out.item())
        assert got == expect, (n, got, expect)
    # Above the static scratch's capacity: rejected on the host before anything is enqueued.
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert f(out.data_ptr(), MAX_N + 1, out.data_ptr(), None) == -1
    msg = core.bhb_last_error().decode()
    assert "exceed the maximum" in msg and str(MAX_N) in msg
