"""User kernels with no GPU: the front end's checks and parameter string (the reference's
bridge/npbackend/bohrium/user_kernel.py:21-150), and the reference's openmp user-kernel test on
the oracle. The CUDA kernels run in tests/test_user_kernel_gpu.py."""
import numpy as np
import pytest

import bohrium_b200 as bh
from bohrium_b200.array import _param_string


def _rt():
    return bh.Runtime(bh.DryRunExecutor())


def test_behaving_arrays():
    rt = _rt()
    a = bh.empty(rt, (110,), np.float64)
    assert bh.is_behaving(a)
    assert not bh.is_behaving(a[10:])        # offset into its base
    assert not bh.is_behaving(a[:100])       # shorter than its base
    m = bh.empty(rt, (20, 5), np.float64)
    assert bh.is_behaving(m) and not bh.is_behaving(m.T)
    b = bh.make_behaving(a[10:])
    assert bh.is_behaving(b) and b.shape == (100,) and b.base is not a.base
    assert bh.make_behaving(a) is a


def test_non_behaving_operands_are_rejected_before_any_call():
    rt = _rt()
    a = bh.empty(rt, (110,), np.float64)
    with pytest.raises(TypeError, match="not behaving"):
        bh.user_kernel("", [a[10:]], tag="cuda")
    with pytest.raises(TypeError, match="Bohrium arrays"):
        bh.user_kernel("", [np.ones(3)], tag="cuda")
    with pytest.raises(ValueError):
        bh.user_kernel("", [], tag="cuda")


def test_param_string_matches_the_reference_front_end():
    assert _param_string({"global_work_size": (20, 5), "local_work_size": (1, 1)}) == \
        "global_work_size: 20 5; local_work_size: 1 1"
    assert _param_string({"global_work_size": 1024, "local_work_size": [128]}) == \
        "global_work_size: 1024; local_work_size: 128"
    assert _param_string(None) == ""


def test_openmp_user_kernel_on_the_oracle(oracle_rt):
    """The reference's own openmp user-kernel test (test/python/tests/test_user_kernel.py) on the
    oracle's restatement of ve/openmp's userKernel."""
    kernel = r"""
#include <stdint.h>
void execute(double *a, double *b, double *c) {
    for (uint64_t i = 0; i < 100; ++i) {
        c[i] = a[i] + b[i] + i;
    }
}
"""
    a = bh.ones(oracle_rt, (100,), np.float64)
    b = bh.make_behaving(bh.ones(oracle_rt, (110,), np.float64)[10:])
    res = bh.empty(oracle_rt, (100,), np.float64)
    bh.user_kernel(kernel, [a, b, res])
    np.testing.assert_array_equal(res.numpy(), 2.0 + np.arange(100))
    with pytest.raises(RuntimeError, match="compilation failed"):
        bh.user_kernel("void execute(double *a) { a[0] = ; }", [a])
