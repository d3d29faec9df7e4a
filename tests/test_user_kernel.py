"""User kernels: the front end's checks and parameter string, with no GPU (the reference's
bridge/npbackend/bohrium/user_kernel.py:21-150). The kernels themselves run in
tests/test_user_kernel_gpu.py."""
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
