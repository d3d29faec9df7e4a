"""User kernels with tag "cuda" on the engine: the reference's own user-kernel tests
(test/python/tests/test_user_kernel.py: a 1-D add of an offset-copied operand, and the OpenCL
engine's 2-D form with global/local work sizes) written as CUDA kernels, with NumPy as the witness,
plus the error messages for sources and parameters the engine refuses. Every kernel here guards
or exactly covers its arrays' bounds."""
import numpy as np
import pytest

import bohrium_b200 as bh

pytestmark = pytest.mark.gpu

ADD_1D = r"""
extern "C" __global__ void execute(const double *a, const double *b, double *c) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 100) c[i] = a[i] + b[i] + i;
}
"""

ADD_2D = r"""
extern "C" __global__ void execute(const double *a, const double *b, double *c) {
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
    const int i1 = blockIdx.y * blockDim.y + threadIdx.y;
    const int gid = i0 * 5 + i1;
    c[gid] = a[gid] + b[gid] + gid;
}
"""


def test_add_one_dimensional(gpu_rt):
    a = bh.ones(gpu_rt, (100,), np.float64)
    b = bh.make_behaving(bh.ones(gpu_rt, (110,), np.float64)[10:])
    res = bh.empty(gpu_rt, (100,), np.float64)
    bh.user_kernel(ADD_1D, [a, b, res], tag="cuda", param={"global_work_size": 128, "local_work_size": 64})
    np.testing.assert_array_equal(res.numpy(), 2.0 + np.arange(100))


def test_add_two_dimensional_work_sizes(gpu_rt):
    a = bh.ones(gpu_rt, (20, 5), np.float64)
    b = bh.make_behaving(bh.ones(gpu_rt, (21, 5), np.float64)[1:, :])
    res = bh.empty(gpu_rt, (20, 5), np.float64)
    bh.user_kernel(ADD_2D, [a, b, res], tag="cuda",
                   param={"global_work_size": (20, 5), "local_work_size": (1, 1)})
    np.testing.assert_array_equal(res.numpy(), 2.0 + np.arange(100).reshape(20, 5))


def test_result_feeds_later_bytecode_and_source_is_cached(gpu_rt):
    """The kernel's output stays on the device for the next flush, and its inputs may come from
    bytecode flushed just before it; a second call reuses the compiled function."""
    host = np.random.default_rng(0).random(100)
    a = bh.array(gpu_rt, host) * 3.0
    b = bh.zeros(gpu_rt, (100,), np.float64)
    res = bh.empty(gpu_rt, (100,), np.float64)
    for _ in range(2):
        bh.user_kernel(ADD_1D, [a, b, res], tag="cuda", param={"global_work_size": 100, "local_work_size": 50})
        total = (res * 2.0).sum().numpy()
        np.testing.assert_allclose(total, np.sum((host * 3.0 + np.arange(100)) * 2.0), rtol=1e-12)


@pytest.mark.parametrize("src,param,match", [
    ("extern \"C\" __global__ void execute(double *a) { a[0] = ; }",
     {"global_work_size": 1, "local_work_size": 1}, "compilation failed"),
    ("extern \"C\" __global__ void run(double *a) { }",
     {"global_work_size": 1, "local_work_size": 1}, "named execute"),
    (ADD_1D, {"global_work_size": (128, 1), "local_work_size": 64}, "must be the same"),
    (ADD_1D, {"global_work_size": 100, "local_work_size": 64}, "multiple of local_work_size"),
    (ADD_1D, {}, "maximum of three dimensions"),
    (ADD_1D, {"global_work_size": 2048, "local_work_size": 2048}, "limits"),
])
def test_refused_kernels_return_the_engine_message(gpu_rt, src, param, match):
    """Nothing is launched in these cases: the engine returns its message and the front end
    raises it, as the reference's does."""
    a = bh.zeros(gpu_rt, (100,), np.float64)
    with pytest.raises(RuntimeError, match=match):
        bh.user_kernel(src, [a, a, a] if src is ADD_1D else [a], tag="cuda", param=param)
