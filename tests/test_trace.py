"""BhIR traces (bohrium_b200/trace.py): a program recorded on one executor replays on another and
gives the same results."""
import numpy as np
import pytest

import bohrium_b200 as bh
from bohrium_b200 import trace
from tests import programs as P


def _record(path, prog):
    from oracle.ve_openmp import OracleExecutor
    rec = trace.Recorder(OracleExecutor(threads=2), path)
    rt = bh.Runtime(rec)
    outs = prog(rt)
    vals = [o.numpy() for o in outs]
    rec.close()
    return outs, vals


def _prog(rt):
    rng = np.random.default_rng(5)
    a = bh.array(rt, rng.random((40, 30)))
    b = bh.array(rt, rng.integers(0, 9, 30).astype(np.int64))
    r = bh.random123(rt, (16,), 3, 9)
    return [(a * 2.0 + b.astype(np.float64)).sum(axis=1), bh.accumulate("ADD_ACCUMULATE", b, 0), r]


def test_trace_replays_on_the_oracle(tmp_path):
    from oracle.ve_openmp import OracleExecutor
    path = str(tmp_path / "t.jsonl")
    outs, vals = _record(path, _prog)
    ex = OracleExecutor(threads=2)
    bases = trace.replay(path, ex)
    for o, v in zip(outs, vals):
        got = ex.get_data(bases[o.base.id])
        assert np.array_equal(got.reshape(v.shape), v)


@pytest.mark.gpu
def test_trace_recorded_on_the_oracle_replays_on_the_gpu(tmp_path, gpu_executor):
    path = str(tmp_path / "t.jsonl")
    outs, vals = _record(path, _prog)
    bases = trace.replay(path, gpu_executor)
    for o, v in zip(outs, vals):
        got = gpu_executor.get_data(bases[o.base.id]).reshape(v.shape)
        if v.dtype.kind in "iu":
            assert np.array_equal(got, v)
        else:
            np.testing.assert_allclose(got, v, rtol=1e-12)
