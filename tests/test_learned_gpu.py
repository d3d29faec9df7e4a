"""Learned fusion end to end on the GPU: the engine records per-kernel timings, the cost model is
trained on them by the GPU kernels, and the learned engine's outputs equal the greedy engine's
bit for bit on held-out DAGs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_records_train_and_bit_identical_learned_plans(gpu_executor, tmp_path):
    from bohrium_b200 import learn
    ex = gpu_executor
    X, t = learn.collect(ex, seeds=range(6), max_elems=2e5)
    assert X.shape[0] == t.shape[0] and X.shape[0] > 50, X.shape
    assert np.isfinite(X).all() and (t > 0).all()
    model, loss = learn.train(X, t, epochs=60)
    assert np.isfinite(loss) and loss < 1.0  # standardised log-time: better than the mean
    path = str(tmp_path / "cm.bin")
    model.save(path)
    rows = learn.evaluate(ex, seeds=range(100, 104), model_path=path, max_elems=2e5, reps=2)
    assert len(rows) == 4
    for r in rows:
        assert r["identical"], r
        assert r["plain_ms"] > 0 and r["batched_ms"] > 0 and r["learned_ms"] > 0
    assert learn.summary(rows)["bit_identical"]


def test_learned_mode_without_a_model_is_the_greedy_engine(gpu_executor):
    from bohrium_b200 import learn
    ex = gpu_executor
    rt, dag, outs, _ = learn.build(ex, seed=7, max_elems=1e4)
    dag.execute()
    want = [ex.peek(o.base) for o in outs]
    ex.message("CUDA: learned on")
    try:
        dag.execute()
        got = [ex.peek(o.base) for o in outs]
    finally:
        ex.message("CUDA: learned off")
    assert all(a.tobytes() == b.tobytes() for a, b in zip(want, got))
