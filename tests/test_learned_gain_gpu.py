"""The learned engine against the greedy fuser it steers (core/jitk/graph.cpp:319-365, the
reference's greedy contraction), on held-out DAGs of the learned-fuser workload. The model is
trained here on this engine's own timings of other DAGs. The learned engine builds a learned plan
for every DAG (the model predicts the merges), times it against the greedy plan and keeps it
only when it is faster (by at least 3 %), so over the held-out set it is never slower than greedy
batching (within timing noise), any plan it keeps is faster there, and its outputs equal the
greedy plan's bit for bit. (How much it gains is measured by bench.py's
learned_fuser_random_dags, with a larger training set; a model trained on eight small DAGs, as
here, keeps few or no learned plans.)"""
import numpy as np
import pytest

from bohrium_b200 import learn

pytestmark = pytest.mark.gpu

# Held-out DAGs (learn.dag_params at max_elems 4e6): six int32 DAGs with two reductions and
# 3e5-1.8e6 elements, and six DAGs of any kind.
INT32_TWO_REDUCTIONS = [2012, 2030, 2094, 2129, 2138, 2343]
OTHERS = [3000, 3001, 3002, 3003, 3004, 3005]


def test_learned_engine_gains_on_held_out_dags(gpu_executor, tmp_path):
    for s in INT32_TWO_REDUCTIONS:
        _, nelem, dt, nred = learn.dag_params(s, 4e6)
        assert dt is np.int32 and nred == 2 and nelem >= 3e5
    X, t = learn.collect(gpu_executor, seeds=range(1000, 1008), max_elems=2e6)
    model, _ = learn.train(X, t, epochs=200)
    path = str(tmp_path / "costmodel.bin")
    model.save(path)
    p0 = learn._stats(gpu_executor).get("learned_predictions", 0)
    rows = learn.evaluate(gpu_executor, INT32_TWO_REDUCTIONS + OTHERS, path, max_elems=4e6, reps=5)
    predictions = learn._stats(gpu_executor).get("learned_predictions", 0) - p0
    table = [(r["seed"], round(r["batched_ms"], 4), round(r["learned_ms"], 4), r["tried"], r["learned_kept"])
             for r in rows]
    assert all(r["identical"] for r in rows), table
    assert predictions > 0, table  # the model steered the contraction
    batched = sum(r["batched_ms"] for r in rows)
    learned = sum(r["learned_ms"] for r in rows)
    assert learned <= 1.05 * batched, table
    kept = [r for r in rows if r["learned_kept"] > 0]
    if kept:
        assert sum(r["learned_ms"] for r in kept) <= 1.02 * sum(r["batched_ms"] for r in kept), table
