"""The random-DAG parity cases cover what the learned-fuser workload mixes: every element type
(float32, float64, int32) with 0, 1, 2 and 3 reductions, and transposed, reversed and broadcast
operand views beside contiguous ones. Checked on the bytecode the front end emits (no execution)."""
import numpy as np

import bohrium_b200 as bh
from bohrium_b200 import ir
from bohrium_b200.workloads import random_dag
from oracle.ve_openmp import OracleExecutor
from tests.test_random_dags_gpu import dag_case


def _forms(flush):
    forms = set()
    for ins in flush.instrs:
        for v in ins.operands[1:]:
            if v is None or v.ndim != 2:
                continue
            s0, s1 = v.stride
            if 0 in (s0, s1) and v.shape[list(v.stride).index(0)] > 1:
                forms.add("broadcast")
            elif s1 < 0:
                forms.add("reversed")
            elif s0 == 1 and s1 > 1:
                forms.add("transposed")
            elif s1 == 1:
                forms.add("contiguous")
    return forms


def test_cases_cover_types_reductions_and_view_forms():
    pairs, forms, reds = set(), set(), set()
    for k in range(24):
        nops, nelem, dt, nred = dag_case(k)
        assert 50 <= nops <= 400 and nelem <= 200_000
        pairs.add((np.dtype(dt).name, nred))
        rt = bh.Runtime(OracleExecutor(threads=1))
        _, outs = random_dag(rt, 500 + k, nops, nelem, dtype=dt, nreductions=nred)
        flush = rt.take()
        forms |= _forms(flush)
        reds |= {ins.name for ins in flush.instrs if ins.name in ir.REDUCTIONS}
        assert len(outs) == 3 + nred
    assert pairs == {(t, r) for t in ("float32", "float64", "int32") for r in range(4)}
    assert forms == {"contiguous", "transposed", "reversed", "broadcast"}, forms
    assert reds == {"ADD_REDUCE"}
