"""Grouped launches of a replayed flush keep their parameter blocks on the device and launch them
again, without packing or copying, while no buffer changed; a changed input buffer makes them
repack. The results equal those of plain launches bit for bit throughout."""
import numpy as np
import pytest

import bohrium_b200 as bh
from bohrium_b200 import workloads as W

pytestmark = pytest.mark.gpu


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


def test_grouped_replays_reuse_parameter_blocks_until_a_buffer_changes():
    ex = bh.NativeExecutor(stack="cuda")
    try:
        rt = bh.Runtime(ex)
        rng = np.random.default_rng(3)
        data = [rng.random(n, dtype=np.float32) for n in (1000, 5000, 70000, 3000, 257)]
        xs = [bh.array(rt, d) for d in data]
        rt.flush()
        outs = []
        for x in xs:
            y = W.batching_chain(x)
            outs += [y, y.sum(), y.max()]
        ir = ex.compile(rt.take())

        def results():
            return [ex.peek(o.base).tobytes() for o in outs]
        ex.message("CUDA: batch off")
        ir.execute()
        want = results()
        ex.message("CUDA: batch grouped")
        r0 = _stats(ex).get("pack_reuses", 0)
        for _ in range(5):
            ir.execute()
        assert _stats(ex)["pack_reuses"] >= r0 + 3
        assert results() == want
        # New data in one input: its buffer changes, the blocks are packed again.
        ex.set_data(xs[2].base, rng.random(70000, dtype=np.float32))
        ir.execute()
        ir.execute()
        got = results()
        assert got[6] != want[6] and got[0] == want[0]
        ex.message("CUDA: batch off")
        ir.execute()
        assert results() == got
        del ir, outs, xs
    finally:
        ex.close()
