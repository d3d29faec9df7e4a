"""BhIR traces: record the flushes a program sends to a stack and replay them elsewhere.

The reference serialises a BhIR with Boost (core/bh_ir.cpp:37-154) for trace replay and cross-
process reuse. Here a trace is a JSON-lines file, one record per event:

    {"base": id, "dtype": "float64", "nelem": n}                  a base array the program created
    {"data": id, "values": [...]}                                  host data handed to the stack
    {"flush": [instr, ...], "syncs": [id, ...], "nrepeats": r, "condition": id | null}
        instr = {"op": opcode, "operands": [null | [id, start, [shape], [stride]]],
                 "constant": null | [value, bh_type], "slides": {operand: [[slide...], {dim: max}]}}

`Recorder(executor)` wraps any executor (the native stack, the oracle) and writes the trace while
forwarding every call; `replay(path, executor)` registers the bases, hands over the recorded data
and executes the flushes in order, returning the bases by id so the caller can read results.
"""
from __future__ import annotations

import json

import numpy as np

from . import ir


def _view(v):
    if v is None:
        return None
    return [v.base.id, int(v.start), [int(s) for s in v.shape], [int(s) for s in v.stride]]


def _constant(c):
    if c is None:
        return None
    if c.dtype == ir.R123:
        return [[int(c.value[0]), int(c.value[1])], c.dtype]
    v = np.asarray(c.value).item()
    if isinstance(v, complex):
        v = [v.real, v.imag]
    return [v, c.dtype]


def _slides(ins):
    out = {}
    for o, (dims, resets) in ins.slides.items():
        out[str(o)] = [[[d.rank, d.offset_change, d.shape_change, d.stride, d.shape, d.step_delay] for d in dims],
                       {str(k): int(v) for k, v in resets.items()}]
    return out


class Recorder:
    """Executor wrapper that writes a trace of everything it forwards."""

    def __init__(self, executor, path: str, with_data: bool = True):
        self.ex = executor
        self.f = open(path, "w")
        self.with_data = with_data

    def close(self):
        self.f.close()

    def _write(self, rec):
        self.f.write(json.dumps(rec) + "\n")

    def register(self, base):
        self.ex.register(base)
        self._write({"base": base.id, "dtype": base.dtype.name, "nelem": base.nelem})

    def release(self, base):
        self.ex.release(base)

    def set_data(self, base, data):
        self.ex.set_data(base, data)
        if self.with_data:
            self._write({"data": base.id, "values": np.asarray(data).reshape(-1).tolist()})

    def get_data(self, base):
        return self.ex.get_data(base)

    def execute(self, flush):
        self._write({"flush": [{"op": int(i.opcode), "operands": [_view(v) for v in i.operands],
                                "constant": _constant(i.constant), "slides": _slides(i)} for i in flush.instrs],
                     "syncs": [b.id for b in flush.syncs], "nrepeats": int(flush.nrepeats),
                     "condition": flush.condition.id if flush.condition is not None else None})
        self.ex.execute(flush)

    def __getattr__(self, name):  # message, compile, extmethod, ...
        return getattr(self.ex, name)


def _decode_constant(c):
    if c is None:
        return None
    value, t = c
    if t == ir.R123:
        return ir.Constant(tuple(value), t)
    if isinstance(value, list):
        value = complex(value[0], value[1])
    return ir.Constant(value, t)


def replay(path: str, executor) -> dict:
    """Execute a recorded trace on `executor`; returns {recorded base id: Base}."""
    bases = {}
    with open(path) as f:
        for line in f:
            rec = json.loads(line)
            if "base" in rec:
                b = ir.Base(rec["dtype"], rec["nelem"])
                executor.register(b)
                bases[rec["base"]] = b
            elif "data" in rec:
                b = bases[rec["data"]]
                executor.set_data(b, np.asarray(rec["values"], dtype=b.dtype))
            elif "flush" in rec:
                instrs = []
                for i in rec["flush"]:
                    ops = [None if v is None else ir.View(bases[v[0]], v[1], tuple(v[2]), tuple(v[3]))
                           for v in i["operands"]]
                    slides = {}
                    for o, (dims, resets) in i.get("slides", {}).items():
                        slides[int(o)] = ([ir.Slide(*d) for d in dims], {int(k): v for k, v in resets.items()})
                    instrs.append(ir.Instr(i["op"], ops, _decode_constant(i["constant"]), slides))
                cond = bases[rec["condition"]] if rec["condition"] is not None else None
                executor.execute(ir.Flush(instrs, [bases[s] for s in rec["syncs"]], rec["nrepeats"], cond))
    return bases
