"""Restatement of the reference fuser (core/jitk) for the CPU oracle -- test infrastructure.

Follows core/jitk/fuser.cpp:35-249 (simplify_instr, simplify_instr_list, pre_fuser_lossy),
core/jitk/graph.cpp:52-365 (block DAG, greedy contraction by eliminated temporary bytes),
core/jitk/block.cpp:37-693 (loop blocks, mergeable, reshape_and_merge), core/jitk/transformer.cpp:
165-246 (collapse_redundant_axes) and core/jitk/apply_fusion.cpp:87-259 (identity blocks, kernel
list), with the configuration of the reference's OpenMP engine: fuser_list = greedy,
collapse_redundant_axes and avoid_rank0_sweep = false (config.ini.in:106-110, engine_cpu.hpp:41).
"""
from __future__ import annotations

import copy
from collections import deque
from typing import Optional

from bohrium_b200 import ir as _ir

OP = _ir.OPCODES
REDUCE_OPS = {OP[k] for k in _ir.REDUCTIONS}
ACCUM_OPS = {OP[k] for k in _ir.ACCUMULATES}
SWEEP_OPS = REDUCE_OPS | ACCUM_OPS
SYSTEM_OPS = {OP["FREE"], OP["NONE"], OP["TALLY"]}
MAXDIM = 16


# ---------------------------------------------------------------------------------------- views
class V:
    __slots__ = ("base", "start", "shape", "stride")

    def __init__(self, base, start, shape, stride):
        self.base, self.start, self.shape, self.stride = base, start, list(shape), list(stride)

    @property
    def ndim(self):
        return len(self.shape)

    def key(self):
        return (self.base.id, self.start, tuple(self.shape), tuple(self.stride))

    def prod(self):
        p = 1
        for s in self.shape:
            p *= s
        return p

    def is_scalar(self):
        return self.prod() == 1

    def is_contiguous(self):
        w = 1
        for d in range(self.ndim - 1, -1, -1):
            if self.shape[d] > 1 and self.stride[d] != w:
                return False
            w *= self.shape[d]
        return True

    def remove_axis(self, d):
        del self.shape[d]
        del self.stride[d]

    def insert_axis(self, d, size, stride):
        self.shape.insert(d, size)
        self.stride.insert(d, stride)

    def transpose(self, a, b):
        self.shape[a], self.shape[b] = self.shape[b], self.shape[a]
        self.stride[a], self.stride[b] = self.stride[b], self.stride[a]

    def clone(self):
        return V(self.base, self.start, self.shape, self.stride)


# --------------------------------------------------------------------------------- instructions
class I:
    __slots__ = ("opcode", "ops", "const", "constructor", "origin_id")

    def __init__(self, opcode, ops, const=None, constructor=False, origin_id=-1):
        self.opcode, self.ops, self.const = opcode, ops, const
        self.constructor, self.origin_id = constructor, origin_id

    def clone(self):
        return I(self.opcode, [o.clone() if o is not None else None for o in self.ops],
                 copy.copy(self.const), self.constructor, self.origin_id)

    def views(self):
        return [o for o in self.ops if o is not None]

    def bases(self):
        out = []
        for v in self.views():
            if v.base not in out:
                out.append(v.base)
        return out

    def same(self, other):
        if self.opcode != other.opcode or len(self.ops) != len(other.ops):
            return False
        for a, b in zip(self.ops, other.ops):
            if (a is None) != (b is None):
                return False
            if a is None:
                if self.const != other.const:
                    return False
            elif a.key() != b.key():
                return False
        return True

    def is_system(self):
        return self.opcode in SYSTEM_OPS

    def shape(self):
        if self.opcode in SWEEP_OPS:
            return list(self.ops[1].shape)
        if self.opcode in (OP["GATHER"], OP["SCATTER"], OP["COND_SCATTER"]):
            return list(self.ops[2].shape)
        if not self.ops:
            return []
        return list(self.ops[0].shape)

    def ndim(self):
        return len(self.shape())

    def sweep_axis(self):
        return int(self.const[0]) if self.opcode in SWEEP_OPS else MAXDIM

    def all_same_shape(self):
        if not self.ops:
            return True
        first = self.ops[0]
        return all(v.shape == first.shape for v in self.ops[1:] if v is not None)

    def reshapable(self):
        return self.all_same_shape() and all(v.is_contiguous() for v in self.views()) and \
            self.opcode not in SWEEP_OPS

    def reshape(self, shape):
        for v in self.views():
            v.shape = list(shape)
            s, st = 1, []
            for n in reversed(shape):
                st.append(s)
                s *= n
            v.stride = list(reversed(st))

    def remove_axis(self, axis):
        if not self.ops:
            return
        for o in range(1, len(self.ops)):
            if self.ops[o] is not None and not (o == 1 and self.opcode == OP["GATHER"]):
                self.ops[o].remove_axis(axis)
        sa = self.sweep_axis()
        if sa > axis and sa < MAXDIM:
            self.const = (sa - 1, self.const[1])
        if self.opcode in (OP["SCATTER"], OP["COND_SCATTER"]):
            return
        if self.opcode in REDUCE_OPS:
            self.ops[0].remove_axis(axis - 1 if sa < axis else axis)
        else:
            self.ops[0].remove_axis(axis)


def simplify(instr: I):
    """Drop size-1 axes, then flatten reshapable instructions (core/jitk/fuser.cpp:35-60)."""
    if not instr.ops:
        return
    shape = instr.shape()
    sa = instr.sweep_axis()
    left = len(shape) - 1 if instr.opcode in REDUCE_OPS else len(shape)
    for i in range(len(shape) - 1, -1, -1):
        if left <= 1:
            break
        if sa != i and shape[i] == 1:
            instr.remove_axis(i)
            left -= 1
    if instr.ndim() > 1 and instr.reshapable():
        n = 1
        for s in instr.shape():
            n *= s
        instr.reshape([n])


def reshape_rank(instr: I, rank: int, size: int) -> I:
    shape = [instr.ops[0].shape[r] for r in range(rank)] + [size]
    total = 1
    for r in range(rank, instr.ops[0].ndim):
        total *= instr.ops[0].shape[r]
    if total != size:
        shape.append(total // size)
    out = instr.clone()
    out.reshape(shape)
    return out


# ---------------------------------------------------------------------------------------- blocks
class IB:
    __slots__ = ("instr", "rank")

    def __init__(self, instr, rank):
        self.instr, self.rank = instr, rank


class Loop:
    def __init__(self, rank, size, items=None):
        self.rank, self.size = rank, size
        self.items = items if items is not None else []
        self.sweeps: list = []
        self.news: set = set()      # base ids created by local instructions
        self.frees: dict = {}       # base id -> Base
        self.reshapable = False

    def clone(self):
        c = Loop(self.rank, self.size, [it.clone() if isinstance(it, Loop) else IB(it.instr, it.rank)
                                        for it in self.items])
        c.sweeps, c.news, c.frees, c.reshapable = list(self.sweeps), set(self.news), dict(self.frees), self.reshapable
        return c

    def all_instr(self, out=None):
        out = [] if out is None else out
        for it in self.items:
            if isinstance(it, Loop):
                it.all_instr(out)
            else:
                out.append(it.instr)
        return out

    def local_instr(self):
        return [it.instr for it in self.items if isinstance(it, IB)]

    def subloops(self):
        return [it for it in self.items if isinstance(it, Loop)]

    def is_system_only(self):
        return all(it.is_system_only() if isinstance(it, Loop) else it.instr.is_system() for it in self.items)

    def is_innermost(self):
        return all(isinstance(it, IB) for it in self.items)

    def all_news(self):
        s = set(self.news)
        for l in self.subloops():
            s |= l.all_news()
        return s

    def all_frees(self):
        d = dict(self.frees)
        for l in self.subloops():
            d.update(l.all_frees())
        return d

    def local_temps(self):
        frees = self.all_frees()
        news = self.all_news()
        return {b for b in self.news if b in frees} | {b for b in self.frees if b in news}

    def all_temps(self):
        s = self.local_temps()
        for l in self.subloops():
            s |= l.all_temps()
        return s

    def all_bases(self):
        out = {}
        for i in self.all_instr():
            for b in i.bases():
                out[b.id] = b
        return out

    def update(self):
        """metadataUpdate(): news, sweeps and the reshapable flag (core/jitk/block.cpp:341-355)."""
        self.news = {i.ops[0].base.id for i in self.local_instr() if i.constructor}
        alli = self.all_instr()
        self.sweeps = [i for i in alli if i.sweep_axis() == self.rank]
        self.reshapable = _reshapable(alli)

    def local_threading(self):
        return self.size if not self.sweeps and not self.is_system_only() else 0


def _reshapable(instrs):
    if not instrs:
        return True
    nd = instrs[0].ndim()
    return all(i.reshapable() and i.ndim() == nd for i in instrs)


def nested(instrs, rank=0, frees=None) -> Loop:
    """create_nested_block(instrs, rank, frees) (core/jitk/block.cpp:425-453)."""
    shape = instrs[0].shape()
    ndim = len(shape)
    loop = Loop(rank, shape[rank])
    if rank == ndim - 1:
        loop.frees = dict(frees or {})
        for i in instrs:
            if i.opcode == OP["FREE"]:
                loop.frees[i.ops[0].base.id] = i.ops[0].base
            else:
                loop.items.append(IB(i, ndim))
    else:
        loop.items.append(nested(instrs, rank + 1, frees))
    loop.update()
    return loop


def nested_sized(instrs, rank, size) -> Loop:
    """create_nested_block(instrs, rank, size_of_rank_dim) (core/jitk/block.cpp:455-468)."""
    loop = Loop(rank, size)
    for i in instrs:
        if i.reshapable() and i.ops[0].shape[rank] != size:
            i = reshape_rank(i, rank, size)
        shape = i.shape()
        if len(shape) > rank + 1:
            loop.items.append(nested_sized([i], rank + 1, shape[rank + 1]))
        elif i.opcode == OP["FREE"]:
            loop.frees[i.ops[0].base.id] = i.ops[0].base
        else:
            loop.items.append(IB(i, rank + 1))
        loop.update()
    return loop


def parallel_ranks(loop: Loop, max_depth=3):
    thds = loop.local_threading()
    if thds == 0:
        return 0
    n = 1
    max_depth -= 1
    if max_depth > 0 and len(loop.subloops()) == 1 and not loop.local_instr():
        n += parallel_ranks(loop.items[0], max_depth)
    return n


def first_loops(loop: Loop):
    out = [loop]
    while loop.items and isinstance(loop.items[0], Loop):
        loop = loop.items[0]
        out.append(loop)
    return out


def _dp_view(w: V, r: V):
    if w is None or r is None or w.base is not r.base:
        return True
    if w.start != r.start:
        return False
    if w.ndim == r.ndim:
        return w.shape == r.shape and w.stride == r.stride
    return w.prod() == r.prod() and w.is_contiguous() and r.is_contiguous()


def _dp_instr(a: I, b: I):
    if a.is_system() or b.is_system():
        return True
    if b.opcode == OP["GATHER"] and a.ops[0].base is b.ops[1].base:
        return False
    if a.opcode in (OP["SCATTER"], OP["COND_SCATTER"]):
        if any(v is not None and a.ops[0].base is v.base for v in b.ops):
            return False
    elif b.opcode in (OP["SCATTER"], OP["COND_SCATTER"]):
        if any(v is not None and b.ops[0].base is v.base for v in a.ops):
            return False
    return all(_dp_view(a.ops[0], v) for v in b.ops) and all(_dp_view(b.ops[0], v) for v in a.ops)


def mergeable(l1, l2, avoid_rank0_sweep=False):
    """core/jitk/block.cpp:662-693."""
    if not isinstance(l1, Loop) or not isinstance(l2, Loop) or isinstance(l1, _InstrHolder) or \
            isinstance(l2, _InstrHolder):
        return False
    if l2.is_system_only():
        return True
    if avoid_rank0_sweep and l1.rank == 0 and l2.rank == 0 and bool(l1.sweeps) != bool(l2.sweeps):
        return False
    if l1.sweeps:
        b2 = l2.all_bases()
        if any(s.ops[0].base.id in b2 for s in l1.sweeps):
            return False
    if l1.size == l2.size or (l2.reshapable and l1.size and l2.size % l1.size == 0) or \
            (l1.reshapable and l2.size and l1.size % l2.size == 0):
        i1s, i2s = l1.all_instr(), l2.all_instr()
        return all(_dp_instr(a, b) for a in i1s for b in i2s if a is not b)
    return False


def _merge(l1: Loop, l2: Loop) -> Loop:
    r = Loop(l1.rank, l1.size, [*l1.items, *l2.items])
    r.sweeps = l1.sweeps + [s for s in l2.sweeps if s not in l1.sweeps]
    r.news = l1.news | l2.news
    r.frees = {**l1.frees, **l2.frees}
    r.reshapable = _reshapable(r.all_instr())
    return r


def _reshape_loop(l: Loop, size: int) -> Loop:
    instrs = [reshape_rank(i, l.rank, size) for i in l.all_instr()]
    if instrs:
        if all(i.shape() == instrs[0].shape() for i in instrs):
            return nested(instrs, l.rank, l.all_frees())
        r = nested_sized(instrs, l.rank, size)
        r.frees.update(l.all_frees())
        return r
    r = l.clone()
    r.size = size
    return r


def reshape_and_merge(l1: Loop, l2: Loop) -> Loop:
    if l1.size == l2.size:
        return _merge(l1, l2)
    if l2.reshapable and l1.size and l2.size % l1.size == 0:
        return _merge(l1, _reshape_loop(l2, l1.size))
    if l1.reshapable and l2.size and l1.size % l2.size == 0:
        return _merge(_reshape_loop(l1, l2.size), l2)
    if not l1.all_instr():
        r = l2.clone()
        r.frees.update(l1.all_frees())
        return r
    if not l2.all_instr():
        r = l1.clone()
        r.frees.update(l2.all_frees())
        return r
    raise RuntimeError("reshape_and_merge: not mergeable")


# -------------------------------------------------------------------------------- instruction list
def remove_non_computed(instrs):
    """core/jitk/instruction.cpp:580-593: frees of never-computed bases leave the list."""
    out, frees, computed = [], [], set()
    for i in instrs:
        if i.opcode == OP["FREE"] and i.ops[0].base.id not in computed:
            frees.append(i.ops[0].base)
        elif i.opcode not in (OP["NONE"], OP["TALLY"]):
            for b in i.bases():
                computed.add(b.id)
            out.append(i)
    return out, frees


def simplify_list(instrs):
    """Move every BH_FREE after the last access of its base (core/jitk/fuser.cpp:167-221)."""
    last_access, base2free, free_instrs, pending = {}, {}, set(), set()
    for i in reversed(instrs):
        if i.opcode == OP["FREE"]:
            free_instrs.add(id(i))
            base2free[i.ops[0].base.id] = i
            pending.add(i.ops[0].base.id)
        else:
            found = [b.id for b in i.bases() if b.id in pending]
            if found:
                last_access[id(i)] = found
                pending -= set(found)
    out = []
    for i in instrs:
        if not i.ops or id(i) in free_instrs:
            continue
        s = i.clone()
        simplify(s)
        out.append(s)
        for bid in last_access.get(id(i), []):
            out.append(base2free[bid].clone())
    return out


def _fully_dp(a: I, b: I):
    if a.is_system() or b.is_system():
        return True

    def fv(w, r):
        if w is None or r is None or w.base is not r.base:
            return True
        return w.start == r.start and w.shape == r.shape and w.stride == r.stride

    if b.opcode == OP["GATHER"] and a.ops[0].base is b.ops[1].base:
        return False
    if a.opcode in (OP["SCATTER"], OP["COND_SCATTER"]):
        if any(v is not None and a.ops[0].base is v.base for v in b.ops):
            return False
    elif b.opcode in (OP["SCATTER"], OP["COND_SCATTER"]):
        if any(v is not None and b.ops[0].base is v.base for v in a.ops):
            return False
    return all(fv(a.ops[0], v) for v in b.ops) and all(fv(b.ops[0], v) for v in a.ops)


def pre_fuser_lossy(instrs):
    simple = simplify_list(instrs)
    groups = []
    k = 0
    while k < len(simple):
        g = [simple[k]]
        k += 1
        while k < len(simple):
            nxt = simple[k]
            if nxt.is_system() or all(i.is_system() or (i.shape() == nxt.shape() and _fully_dp(i, nxt)) for i in g):
                g.append(nxt)
                k += 1
            else:
                break
        groups.append(g)
    return [nested(g) for g in groups]


# ------------------------------------------------------------------------------------ block DAG
def _merge_weight(a: Loop, b: Loop):
    news = a.all_news()
    frees = b.all_frees()
    return sum(frees[x].nbytes for x in news if x in frees)


class _DAG:
    def __init__(self, blocks):
        self.block = list(blocks)
        self.out = [set() for _ in blocks]
        self.inn = [set() for _ in blocks]
        self.alive = [True] * len(blocks)
        base2v = {}
        for vtx, blk in enumerate(self.block):
            conn = set()
            for bid in blk.all_bases():
                conn |= base2v.setdefault(bid, set())
                base2v[bid].add(vtx)
            mine = blk.all_instr()
            for u in conn:
                if u != vtx and any(self._dep(a, b) for a in mine for b in self.block[u].all_instr()):
                    self.add(u, vtx)
            connf = set()
            for bid in blk.all_frees():
                connf |= base2v.setdefault(bid, set())
                base2v[bid].add(vtx)
            for u in connf:
                if u != vtx:
                    self.add(u, vtx)

    @staticmethod
    def _dep(a: I, b: I):
        if not a.ops or not b.ops:
            return False
        ao, bo = a.ops[0], b.ops[0]
        return any(v is not None and bo is not None and v.base is bo.base for v in a.ops) or \
            any(v is not None and ao is not None and v.base is ao.base for v in b.ops)

    def add(self, a, b):
        self.out[a].add(b)
        self.inn[b].add(a)

    def remove_edge(self, a, b):
        self.out[a].discard(b)
        self.inn[b].discard(a)

    def edges(self):
        return [(a, b) for a in range(len(self.block)) if self.alive[a] for b in sorted(self.out[a])]

    def long_path(self, a, b):
        seen = {a}
        q = deque([a])
        while q:
            u = q.popleft()
            for w in sorted(self.out[u]):
                if w == b and u != a:
                    return True
                if w not in seen:
                    seen.add(w)
                    q.append(w)
        return False

    def merge(self, a, b):
        self.block[a] = reshape_and_merge(self.block[a], self.block[b])
        for c in list(self.out[b]):
            self.add(a, c)
        for p in list(self.inn[b]):
            if p != a:
                self.add(p, a)
        for c in list(self.out[b]):
            self.inn[c].discard(b)
        for p in list(self.inn[b]):
            self.out[p].discard(b)
        self.out[b].clear()
        self.inn[b].clear()
        self.alive[b] = False

    def topo(self):
        finished, state = [], [False] * len(self.block)
        for s in range(len(self.block)):
            if not self.alive[s] or state[s]:
                continue
            state[s] = True
            stack = [(s, iter(sorted(self.out[s])))]
            while stack:
                node, it = stack[-1]
                nxt = next(it, None)
                if nxt is None:
                    finished.append(node)
                    stack.pop()
                elif not state[nxt]:
                    state[nxt] = True
                    stack.append((nxt, iter(sorted(self.out[nxt]))))
        return [self.block[v] for v in reversed(finished)]


def greedy(blocks, avoid_rank0_sweep=False, threshold=10000):
    dag = _DAG(blocks)
    if sum(len(o) for o in dag.out) > threshold:
        return serial(blocks, avoid_rank0_sweep)
    while True:
        fusible = []
        for a, b in dag.edges():
            if dag.long_path(a, b):
                dag.remove_edge(a, b)
            elif mergeable(dag.block[a], dag.block[b], avoid_rank0_sweep):
                fusible.append((a, b))
        if not fusible:
            break
        best, bw = fusible[0], _merge_weight(dag.block[fusible[0][0]], dag.block[fusible[0][1]])
        for e in fusible:
            w = _merge_weight(dag.block[e[0]], dag.block[e[1]])
            if w > bw:
                best, bw = e, w
        dag.merge(*best)
    out = dag.topo()
    for blk in out:
        blk.items = _greedy_items(blk.items, threshold)
    return out


def _greedy_items(items, threshold):
    loops = [it for it in items if isinstance(it, Loop)]
    if len(loops) < 2:
        for l in loops:
            l.items = _greedy_items(l.items, threshold)
        return items
    # Instruction blocks never merge; run the DAG contraction over the loop sub-blocks and keep
    # instruction blocks in their order relative to each other.
    dag_blocks = [it if isinstance(it, Loop) else _InstrHolder(it) for it in items]
    fused = greedy(dag_blocks, False, threshold)
    return [b.ib if isinstance(b, _InstrHolder) else b for b in fused]


class _InstrHolder(Loop):
    """An instruction block inside a DAG: never mergeable (merges require two loops)."""

    def __init__(self, ib):
        super().__init__(ib.rank, -1, [ib])
        self.ib = ib
        self.reshapable = False

    def is_system_only(self):
        return False


def serial(blocks, avoid_rank0_sweep=False):
    """fuser_serial (core/jitk/fuser.cpp:271-293): merge consecutive mergeable blocks."""
    out = []
    for b in blocks:
        if out and isinstance(out[-1], Loop) and not isinstance(out[-1], _InstrHolder) and \
                not isinstance(b, _InstrHolder) and mergeable(out[-1], b, avoid_rank0_sweep):
            out[-1] = reshape_and_merge(out[-1], b)
        else:
            out.append(b)
    return out


def _collapse_axes(loop: Loop, axis: int) -> bool:
    for it in loop.items:
        if isinstance(it, IB):
            ins = it.instr.clone()
            sa = ins.sweep_axis()
            if sa in (axis, axis + 1):
                return False
            for k, v in enumerate(ins.ops):
                if v is None:
                    continue
                ax = axis
                if k == 0 and ins.opcode in REDUCE_OPS:
                    ax = ax - 1 if sa < ax else ax
                if v.ndim <= ax + 1 or v.shape[ax + 1] * v.stride[ax + 1] != v.stride[ax]:
                    return False
                v.shape[ax] *= v.shape[ax + 1]
                v.stride[ax] = v.stride[ax + 1]
            ins.remove_axis(axis + 1)
            it.instr = ins
            it.rank = ins.ndim()
        else:
            it.rank -= 1
            if not _collapse_axes(it, axis):
                return False
    loop.update()
    return True


def collapse_redundant_axes(blocks):
    """core/jitk/transformer.cpp:226-246."""
    out = []
    for b in blocks:
        if isinstance(b, Loop):
            b.items = collapse_redundant_axes(b.items)
            c = b.clone()
            if not c.sweeps and len(c.items) == 1 and c.reshapable and isinstance(c.items[0], Loop) and \
                    not c.items[0].sweeps and c.items[0].reshapable:
                child = c.items[0]
                c.size *= child.size
                c.frees.update(child.frees)
                c.items = [it.clone() if isinstance(it, Loop) else IB(it.instr, it.rank) for it in child.items]
                if _collapse_axes(c, c.rank):
                    out.append(c)
                    continue
        out.append(b)
    return out


# ---------------------------------------------------------------------------------- kernel list
def sweep_identity(opcode, dtype):
    """core/jitk/instruction.cpp:546-578 (including its choices of identity values)."""
    import numpy as np
    name = _ir.OPNAMES[opcode]
    t = np.dtype(dtype)
    if name in ("ADD_REDUCE", "BITWISE_OR_REDUCE", "BITWISE_XOR_REDUCE", "LOGICAL_OR_REDUCE",
                "LOGICAL_XOR_REDUCE", "ADD_ACCUMULATE"):
        return 0
    if name in ("MULTIPLY_REDUCE", "MULTIPLY_ACCUMULATE"):
        return 1
    if name in ("BITWISE_AND_REDUCE", "LOGICAL_AND_REDUCE"):
        return True if t == np.bool_ else int(np.array(0xFFFFFFFF, dtype=np.uint64).astype(t))
    if name == "MAXIMUM_REDUCE":
        if t == np.bool_:
            return True
        if np.issubdtype(t, np.floating):
            return float(np.finfo(t).tiny)
        if np.issubdtype(t, np.signedinteger):
            return int(np.iinfo(t).min) + 1
        return 0
    if name == "MINIMUM_REDUCE":
        if t == np.bool_:
            return True
        if np.issubdtype(t, np.floating):
            return float(np.finfo(t).max)
        return int(np.iinfo(t).max)
    raise ValueError(name)


def _identity_for(sweep: I, origin):
    v = sweep.ops[0].clone()
    if sweep.opcode in ACCUM_OPS:
        v.shape[sweep.sweep_axis()] = 1
    return I(OP["IDENTITY"], [v, None], (sweep_identity(sweep.opcode, v.base.dtype), _ir.bh_type(v.base.dtype)),
             sweep.constructor, origin)


def _add_identity(loop: Loop, counter):
    out = []
    for it in loop.items:
        if isinstance(it, IB):
            out.append(it)
            continue
        _add_identity(it, counter)
        for sw in sorted(it.sweeps, key=lambda s: -s.origin_id):
            ident = _identity_for(sw, counter[0])
            counter[0] += 1
            if loop.rank == -1 and sw.ops[0].is_scalar():
                out.append(IB(ident, 0))
            elif loop.rank == sw.ops[0].ndim - 1:
                out.append(IB(ident, sw.ops[0].ndim))
            else:
                out.append(nested([ident], loop.rank + 1))
            _replace(it, sw)
            it.update()
        out.append(it)
    loop.items = out
    loop.update()


def _replace(loop: Loop, sweep: I):
    for it in loop.items:
        if isinstance(it, IB):
            if it.instr.same(sweep):
                c = it.instr.clone()
                c.constructor = False
                it.instr = c
        else:
            _replace(it, sweep)


def kernel_list(instrs, fuser=("greedy", "collapse_redundant_axes")):
    """get_kernel_list() for the OpenMP configuration (avoid_rank0_sweep = false)."""
    for k, i in enumerate(instrs):
        i.origin_id = k
    blocks = pre_fuser_lossy(instrs)
    for t in fuser:
        if t == "greedy":
            blocks = greedy(blocks)
        elif t == "serial":
            blocks = serial(blocks)
        elif t == "collapse_redundant_axes":
            blocks = collapse_redundant_axes(blocks)
        elif t == "none":
            pass
        else:
            raise ValueError(t)
    counter = [len(instrs)]
    kernels = []
    for b in blocks:
        k = Loop(-1, 1, [b])
        _add_identity(k, counter)
        kernels.append(k)
    return kernels
