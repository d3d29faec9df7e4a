#include "filters.hpp"

#include <algorithm>
#include <cstdint>
#include <map>
#include <set>

using namespace std;

namespace bohrium {
namespace filter {

namespace {

bh_view constant_operand() { return bh_view(); }

bh_instruction make(bh_opcode op, vector<bh_view> operands) { return bh_instruction(op, std::move(operands)); }

// A contiguous view of a new base with the shape of `like`.
bh_view fresh_view(BaseStore &created, const bh_view &like, bh_type t) {
    int64_t n = 1;
    for (int64_t d = 0; d < like.ndim; ++d) n *= like.shape[d];
    created.emplace_back(new bh_base(n, t));
    bh_view v;
    v.base = created.back().get();
    v.start = 0;
    v.ndim = like.ndim;
    v.shape = like.shape;
    v.stride = like.shape;
    int64_t s = 1;
    for (int64_t d = like.ndim - 1; d >= 0; --d) {
        v.stride[static_cast<size_t>(d)] = s;
        s *= like.shape[static_cast<size_t>(d)];
    }
    return v;
}

bool int_type(bh_type t) { return bh_type_is_integer(t) != 0; }

bool reduce1d_opcode(bh_opcode op) {
    switch (op) {
        case BH_ADD_REDUCE:
        case BH_MULTIPLY_REDUCE:
        case BH_MINIMUM_REDUCE:
        case BH_MAXIMUM_REDUCE:
        case BH_LOGICAL_AND_REDUCE:
        case BH_BITWISE_AND_REDUCE:
        case BH_LOGICAL_OR_REDUCE:
        case BH_BITWISE_OR_REDUCE:
        case BH_LOGICAL_XOR_REDUCE:
        case BH_BITWISE_XOR_REDUCE: return true;
        default: return false;
    }
}

// The fold of a 1-D reduction of `n` elements: the largest divisor of n in [2, n / limit], or 1.
int64_t reduce1d_fold(int64_t n, int64_t limit) {
    for (int64_t i = n / limit; i > 1; --i)
        if (n % i == 0) return i;
    return 1;
}

} // namespace

int expand(BhIR &bhir, const ExpandOptions &opt, BaseStore &created) {
    int rewrites = 0;
    vector<bh_instruction> out;
    out.reserve(bhir.instr_list.size());
    for (bh_instruction &instr : bhir.instr_list) {
        if (opt.powk && instr.opcode == BH_POWER && instr.operand.size() == 3 && instr.operand[2].isConstant() &&
            !instr.operand[1].isConstant() && int_type(instr.constant.type) &&
            instr.operand[0].base != instr.operand[1].base) {
            const int64_t k = instr.constant.get_int64();
            if (k >= 0 && k <= 100) {
                const bh_view o = instr.operand[0], x = instr.operand[1];
                if (k == 0) {
                    bh_instruction one = make(BH_IDENTITY, {o, constant_operand()});
                    one.constant = bh_constant(1, o.base->dtype());
                    out.push_back(one);
                } else if (k == 1) {
                    out.push_back(make(BH_IDENTITY, {o, x}));
                } else {
                    int64_t p = 1;
                    while (p * 2 <= k) p *= 2;
                    out.push_back(make(BH_MULTIPLY, {o, x, x}));
                    for (int64_t q = 4; q <= p; q *= 2) out.push_back(make(BH_MULTIPLY, {o, o, o}));
                    for (int64_t r = 0; r < k - p; ++r) out.push_back(make(BH_MULTIPLY, {o, o, x}));
                }
                ++rewrites;
                continue;
            }
        }
        if (opt.sign && instr.opcode == BH_SIGN && instr.operand.size() == 2 && !instr.operand[1].isConstant()) {
            const bh_type t = instr.operand[1].base->dtype();
            if (t != bh_type::COMPLEX64 && t != bh_type::COMPLEX128) {
                const bh_view o = instr.operand[0], x = instr.operand[1];
                const bh_type ot = o.base->dtype();
                const bh_view gt = fresh_view(created, o, bh_type::BOOL), lt = fresh_view(created, o, bh_type::BOOL);
                const bh_view g = fresh_view(created, o, ot), l = fresh_view(created, o, ot);
                bh_instruction a = make(BH_GREATER, {gt, x, constant_operand()});
                a.constant = bh_constant(0, t);
                bh_instruction b = make(BH_LESS, {lt, x, constant_operand()});
                b.constant = bh_constant(0, t);
                out.push_back(a);
                out.push_back(make(BH_IDENTITY, {g, gt}));
                out.push_back(make(BH_FREE, {gt}));
                out.push_back(b);
                out.push_back(make(BH_IDENTITY, {l, lt}));
                out.push_back(make(BH_FREE, {lt}));
                out.push_back(make(BH_SUBTRACT, {o, g, l}));
                out.push_back(make(BH_FREE, {g}));
                out.push_back(make(BH_FREE, {l}));
                ++rewrites;
                continue;
            }
        }
        if (opt.reduce1d > 0 && reduce1d_opcode(instr.opcode) && instr.operand.size() == 3 &&
            !instr.operand[1].isConstant() && instr.operand[1].ndim == 1) {
            // out = reduce(x) over n elements -> t[n/f] = reduce over axis 0 of x viewed as [f, n/f];
            // out = reduce(t); free t
            const int64_t n = instr.operand[1].shape[0];
            const int64_t fold = n * 2 < opt.reduce1d ? 1 : reduce1d_fold(n, opt.reduce1d);
            if (fold >= 2) {
                bh_view x = instr.operand[1];
                const int64_t st = x.stride[0];
                x.ndim = 2;
                x.shape = {fold, n / fold};
                x.stride = {st * (n / fold), st};
                bh_view like;
                like.ndim = 1;
                like.shape = {n / fold};
                const bh_view t = fresh_view(created, like, x.base->dtype());
                bh_instruction first = make(instr.opcode, {t, x, constant_operand()});
                first.constant = bh_constant(static_cast<int64_t>(0));
                bh_instruction second = make(instr.opcode, {instr.operand[0], t, constant_operand()});
                second.constant = bh_constant(static_cast<int64_t>(0));
                out.push_back(first);
                out.push_back(second);
                out.push_back(make(BH_FREE, {t}));
                ++rewrites;
                continue;
            }
        }
        out.push_back(instr);
    }
    if (rewrites) bhir.instr_list = std::move(out);
    return rewrites;
}

namespace {

// Uses of every base: number of reads (non-output operands) per instruction index, and the index
// of the BH_FREE of each base.
struct Uses {
    map<const bh_base *, vector<size_t>> reads, writes;
    map<const bh_base *, size_t> freed;
    explicit Uses(const vector<bh_instruction> &list) {
        for (size_t i = 0; i < list.size(); ++i) {
            const bh_instruction &in = list[i];
            if (in.opcode == BH_NONE) continue;
            if (in.opcode == BH_FREE) {
                freed[in.operand[0].base] = i;
                continue;
            }
            for (size_t o = 0; o < in.operand.size(); ++o) {
                if (in.operand[o].isConstant()) continue;
                (o == 0 ? writes : reads)[in.operand[o].base].push_back(i);
            }
        }
    }
    // `b` is written once at `w`, read only at `r` (once), and freed after `r`.
    bool single_link(const bh_base *b, size_t w, size_t r) const {
        auto wi = writes.find(b), ri = reads.find(b);
        auto fi = freed.find(b);
        return wi != writes.end() && wi->second.size() == 1 && wi->second[0] == w && ri != reads.end() &&
               ri->second.size() == 1 && ri->second[0] == r && fi != freed.end() && fi->second > r;
    }
};

// Does an instruction strictly between lo and hi access `b` (write only, with `writes_only`)?
bool touched_between(const vector<bh_instruction> &list, const bh_base *b, size_t lo, size_t hi, bool writes_only) {
    for (size_t i = lo + 1; i < hi; ++i) {
        const bh_instruction &in = list[i];
        if (in.opcode == BH_NONE) continue;
        for (size_t o = 0; o < in.operand.size(); ++o) {
            if (in.operand[o].isConstant() || in.operand[o].base != b) continue;
            if (!writes_only || o == 0 || in.opcode == BH_FREE) return true;
        }
    }
    return false;
}

bool const_right(const bh_instruction &i) {
    return i.operand.size() == 3 && i.operand[2].isConstant() && !i.operand[1].isConstant();
}

} // namespace

int collect_once(vector<bh_instruction> &list);
int muladd_once(vector<bh_instruction> &list);

int contract(BhIR &bhir, const ContractOptions &opt) {
    vector<bh_instruction> &list = bhir.instr_list;
    int rewrites = 0;
    if (opt.stupidmath) {
        for (bh_instruction &in : list) {
            if (in.operand.size() != 3 || !in.has_constant() || !int_type(in.constant.type)) continue;
            const bool cr = in.operand[2].isConstant(), cl = in.operand[1].isConstant();
            if (cr == cl) continue;
            const int64_t c = in.constant.get_int64();
            bool ok = false;
            switch (in.opcode) {
                case BH_MULTIPLY: ok = c == 1; break;
                case BH_ADD: ok = c == 0; break;
                case BH_DIVIDE: ok = cr && c == 1; break;
                case BH_SUBTRACT: ok = cr && c == 0; break;
                default: break;
            }
            if (!ok) continue;
            in.opcode = BH_IDENTITY;
            in.operand.erase(in.operand.begin() + (cr ? 2 : 1));
            ++rewrites;
        }
    }
    // Each pass rewrites at most one chain (the use lists are rebuilt in between).
    for (int pass = 0; pass < 10000; ++pass) {
        int r = 0;
        if (opt.collect) r += collect_once(list);
        if (opt.muladd) r += muladd_once(list);
        if (r == 0) break;
        rewrites += r;
    }
    return rewrites;
}

int collect_once(vector<bh_instruction> &list) {
    int rewrites = 0;
    {
        const Uses uses(list);
        for (size_t i = 0; i < list.size(); ++i) {
            bh_instruction &first = list[i];
            const bh_opcode op = first.opcode;
            const bool addsub = op == BH_ADD || op == BH_SUBTRACT;
            if (!(addsub || op == BH_MULTIPLY) || !const_right(first)) continue;
            const bh_type t = first.operand[0].base->dtype();
            if (!int_type(t) || first.constant.type != t || first.operand[1].base->dtype() != t) continue;
            // Follow the chain: the next reader of the link's output, the same kind of operation.
            vector<size_t> chain{i};
            // Integer arithmetic wraps modulo 2^bits, so folding the constants (also modulo 2^64,
            // then converted to the type) is exact.
            const uint64_t c0 = static_cast<uint64_t>(first.constant.get_int64());
            uint64_t acc = addsub ? (op == BH_ADD ? c0 : uint64_t(0) - c0) : c0;
            size_t cur = i;
            while (true) {
                const bh_base *b = list[cur].operand[0].base;
                auto ri = uses.reads.find(b);
                if (ri == uses.reads.end() || ri->second.size() != 1) break;
                const size_t nx = ri->second[0];
                bh_instruction &next = list[nx];
                const bool ok_kind = addsub ? (next.opcode == BH_ADD || next.opcode == BH_SUBTRACT)
                                            : next.opcode == BH_MULTIPLY;
                if (!ok_kind || !const_right(next) || !(next.operand[1] == list[cur].operand[0]) ||
                    next.constant.type != t || next.operand[0].base->dtype() != t || !uses.single_link(b, cur, nx))
                    break;
                const uint64_t c = static_cast<uint64_t>(next.constant.get_int64());
                acc = addsub ? acc + (next.opcode == BH_ADD ? c : uint64_t(0) - c) : acc * c;
                chain.push_back(nx);
                cur = nx;
            }
            if (chain.size() < 2) continue;
            // first computes the chain's final output directly (its output must not be touched
            // before the last link wrote it); the links and their frees go.
            bh_instruction &last = list[chain.back()];
            if (touched_between(list, last.operand[0].base, i, chain.back(), false)) continue;
            first.operand[0] = last.operand[0];
            first.opcode = addsub ? BH_ADD : BH_MULTIPLY;
            first.constant.set_value(static_cast<int64_t>(acc));
            for (size_t k = 1; k < chain.size(); ++k) {
                const bh_base *link = list[chain[k - 1]].operand[0].base;
                list[chain[k]].opcode = BH_NONE;
                auto fi = uses.freed.find(link);
                if (fi != uses.freed.end()) list[fi->second].opcode = BH_NONE;
            }
            ++rewrites;
            break;  // uses are stale now; one chain per pass
        }
    }
    return rewrites;
}

int muladd_once(vector<bh_instruction> &list) {
    int rewrites = 0;
    {
        const Uses uses(list);
        for (size_t k = 0; k < list.size(); ++k) {
            bh_instruction &sum = list[k];
            if ((sum.opcode != BH_ADD && sum.opcode != BH_SUBTRACT) || sum.operand.size() != 3 ||
                sum.operand[1].isConstant() || sum.operand[2].isConstant())
                continue;
            const bh_type t = sum.operand[0].base->dtype();
            if (!int_type(t)) continue;
            // Producers of the two operands.
            auto producer = [&](const bh_view &v) -> long {
                auto wi = uses.writes.find(v.base);
                if (wi == uses.writes.end() || wi->second.size() != 1) return -1;
                const size_t w = wi->second[0];
                const bh_instruction &p = list[w];
                if (p.opcode != BH_MULTIPLY || p.operand.size() != 3 || !(p.operand[0] == v) ||
                    !uses.single_link(v.base, w, k))
                    return -1;
                if (p.operand[1].isConstant() == p.operand[2].isConstant()) return -1;
                if (p.constant.type != t) return -1;
                return static_cast<long>(w);
            };
            const long p1 = producer(sum.operand[1]), p2 = producer(sum.operand[2]);
            if (p1 < 0 || p2 < 0) continue;
            bh_instruction &m1 = list[static_cast<size_t>(p1)], &m2 = list[static_cast<size_t>(p2)];
            const bh_view &x1 = m1.operand[1].isConstant() ? m1.operand[2] : m1.operand[1];
            const bh_view &x2 = m2.operand[1].isConstant() ? m2.operand[2] : m2.operand[1];
            if (!(x1 == x2) || x1.base->dtype() != t) continue;
            // x keeps its value from the products to the sum.
            if (touched_between(list, x1.base, static_cast<size_t>(min(p1, p2)), k, true)) continue;
            const uint64_t a = static_cast<uint64_t>(m1.constant.get_int64());
            const uint64_t b = static_cast<uint64_t>(m2.constant.get_int64());
            const int64_t c = static_cast<int64_t>(sum.opcode == BH_ADD ? a + b : a - b);
            const bh_view x = x1, y = sum.operand[0];
            const bh_base *t1 = sum.operand[1].base, *t2 = sum.operand[2].base;
            // y = c * x at the place of the sum; the products and their frees go.
            sum.opcode = BH_MULTIPLY;
            sum.operand = {y, x, constant_operand()};
            sum.constant = bh_constant(c, t);
            m1.opcode = BH_NONE;
            m2.opcode = BH_NONE;
            for (const bh_base *tb : {t1, t2}) {
                auto fi = uses.freed.find(tb);
                if (fi != uses.freed.end()) list[fi->second].opcode = BH_NONE;
            }
            ++rewrites;
            break;
        }
    }
    return rewrites;
}

} // namespace filter
} // namespace bohrium
