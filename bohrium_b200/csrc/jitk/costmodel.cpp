#include "costmodel.hpp"

#include <cmath>
#include <map>
#include <set>

using namespace std;

namespace bohrium {
namespace jitk {

namespace {

bool transcendental(bh_opcode op) {
    switch (op) {
        case BH_POWER: case BH_SIN: case BH_COS: case BH_TAN: case BH_SINH: case BH_COSH: case BH_TANH:
        case BH_ARCSIN: case BH_ARCCOS: case BH_ARCTAN: case BH_ARCSINH: case BH_ARCCOSH: case BH_ARCTANH:
        case BH_ARCTAN2: case BH_EXP: case BH_EXP2: case BH_EXPM1: case BH_LOG: case BH_LOG2: case BH_LOG10:
        case BH_LOG1P: case BH_SQRT: case BH_DIVIDE: case BH_MOD: case BH_REMAINDER:
            return true;
        default:
            return false;
    }
}

float lg(double x) { return static_cast<float>(std::log2(1.0 + x)); }

struct Walk {
    int max_rank = -1;
    set<int> sweep_ranks;
    int sweeps_rank0 = 0, sweeps_deeper = 0;
    void loop(const LoopB &l) {
        if (l.rank > max_rank) max_rank = l.rank;
        for (const InstrPtr &s : l._sweeps) {
            if (!bh_opcode_is_sweep(s->opcode)) continue;
            sweep_ranks.insert(l.rank);
            if (l.rank <= 0) {
                ++sweeps_rank0;
            } else {
                ++sweeps_deeper;
            }
        }
        for (const Block &b : l._block_list)
            if (!b.isInstr()) loop(b.getLoop());
    }
};

int64_t view_elements(const bh_view &v) {
    int64_t n = 1;
    for (int64_t d = 0; d < v.ndim; ++d) n *= v.shape[d];
    return n;
}

} // namespace

CostFeatures block_features(const LoopB &loop) {
    CostFeatures f{};
    const vector<InstrPtr> instrs = all_instr(loop);
    const set<bh_base *> temps = loop.getAllTemps();
    map<const bh_base *, int64_t> reads, writes;  // elements touched per non-temporary array
    set<const bh_base *> bases;
    int n_instr = 0, n_trans = 0, n_f64 = 0, n_int = 0, n_views = 0, n_unit = 0, n_bcast = 0;
    int64_t space = 0;
    for (const InstrPtr &ip : instrs) {
        const bh_instruction &in = *ip;
        if (bh_opcode_is_system(in.opcode)) continue;
        ++n_instr;
        if (transcendental(in.opcode)) ++n_trans;
        const bh_view &out = in.operand[0];
        if (!out.isConstant()) {
            const bh_type t = out.base->dtype();
            if (t == bh_type::FLOAT64 || t == bh_type::COMPLEX128) {
                ++n_f64;
            } else if (t != bh_type::FLOAT32 && t != bh_type::COMPLEX64) {
                ++n_int;
            }
        }
        for (size_t o = 0; o < in.operand.size(); ++o) {
            const bh_view &v = in.operand[o];
            if (v.isConstant()) continue;
            bases.insert(v.base);
            const int64_t n = view_elements(v);
            if (n > space) space = n;
            ++n_views;
            bool bcast = false;
            for (int64_t d = 0; d < v.ndim; ++d)
                if (v.stride[d] == 0 && v.shape[d] > 1) bcast = true;
            if (bcast) {
                ++n_bcast;
            } else if (v.ndim == 0 || v.stride[v.ndim - 1] == 1 || v.shape[v.ndim - 1] == 1) {
                ++n_unit;
            }
            if (temps.count(v.base)) continue;
            auto &m = o == 0 ? writes : reads;
            int64_t &cur = m[v.base];
            if (n > cur) cur = n;
        }
    }
    double rbytes = 0, wbytes = 0;
    for (const auto &kv : reads)
        rbytes += static_cast<double>(min<int64_t>(kv.second, kv.first->nelem())) * bh_type_size(kv.first->dtype());
    for (const auto &kv : writes)
        wbytes += static_cast<double>(min<int64_t>(kv.second, kv.first->nelem())) * bh_type_size(kv.first->dtype());
    Walk w;
    w.loop(loop);
    uint64_t par = 0;
    if (loop.rank >= 0) {
        par = parallel_ranks(loop).second;
    } else {
        for (const Block &b : loop._block_list)
            if (!b.isInstr()) par = max(par, parallel_ranks(b.getLoop()).second);
    }
    const float nv = n_views > 0 ? static_cast<float>(n_views) : 1.f;
    const float ni = n_instr > 0 ? static_cast<float>(n_instr) : 1.f;
    f[0] = lg(n_instr);
    f[1] = lg(n_trans);
    f[2] = lg(rbytes);
    f[3] = lg(wbytes);
    f[4] = lg(static_cast<double>(space));
    f[5] = lg(static_cast<double>(par));
    f[6] = static_cast<float>(w.sweeps_rank0);
    f[7] = static_cast<float>(w.sweeps_deeper);
    f[8] = w.sweep_ranks.size() > 1 ? 1.f : 0.f;
    f[9] = static_cast<float>(w.max_rank + 1);
    f[10] = static_cast<float>(n_unit) / nv;
    f[11] = static_cast<float>(n_bcast) / nv;
    f[12] = static_cast<float>(n_views - n_unit - n_bcast) / nv;
    f[13] = static_cast<float>(n_f64) / ni;
    f[14] = static_cast<float>(n_int) / ni;
    f[15] = lg(static_cast<double>(bases.size()));
    return f;
}

CostFeatures block_features(const Block &block) {
    if (block.isInstr()) {
        LoopB l;
        l.rank = 0;
        l.size = 1;
        l._block_list.push_back(block);
        return block_features(l);
    }
    return block_features(block.getLoop());
}

} // namespace jitk
} // namespace bohrium
