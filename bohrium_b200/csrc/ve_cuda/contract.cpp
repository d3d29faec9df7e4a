// Multiply-add contraction on the bytecode, before fusion.
//
// A product that exists only to be added (`MUL t, a, b; ADD r, t, c; ... FREE t`) is replaced by
// one instruction `r = a*b + c` with a single rounding (fma). Because the rewrite happens on the
// instruction list and not in the generated code, every fusion plan -- greedy, grouped, graph
// replay, learned -- sees the same instructions and computes the same bits, and kernels are still
// compiled with --fmad=false so the compiler contracts nothing else. The reference's engines
// leave contraction to their C compilers (ve/openmp compiles with gcc -O3 -march=native, whose
// default -ffp-contract=fast contracts wherever the fused code allows), so results agree with the
// oracle within the elementwise tolerance either way.
#include <algorithm>
#include <functional>
#include <map>
#include "codegen.hpp"

using namespace std;

namespace bohrium {
namespace cuda {

namespace {

constexpr size_t kWindow = 64;  // how far to look for the consumer of a product and for its FREE

bool touches(const bh_instruction &in, const bh_base *b) {
    for (const bh_view &v : in.operand)
        if (!v.isConstant() && v.base == b) return true;
    return false;
}

bool writes(const bh_instruction &in, const bh_base *b) {
    return !in.operand.empty() && !in.operand[0].isConstant() && in.operand[0].base == b;
}

// An operand of `in` usable in a contraction of element type `t`: a constant of that type, or a
// view of an array of that type without sliding.
bool plain_float(const bh_instruction &in, const bh_view &v, bh_type t) {
    return v.isConstant() ? in.constant.type == t : v.base->dtype() == t && !v.hasSlide();
}

} // namespace

bool is_fma_opcode(bh_opcode op) { return op == BH_X_FMA || op == BH_X_FMS || op == BH_X_FNMA; }

int contract_multiply_add(vector<bh_instruction> &list, const set<bh_base *> &syncs,
                          const function<bool(const bh_base *)> &holds_nothing) {
    int made = 0;
    const size_t n = list.size();
    map<size_t, vector<bh_instruction>> moved;  // FREEs of multiply inputs, re-inserted after the add
    for (size_t i = 0; i < n; ++i) {
        bh_instruction &mul = list[i];
        if (mul.opcode != BH_MULTIPLY || mul.operand.size() != 3 || mul.operand[0].isConstant()) continue;
        const bh_view t = mul.operand[0];
        const bh_type ty = t.base->dtype();
        if ((ty != bh_type::FLOAT32 && ty != bh_type::FLOAT64) || t.hasSlide() || syncs.count(t.base)) continue;
        const bh_view &a0 = mul.operand[1], &b0 = mul.operand[2];
        if (!plain_float(mul, a0, ty) || !plain_float(mul, b0, ty) || (a0.isConstant() && b0.isConstant())) continue;
        if ((!a0.isConstant() && a0.base == t.base) || (!b0.isConstant() && b0.base == t.base)) continue;  // t = t * x
        // The next instruction that touches t must read it once, as one input of an ADD or SUBTRACT.
        size_t j = i + 1;
        const size_t jend = min(n, i + 1 + kWindow);
        while (j < jend && !touches(list[j], t.base)) ++j;
        if (j >= jend) continue;
        bh_instruction &add = list[j];
        if ((add.opcode != BH_ADD && add.opcode != BH_SUBTRACT) || add.operand.size() != 3 ||
            add.operand[0].isConstant() || add.operand[0].base == t.base)
            continue;
        const bool t1 = !add.operand[1].isConstant() && add.operand[1].base == t.base;
        const bool t2 = !add.operand[2].isConstant() && add.operand[2].base == t.base;
        if (t1 == t2) continue;
        const bh_view &tv = add.operand[t1 ? 1 : 2];
        if (!(tv == t)) continue;
        const bh_view c = add.operand[t1 ? 2 : 1];
        const bh_view r = add.operand[0];
        if (r.base->dtype() != ty || r.hasSlide() || !plain_float(add, c, ty)) continue;
        // a and b are read at the ADD instead of the MULTIPLY: nothing in between may write them,
        // a FREE of them in between moves to just after the ADD, and the result may only overlap
        // them as the very same view.
        bool ok = true;
        vector<size_t> frees;
        for (size_t k = i + 1; k < j && ok; ++k) {
            for (const bh_view *v : {&a0, &b0}) {
                if (v->isConstant() || !writes(list[k], v->base)) continue;
                if (list[k].opcode == BH_FREE) {
                    if (find(frees.begin(), frees.end(), k) == frees.end()) frees.push_back(k);
                } else {
                    ok = false;
                }
            }
        }
        for (const bh_view *v : {&a0, &b0})
            if (!v->isConstant() && v->base == r.base && !(*v == r)) ok = false;
        if (!ok) continue;
        // After the ADD, t is only freed.
        size_t f = j + 1;
        const size_t fend = min(n, j + 1 + kWindow);
        while (f < fend && !touches(list[f], t.base)) ++f;
        if (f >= fend || list[f].opcode != BH_FREE) continue;

        // The constant multiplier, if any, goes second (multiplication commutes exactly).
        const bh_view &a = a0.isConstant() ? b0 : a0;
        const bh_view &b = a0.isConstant() ? a0 : b0;
        bh_instruction fma;
        fma.opcode = add.opcode == BH_ADD ? BH_X_FMA : (t1 ? BH_X_FMS : BH_X_FNMA);
        fma.operand = {r, a, b, c};
        fma.origin_id = add.origin_id;
        if (b.isConstant() && c.isConstant()) {
            // Two constants: the multiplier as the real part and the addend as the imaginary part
            // of one complex constant of the same precision.
            if (ty == bh_type::FLOAT32) {
                fma.constant = bh_constant(std::complex<float>(mul.constant.value.float32, add.constant.value.float32));
            } else {
                fma.constant = bh_constant(std::complex<double>(mul.constant.value.float64, add.constant.value.float64));
            }
        } else if (b.isConstant()) {
            fma.constant = mul.constant;
        } else if (c.isConstant()) {
            fma.constant = add.constant;
        }
        add = std::move(fma);
        mul.opcode = BH_NONE;
        mul.operand.clear();
        // The product's array is now never computed; when nothing is held for it, its FREE has
        // nothing to release either and goes too (an engine would otherwise free it on every
        // execution of the flush).
        if (holds_nothing && holds_nothing(list[f].operand[0].base)) {
            list[f] = bh_instruction();
            list[f].opcode = BH_NONE;
        }
        for (size_t k : frees) {
            moved[j].push_back(std::move(list[k]));
            list[k] = bh_instruction();
            list[k].opcode = BH_NONE;
        }
        ++made;
    }
    if (!moved.empty()) {
        vector<bh_instruction> out;
        out.reserve(list.size() + 8);
        for (size_t k = 0; k < n; ++k) {
            out.push_back(std::move(list[k]));
            auto it = moved.find(k);
            if (it != moved.end())
                for (bh_instruction &f : it->second) out.push_back(std::move(f));
        }
        list = std::move(out);
    }
    return made;
}

} // namespace cuda
} // namespace bohrium
