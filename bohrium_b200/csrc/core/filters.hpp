// Bytecode filters: rewrites of a BhIR applied by filter components before the vector engine.
//
// bcexp (filter/bcexp/expander.cpp:42-87 of the reference):
//   powk  BH_POWER x, k with an integer constant 0 <= k <= 100 -> BH_IDENTITY / BH_MULTIPLY chain
//         (square while a power of two fits, then multiply by x for the rest), written into the
//         output, when the output is not the input's base
//   sign  BH_SIGN x (real types) -> (x > 0) - (x < 0) through two temporaries
// bccon (filter/bccon/contracter.cpp:46-52 and the contract_*.cpp files):
//   stupidmath  x*1, x/1, x+0, x-0 (and 1*x, 0+x) with an integer-typed constant -> BH_IDENTITY;
//               only the forms whose value really is x (the reference also rewrites 1/x and 0-x)
//   collect     chains `t1 = x op c1; t2 = t1 op c2; ...` of ADD/SUBTRACT (or MULTIPLY) by
//               constants on integer arrays -> one instruction, when every link but the last is
//               a temporary freed right after its only use (exact: integers)
//   muladd      `t1 = a*x; t2 = b*x; y = t1 +- t2` on integer arrays with t1, t2 temporaries
//               used only there -> y = (a +- b)*x (exact: integers)
// reduce1d (bcexp) and the reduction contraction (bccon) are off in the GPU stack and not
// provided. Every rewrite keeps the results bit for bit except powk on floating-point data, whose
// products may round differently from pow().
#pragma once

#include <memory>
#include <string>
#include <vector>
#include <bohrium/bh_ir.hpp>

namespace bohrium {
namespace filter {

struct ExpandOptions {
    bool powk = true;
    bool sign = false;
};
struct ContractOptions {
    bool stupidmath = true;
    bool collect = true;
    bool muladd = true;
};

// Bases created by a rewrite (temporaries); they must outlive the execution of the BhIR.
typedef std::vector<std::unique_ptr<bh_base>> BaseStore;

// Rewrite `bhir` in place. Return the number of rewrites.
int expand(BhIR &bhir, const ExpandOptions &opt, BaseStore &created);
int contract(BhIR &bhir, const ContractOptions &opt);

} // namespace filter
} // namespace bohrium
