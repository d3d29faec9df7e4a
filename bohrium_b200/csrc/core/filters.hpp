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
//   reduce1d  (expand_reduce1d.cpp:31-80) with a thread limit L > 0: a reduction of a 1-D view
//         of n >= L/2 elements -> the same reduction over axis 0 of the view reshaped to
//         [f, n/f] into a new temporary, then over that temporary, where f is the largest divisor
//         of n in [2, n/L]; no rewrite when there is none. Off (0) by default: the CUDA engine
//         reduces 1-D arrays in one GRID_REDUCE kernel, and the split changes the floating-point
//         summation order.
// The reduction contraction (bccon) is off in the reference's configs and not provided. Every
// rewrite keeps the results bit for bit except powk on floating-point data, whose products may
// round differently from pow(), and reduce1d on floating-point sums and products.
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
    int64_t reduce1d = 0; // thread limit of the 1-D reduction split; 0: off
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
