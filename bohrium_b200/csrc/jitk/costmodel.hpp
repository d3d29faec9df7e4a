// Features of a fused block for the learned fusion cost model.
//
// The cost model (an MLP trained on the device times that the engine records) predicts the device
// time of a candidate fused block from these features. The reference has no learned fuser; its
// greedy fuser (core/jitk/graph.cpp:319-365) stays both the fallback and the legality rule: the
// learned chooser only picks among merges that mergeable() allows.
#pragma once

#include <array>
#include "block.hpp"

namespace bohrium {
namespace jitk {

constexpr int kCostFeatures = 16;
typedef std::array<float, kCostFeatures> CostFeatures;

// Feature vector of a block (a rank-0 block of the fuser or a whole kernel at rank -1):
//   0 log2(1 + instructions)            8 sweeps at more than one rank (0/1)
//   1 log2(1 + transcendental ops)      9 loop-nest depth
//   2 log2(1 + bytes read)             10 fraction of views with unit innermost stride
//   3 log2(1 + bytes written)          11 fraction of views with a broadcast (zero) stride
//   4 log2(1 + iteration-space size)   12 fraction of other (strided/transposed) views
//   5 log2(1 + parallel iterations)    13 fraction of instructions on float64
//   6 reductions sweeping rank 0       14 fraction of instructions on integers/bools
//   7 reductions sweeping deeper ranks 15 log2(1 + distinct arrays)
// Bytes count the arrays that are not temporaries of the block (temporaries are contracted).
CostFeatures block_features(const Block &block);
CostFeatures block_features(const LoopB &loop);

} // namespace jitk
} // namespace bohrium
