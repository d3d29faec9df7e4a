// Instruction fusion: from a flushed instruction list to a list of kernels (loop nests).
//
// Pipeline (core/jitk/apply_fusion.cpp:177-259 of the reference):
//   simplify_instr_list -> pre-fuser (lossy | singleton) -> transformers in `fuser_list`
//   -> identity blocks in front of every sweep -> kernel list.
// The transformer names and their semantics follow core/jitk/fuser.cpp, graph.cpp and
// transformer.cpp. A learned cost model can replace the greedy merge order ("learned" in
// fuser_list) but merges still go through mergeable(); see costmodel.hpp.
#pragma once

#include <cstdint>
#include <functional>
#include <string>
#include <vector>
#include <bohrium/bh_config_parser.hpp>
#include "block.hpp"

namespace bohrium {
namespace jitk {

struct FusionConfig {
    std::string pre_fuser = "lossy";
    std::vector<std::string> fuser_list = {"greedy", "collapse_redundant_axes"};
    uint64_t greedy_threshold = 10000;
    bool avoid_rank0_sweep = false;
    bool avoid_mixed_sweeps = false; // see MixedSweepRule (block.hpp)
    bool monolithic = false;
    FusionConfig() = default;
    FusionConfig(const ConfigParser &config, bool avoid_rank0_sweep);
};

// Picks the next merge for the "learned" transformer: given the candidate (mergeable) edges of a
// block DAG as (block a, block b) pairs, return the index of the edge to merge, or -1 to stop.
typedef std::function<int(const std::vector<std::pair<const Block *, const Block *>> &)> MergeChooser;

void simplify_instr(bh_instruction &instr);
std::vector<InstrPtr> simplify_instr_list(const std::vector<bh_instruction *> &instr_list);
std::vector<Block> pre_fuser_lossy(const std::vector<bh_instruction *> &instr_list);
std::vector<Block> fuser_singleton(const std::vector<bh_instruction *> &instr_list);
void fuser_serial(std::vector<Block> &block_list, bool avoid_rank0_sweep);
void fuser_breadth_first(std::vector<Block> &block_list, bool avoid_rank0_sweep);
void fuser_reshapable_first(std::vector<Block> &block_list, bool avoid_rank0_sweep);
void fuser_greedy(const FusionConfig &config, std::vector<Block> &block_list);
// Greedy-style DAG contraction where `chooser` picks the merge order (the legality test is still
// mergeable()). The recursion into deeper ranks uses the plain greedy fuser.
void fuser_chosen(const FusionConfig &config, std::vector<Block> &block_list, const MergeChooser &chooser);
void push_reductions_inwards(std::vector<Block> &block_list);
void split_for_threading(std::vector<Block> &block_list, uint64_t min_threading = 1000);
void collapse_redundant_axes(std::vector<Block> &block_list);

// Bytes of temporaries eliminated by merging b1 into b2 (core/jitk/graph.cpp:136-150).
uint64_t merge_weight(const Block &b1, const Block &b2);
// Bytes of non-temporary arrays a block touches (core/jitk/graph.cpp:152-170).
uint64_t block_cost(const Block &block);

// Run the pre-fuser and the transformers on `instr_list` (no kernel-level identity blocks).
std::vector<Block> fuse_block_list(const std::vector<bh_instruction *> &instr_list, const FusionConfig &config,
                                   const MergeChooser *chooser = nullptr);
// Assign origin ids, fuse, and wrap every block into a kernel (rank -1) with identity blocks.
std::vector<LoopB> get_kernel_list(const std::vector<bh_instruction *> &instr_list, const FusionConfig &config,
                                   const std::vector<Block> *cached_block_list = nullptr,
                                   std::vector<Block> *block_list_out = nullptr,
                                   const MergeChooser *chooser = nullptr);

} // namespace jitk
} // namespace bohrium
