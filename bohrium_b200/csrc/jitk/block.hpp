// Loop-nest blocks produced by the fuser.
//
// A Block is either a loop (LoopB, rank >= 0; rank -1 is a whole kernel) or a single instruction
// (InstrB). This is the block model of include/bohrium/jitk/block.hpp:39-321 of the reference,
// re-written on std::variant; the fusion legality rules (mergeable, data-parallel compatibility,
// reshape-and-merge) follow core/jitk/block.cpp:513-693.
#pragma once

#include <memory>
#include <set>
#include <string>
#include <utility>
#include <variant>
#include <vector>
#include <bohrium/bh_instruction.hpp>

namespace bohrium {
namespace jitk {

typedef std::shared_ptr<const bh_instruction> InstrPtr;

class Block;

class LoopB {
public:
    int rank = -42;
    int64_t size = -42;
    std::vector<Block> _block_list;
    std::set<InstrPtr> _sweeps;   // instructions sweeping this loop's axis
    std::set<bh_base *> _news;    // arrays created by local instructions
    std::set<bh_base *> _frees;   // arrays freed in this loop
    bool _reshapable = false;

    LoopB() = default;
    LoopB(int rank, int64_t size, std::vector<Block> block_list = {});

    const std::set<InstrPtr> &getSweeps() const { return _sweeps; }
    const std::set<bh_base *> &getNews() const { return _news; }
    const std::set<bh_base *> &getFrees() const { return _frees; }
    int replaceInstr(const InstrPtr &subject, const bh_instruction &replacement);
    bool isInnermost() const;
    void getAllSubBlocks(std::vector<const LoopB *> &out) const;
    std::vector<const LoopB *> getLocalSubBlocks() const;
    std::set<const bh_base *> getAllBases() const;
    void getAllNews(std::set<bh_base *> &out) const;
    std::set<bh_base *> getAllNews() const;
    void getAllFrees(std::set<bh_base *> &out) const;
    std::set<bh_base *> getAllFrees() const;
    void getLocalTemps(std::set<bh_base *> &out) const;
    std::set<bh_base *> getLocalTemps() const;
    void getAllTemps(std::set<bh_base *> &out) const;
    std::set<bh_base *> getAllTemps() const;
    std::set<bh_base *> getAllNonTemps() const;
    bool isSystemOnly() const;
    bool validation() const;
    uint64_t localThreading() const;
    std::string pprint(const char *newline = "\n") const;
    void metadataUpdate();
};

class InstrB {
public:
    InstrPtr instr;
    int rank;
};

class Block {
    std::variant<std::monostate, LoopB, InstrB> _var;

public:
    Block() = default;
    explicit Block(const LoopB &l) : _var(l) {}
    explicit Block(LoopB &&l) : _var(std::move(l)) {}
    Block(const bh_instruction &instr, int rank) : _var(InstrB{std::make_shared<bh_instruction>(instr), rank}) {}
    Block(InstrPtr instr, int rank) : _var(InstrB{std::move(instr), rank}) {}

    bool isInstr() const { return _var.index() == 2; }
    LoopB &getLoop() { return std::get<LoopB>(_var); }
    const LoopB &getLoop() const { return std::get<LoopB>(_var); }
    InstrPtr &getInstr() { return std::get<InstrB>(_var).instr; }
    const InstrPtr &getInstr() const { return std::get<InstrB>(_var).instr; }
    void setInstr(const bh_instruction &instr) {
        InstrB &ib = std::get<InstrB>(_var);
        ib.rank = static_cast<int>(instr.ndim());
        ib.instr = std::make_shared<bh_instruction>(instr);
    }
    int rank() const { return isInstr() ? std::get<InstrB>(_var).rank : getLoop().rank; }
    bool validation() const;
    std::set<const bh_base *> getAllBases() const;
    bool isSystemOnly() const;
    bool isReshapable() const { return isInstr() ? getInstr()->reshapable() : getLoop()._reshapable; }
    // True when this block must execute after `other`.
    bool dependOn(const Block &other) const;
    std::string pprint(const char *newline = "\n") const;
};

// Instruction iteration helpers (include/bohrium/jitk/iterator.hpp of the reference).
void all_instr(const LoopB &loop, std::vector<InstrPtr> &out);
std::vector<InstrPtr> all_instr(const LoopB &loop);
std::vector<InstrPtr> all_instr(const Block &block);
std::vector<InstrPtr> all_local_instr(const LoopB &loop);
std::vector<const bh_base *> instr_bases(const bh_instruction &instr);

LoopB merge(const LoopB &a, const LoopB &b);
// Nest `instr_list` from `rank` down to the innermost loop (all instructions share one shape).
Block create_nested_block(const std::vector<InstrPtr> &instr_list, int rank = 0, std::set<bh_base *> frees = {});
// Nest `instr_list` at `rank` with the given loop size (reshaping reshapable instructions).
Block create_nested_block(const std::vector<InstrPtr> &instr_list, int rank, int64_t size_of_rank_dim);
// (number of leading ranks that can run in parallel, total parallelism)
std::pair<uint64_t, uint64_t> parallel_ranks(const LoopB &block, unsigned int max_depth = 3);
std::vector<const LoopB *> get_first_loop_blocks(const LoopB &block);
bool mergeable(const Block &b1, const Block &b2, bool avoid_rank0_sweep);
// While an instance lives (on this thread), mergeable() also refuses merges whose result sweeps
// axes at more than one loop rank (e.g. a column sum fused with a row sum): such a nest can only
// run on one thread, so the GPU keeps the two reductions in separate kernels.
struct MixedSweepRule {
    explicit MixedSweepRule(bool on);
    ~MixedSweepRule();
    static bool active();
    bool previous;
};
Block reshape_and_merge(const LoopB &l1, const LoopB &l2);

// Reshape the dimensions from `rank` inwards of a reshapable instruction to `size_of_rank_dim`
// (core/jitk/instruction.cpp:595-616 of the reference).
InstrPtr reshape_rank(const InstrPtr &instr, int rank, int64_t size_of_rank_dim);
// The identity value a reduction/accumulate starts from (core/jitk/instruction.cpp:546-578).
bh_constant sweep_identity(bh_opcode opcode, bh_type dtype);
// Drop BH_NONE/BH_TALLY and collect frees of bases never computed on
// (core/jitk/instruction.cpp:580-593).
std::vector<bh_instruction *> remove_non_computed_system_instr(std::vector<bh_instruction> &instr_list,
                                                               std::set<bh_base *> &frees);
// True when `instr` reduces over its innermost axis.
bool sweeping_innermost_axis(const InstrPtr &instr);

std::ostream &operator<<(std::ostream &out, const LoopB &b);
std::ostream &operator<<(std::ostream &out, const Block &b);

} // namespace jitk
} // namespace bohrium
