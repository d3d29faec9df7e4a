// Block model and fusion legality; see block.hpp for the reference correspondence.
#include <algorithm>
#include <cassert>
#include <iterator>
#include <sstream>
#include <stdexcept>
#include "block.hpp"

using namespace std;

namespace bohrium {
namespace jitk {

// ------------------------------------------------------------------------- iteration helpers
namespace {
void collect(const vector<Block> &list, vector<InstrPtr> &out) {
    for (const Block &b : list) {
        if (b.isInstr()) {
            out.push_back(b.getInstr());
        } else {
            collect(b.getLoop()._block_list, out);
        }
    }
}
template <typename C, typename T>
bool contains(const C &c, const T &v) {
    return c.find(v) != c.end();
}
} // namespace

void all_instr(const LoopB &loop, vector<InstrPtr> &out) { collect(loop._block_list, out); }
vector<InstrPtr> all_instr(const LoopB &loop) {
    vector<InstrPtr> ret;
    collect(loop._block_list, ret);
    return ret;
}
vector<InstrPtr> all_instr(const Block &block) {
    if (block.isInstr()) return {block.getInstr()};
    return all_instr(block.getLoop());
}
vector<InstrPtr> all_local_instr(const LoopB &loop) {
    vector<InstrPtr> ret;
    for (const Block &b : loop._block_list)
        if (b.isInstr()) ret.push_back(b.getInstr());
    return ret;
}
vector<const bh_base *> instr_bases(const bh_instruction &instr) {
    vector<const bh_base *> ret;
    for (const bh_view &v : instr.getViews())
        if (find(ret.begin(), ret.end(), v.base) == ret.end()) ret.push_back(v.base);
    return ret;
}

bool sweeping_innermost_axis(const InstrPtr &instr) {
    if (!bh_opcode_is_sweep(instr->opcode)) return false;
    return instr->sweep_axis() == instr->operand[1].ndim - 1;
}

InstrPtr reshape_rank(const InstrPtr &instr, int rank, int64_t size_of_rank_dim) {
    vector<int64_t> shape(static_cast<size_t>(rank) + 1);
    for (int r = 0; r < rank; ++r) shape[r] = instr->operand[0].shape[r];
    int64_t size = 1;
    for (int64_t r = rank; r < instr->operand[0].ndim; ++r) size *= instr->operand[0].shape[r];
    shape[rank] = size_of_rank_dim;
    if (size != size_of_rank_dim) {
        if (size_of_rank_dim == 0 || size % size_of_rank_dim != 0)
            throw runtime_error("reshape_rank(): shape is not divisible with 'size_of_rank_dim'");
        shape.push_back(size / size_of_rank_dim);
    }
    bh_instruction ret(*instr);
    ret.reshape(shape);
    return make_shared<bh_instruction>(ret);
}

bh_constant sweep_identity(bh_opcode opcode, bh_type dtype) {
    switch (opcode) {
        case BH_ADD_REDUCE:
        case BH_BITWISE_OR_REDUCE:
        case BH_BITWISE_XOR_REDUCE:
        case BH_LOGICAL_OR_REDUCE:
        case BH_LOGICAL_XOR_REDUCE:
        case BH_ADD_ACCUMULATE:
            return bh_constant(0, dtype);
        case BH_MULTIPLY_REDUCE:
        case BH_MULTIPLY_ACCUMULATE:
            return bh_constant(1, dtype);
        case BH_BITWISE_AND_REDUCE:
        case BH_LOGICAL_AND_REDUCE:
            // ~0u converted to the element type: all ones up to 32 bits (as in the reference).
            return bh_constant(~0u, dtype);
        case BH_MAXIMUM_REDUCE:
            return dtype == bh_type::BOOL ? bh_constant(bh_bool{1}) : bh_constant::get_min(dtype);
        case BH_MINIMUM_REDUCE:
            return dtype == bh_type::BOOL ? bh_constant(bh_bool{1}) : bh_constant::get_max(dtype);
        default:
            throw runtime_error(string("sweep_identity(): unsupported operation: ") + bh_opcode_text(opcode));
    }
}

vector<bh_instruction *> remove_non_computed_system_instr(vector<bh_instruction> &instr_list, set<bh_base *> &frees) {
    vector<bh_instruction *> ret;
    set<const bh_base *> computes;
    for (bh_instruction &instr : instr_list) {
        if (instr.opcode == BH_FREE && !contains(computes, static_cast<const bh_base *>(instr.operand[0].base))) {
            frees.insert(instr.operand[0].base);
        } else if (!(instr.opcode == BH_NONE || instr.opcode == BH_TALLY)) {
            for (const bh_base *b : instr_bases(instr)) computes.insert(b);
            ret.push_back(&instr);
        }
    }
    return ret;
}

// ---------------------------------------------------------------------------------------- LoopB
namespace {
bool is_reshapable(const vector<InstrPtr> &instr_list) {
    if (instr_list.empty()) return true;
    const int64_t rank = instr_list.front()->ndim();
    for (const InstrPtr &instr : instr_list) {
        if (!instr->reshapable() || instr->ndim() != rank) return false;
    }
    return true;
}

void add_instr_to_block(LoopB &block, InstrPtr instr, int rank, int64_t size_of_rank_dim) {
    if (instr->ndim() <= rank) throw runtime_error("add_instr_to_block(): instruction with ndim <= rank");
    if (instr->reshapable() && instr->operand[0].shape[rank] != size_of_rank_dim) {
        instr = reshape_rank(instr, rank, size_of_rank_dim);
    }
    const BhIntVec shape = instr->shape();
    if (shape[rank] != size_of_rank_dim)
        throw runtime_error("create_nested_block(): instruction where shape[rank] != size_of_rank_dim");
    const int64_t max_ndim = instr->ndim();
    if (max_ndim > rank + 1) {
        block._block_list.push_back(create_nested_block(vector<InstrPtr>{instr}, rank + 1, shape[rank + 1]));
    } else if (instr->opcode == BH_FREE) {
        block._frees.insert(instr->operand[0].base);
    } else {
        block._block_list.emplace_back(instr, rank + 1);
    }
    block.metadataUpdate();
}
} // namespace

LoopB::LoopB(int r, int64_t s, vector<Block> block_list) : rank(r), size(s), _block_list(std::move(block_list)) {}

namespace {
// `f(loop)` for `loop` and then for every loop nested in it, depth first, in block-list order.
template <typename L, typename F>
void visit_loops(L &loop, F &&f) {
    f(loop);
    for (auto &b : loop._block_list)
        if (!b.isInstr()) visit_loops(b.getLoop(), f);
}
} // namespace

int LoopB::replaceInstr(const InstrPtr &subject, const bh_instruction &replacement) {
    int replaced = 0;
    visit_loops(*this, [&](LoopB &l) {
        for (Block &b : l._block_list)
            if (b.isInstr() && *b.getInstr() == *subject) {
                b.setInstr(replacement);
                ++replaced;
            }
    });
    return replaced;
}

bool LoopB::isInnermost() const {
    return none_of(_block_list.begin(), _block_list.end(), [](const Block &b) { return !b.isInstr(); });
}

bool LoopB::isSystemOnly() const {
    return all_of(_block_list.begin(), _block_list.end(), [](const Block &b) { return b.isSystemOnly(); });
}

void LoopB::getAllSubBlocks(vector<const LoopB *> &out) const {
    visit_loops(*this, [&](const LoopB &l) {
        if (&l != this) out.push_back(&l);
    });
}

vector<const LoopB *> LoopB::getLocalSubBlocks() const {
    vector<const LoopB *> children;
    for (const Block &b : _block_list)
        if (!b.isInstr()) children.push_back(&b.getLoop());
    return children;
}

set<const bh_base *> LoopB::getAllBases() const {
    set<const bh_base *> bases;
    for (const InstrPtr &instr : all_instr(*this))
        for (const bh_view &v : instr->getViews()) bases.insert(v.base);
    return bases;
}

void LoopB::getAllNews(set<bh_base *> &out) const {
    visit_loops(*this, [&](const LoopB &l) { out.insert(l._news.begin(), l._news.end()); });
}
set<bh_base *> LoopB::getAllNews() const {
    set<bh_base *> news;
    getAllNews(news);
    return news;
}
void LoopB::getAllFrees(set<bh_base *> &out) const {
    visit_loops(*this, [&](const LoopB &l) { out.insert(l._frees.begin(), l._frees.end()); });
}
set<bh_base *> LoopB::getAllFrees() const {
    set<bh_base *> frees;
    getAllFrees(frees);
    return frees;
}

// A temporary of this loop is created here and freed here or in a nested loop, or freed here and
// created here or in a nested loop (the reference's rule, core/jitk/block.cpp:174-181).
void LoopB::getLocalTemps(set<bh_base *> &out) const {
    const set<bh_base *> frees_below = getAllFrees(), news_below = getAllNews();
    for (bh_base *b : _news)
        if (frees_below.count(b)) out.insert(b);
    for (bh_base *b : _frees)
        if (news_below.count(b)) out.insert(b);
}
set<bh_base *> LoopB::getLocalTemps() const {
    set<bh_base *> temps;
    getLocalTemps(temps);
    return temps;
}
void LoopB::getAllTemps(set<bh_base *> &out) const {
    visit_loops(*this, [&](const LoopB &l) { l.getLocalTemps(out); });
}
set<bh_base *> LoopB::getAllTemps() const {
    set<bh_base *> temps;
    getAllTemps(temps);
    return temps;
}
set<bh_base *> LoopB::getAllNonTemps() const {
    const set<bh_base *> temps = getAllTemps();
    set<bh_base *> rest;
    for (const bh_base *b : getAllBases())
        if (!temps.count(const_cast<bh_base *>(b))) rest.insert(const_cast<bh_base *>(b));
    return rest;
}

bool LoopB::validation() const {
    if (size < 0 || rank < 0) return false;
    for (const InstrPtr &instr : all_instr(*this)) {
        if (bh_opcode_is_system(instr->opcode)) return false;
        if (instr->ndim() <= rank) return false;
        if (instr->shape()[rank] != size) return false;
    }
    for (const Block &b : _block_list)
        if (!b.validation()) return false;
    for (const InstrPtr &instr : all_local_instr(*this))
        if (instr->ndim() != rank + 1) return false;
    return true;
}

uint64_t LoopB::localThreading() const {
    if (_sweeps.empty() && !isSystemOnly()) return static_cast<uint64_t>(size);
    return 0;
}

string LoopB::pprint(const char *newline) const {
    stringstream ss;
    ss << string(static_cast<size_t>(max(rank, 0) * 4), ' ') << "rank: " << rank << ", size: " << size;
    if (!_sweeps.empty()) {
        ss << ", sweeps: { ";
        for (const InstrPtr &instr : _sweeps) ss << *instr << ",";
        ss << "}";
    }
    if (_reshapable) ss << ", reshapable";
    if (!_news.empty()) {
        ss << ", news: {";
        for (const bh_base *b : _news) ss << "a" << b->getLabel() << ",";
        ss << "}";
    }
    if (!_frees.empty()) {
        ss << ", frees: {";
        for (const bh_base *b : _frees) ss << "a" << b->getLabel() << ",";
        ss << "}";
    }
    ss << ", block list:" << newline;
    for (const Block &b : _block_list) ss << b.pprint(newline);
    return ss.str();
}

void LoopB::metadataUpdate() {
    _news.clear();
    _sweeps.clear();
    for (const InstrPtr &instr : all_local_instr(*this))
        if (instr->constructor) _news.insert(instr->operand[0].base);
    for (const InstrPtr &instr : all_instr(*this))
        if (instr->sweep_axis() == rank) _sweeps.insert(instr);
    _reshapable = is_reshapable(all_instr(*this));
}

// ---------------------------------------------------------------------------------------- Block
bool Block::validation() const {
    if (isInstr()) return getInstr()->ndim() == rank();
    return getLoop().validation();
}

set<const bh_base *> Block::getAllBases() const {
    set<const bh_base *> ret;
    for (const InstrPtr &instr : all_instr(*this))
        for (const bh_base *b : instr_bases(*instr)) ret.insert(b);
    return ret;
}

bool Block::isSystemOnly() const {
    if (isInstr()) return bh_opcode_is_system(getInstr()->opcode);
    return getLoop().isSystemOnly();
}

bool Block::dependOn(const Block &other) const {
    const vector<InstrPtr> mine = all_instr(*this), theirs = all_instr(other);
    for (const InstrPtr &a : mine)
        for (const InstrPtr &b : theirs)
            if (bh_instr_dependency(a.get(), b.get())) return true;
    return false;
}

string Block::pprint(const char *newline) const {
    if (isInstr()) {
        stringstream ss;
        ss << string(static_cast<size_t>(max(rank(), 0) * 4), ' ') << *getInstr() << newline;
        return ss.str();
    }
    return getLoop().pprint(newline);
}

// ------------------------------------------------------------------------------ block functions
LoopB merge(const LoopB &l1, const LoopB &l2) {
    LoopB ret(l1);
    ret._block_list.clear();
    ret._block_list.insert(ret._block_list.end(), l1._block_list.begin(), l1._block_list.end());
    ret._block_list.insert(ret._block_list.end(), l2._block_list.begin(), l2._block_list.end());
    ret._sweeps.insert(l2._sweeps.begin(), l2._sweeps.end());
    ret._news.insert(l2._news.begin(), l2._news.end());
    ret._frees.insert(l2._frees.begin(), l2._frees.end());
    ret._reshapable = is_reshapable(all_instr(ret));
    return ret;
}

Block create_nested_block(const vector<InstrPtr> &instr_list, int rank, set<bh_base *> frees) {
    if (instr_list.empty()) throw runtime_error("create_nested_block: 'instr_list' is empty!");
    if (instr_list[0]->opcode == BH_NONE) throw runtime_error("create_nested_block: first instruction is BH_NONE!");
    const BhIntVec shape = instr_list[0]->shape();
    const int ndim = static_cast<int>(shape.size());
    LoopB ret;
    ret.rank = rank;
    ret.size = shape[rank];
    if (rank == ndim - 1) {
        ret._frees = std::move(frees);
        for (const InstrPtr &instr : instr_list) {
            if (instr->opcode == BH_FREE) {
                ret._frees.insert(instr->operand[0].base);
            } else {
                ret._block_list.emplace_back(instr, ndim);
            }
        }
    } else {
        ret._block_list.push_back(create_nested_block(instr_list, rank + 1, std::move(frees)));
    }
    ret.metadataUpdate();
    return Block(std::move(ret));
}

Block create_nested_block(const vector<InstrPtr> &instr_list, int rank, int64_t size_of_rank_dim) {
    if (instr_list.empty()) throw runtime_error("create_nested_block: 'instr_list' is empty!");
    LoopB ret{rank, size_of_rank_dim};
    for (const InstrPtr &instr : instr_list) add_instr_to_block(ret, instr, rank, size_of_rank_dim);
    return Block(std::move(ret));
}

pair<uint64_t, uint64_t> parallel_ranks(const LoopB &block, unsigned int max_depth) {
    pair<uint64_t, uint64_t> ret(0, 0);
    const uint64_t thds = block.localThreading();
    --max_depth;
    if (thds > 0) {
        if (max_depth > 0) {
            const size_t nblocks = block.getLocalSubBlocks().size();
            const bool no_instr = all_local_instr(block).empty();
            // Several sub-blocks, or instructions mixed with a sub-block, serialise the sub-blocks.
            if (nblocks == 1 && no_instr) {
                const auto sub = parallel_ranks(block._block_list[0].getLoop(), max_depth);
                ret.first += sub.first;
                ret.second += sub.second;
            }
        }
        ret.second += thds;
        ++ret.first;
    }
    return ret;
}

vector<const LoopB *> get_first_loop_blocks(const LoopB &block) {
    vector<const LoopB *> ret;
    const LoopB *cur = &block;
    while (true) {
        ret.push_back(cur);
        if (cur->_block_list.empty() || cur->_block_list[0].isInstr()) break;
        cur = &cur->_block_list[0].getLoop();
    }
    return ret;
}

namespace {
// Can `writer` and `reader` of the same base run element-wise in one loop nest?
bool dp_compatible(const bh_view &writer, const bh_view &reader) {
    if (writer.isConstant() || reader.isConstant() || writer.base != reader.base) return true;
    if (writer.start != reader.start) return false;
    if (writer.ndim == reader.ndim) return writer.shape == reader.shape && writer.stride == reader.stride;
    return writer.shape.prod() == reader.shape.prod() && writer.isContiguous() && reader.isContiguous();
}

bool dp_compatible(const InstrPtr &a, const InstrPtr &b) {
    if (bh_opcode_is_system(a->opcode) || bh_opcode_is_system(b->opcode)) return true;
    if (b->opcode == BH_GATHER && a->operand[0].base == b->operand[1].base) return false;
    if (a->opcode == BH_SCATTER || a->opcode == BH_COND_SCATTER) {
        for (const bh_view &v : b->operand)
            if (!v.isConstant() && a->operand[0].base == v.base) return false;
    } else if (b->opcode == BH_SCATTER || b->opcode == BH_COND_SCATTER) {
        for (const bh_view &v : a->operand)
            if (!v.isConstant() && b->operand[0].base == v.base) return false;
    }
    for (const bh_view &v : b->operand)
        if (!dp_compatible(a->operand[0], v)) return false;
    for (const bh_view &v : a->operand)
        if (!dp_compatible(b->operand[0], v)) return false;
    return true;
}

bool dp_compatible(const LoopB &b1, const LoopB &b2) {
    const vector<InstrPtr> i1s = all_instr(b1), i2s = all_instr(b2);
    for (const InstrPtr &i1 : i1s)
        for (const InstrPtr &i2 : i2s)
            if (i1.get() != i2.get() && !dp_compatible(i1, i2)) return false;
    return true;
}

bool sweeps_accessed_by_block(const set<InstrPtr> &sweeps, const LoopB &loop) {
    if (sweeps.empty()) return false;
    const set<const bh_base *> bases = loop.getAllBases();
    for (const InstrPtr &instr : sweeps)
        if (contains(bases, static_cast<const bh_base *>(instr->operand[0].base))) return true;
    return false;
}

// Reshape a reshapable loop so that its size at l1.rank becomes `size_of_rank_dim`; all frees move
// to the innermost loop (core/jitk/block.cpp:609-627 of the reference).
Block reshape_block(const LoopB &l1, int64_t size_of_rank_dim) {
    vector<InstrPtr> instr_list;
    for (const InstrPtr &instr : all_instr(l1)) instr_list.push_back(reshape_rank(instr, l1.rank, size_of_rank_dim));
    if (!instr_list.empty()) {
        bool same_shape = true;
        for (const InstrPtr &i : instr_list) same_shape = same_shape && i->shape() == instr_list[0]->shape();
        if (same_shape) return create_nested_block(instr_list, l1.rank, l1.getAllFrees());
        Block ret = create_nested_block(instr_list, l1.rank, size_of_rank_dim);
        const auto frees = l1.getAllFrees();
        ret.getLoop()._frees.insert(frees.begin(), frees.end());
        return ret;
    }
    LoopB ret = l1;
    ret.size = size_of_rank_dim;
    return Block(std::move(ret));
}
} // namespace

Block reshape_and_merge(const LoopB &l1, const LoopB &l2) {
    if (l1.size == l2.size) return Block(merge(l1, l2));
    if (l2._reshapable && l1.size != 0 && l2.size % l1.size == 0) {
        const LoopB new_l2 = reshape_block(l2, l1.size).getLoop();
        return Block(merge(l1, new_l2));
    }
    if (l1._reshapable && l2.size != 0 && l1.size % l2.size == 0) {
        const LoopB new_l1 = reshape_block(l1, l2.size).getLoop();
        return Block(merge(new_l1, l2));
    }
    if (all_instr(l1).empty()) {
        LoopB ret = l2;
        const auto frees = l1.getAllFrees();
        ret._frees.insert(frees.begin(), frees.end());
        return Block(std::move(ret));
    }
    if (all_instr(l2).empty()) {
        LoopB ret = l1;
        const auto frees = l2.getAllFrees();
        ret._frees.insert(frees.begin(), frees.end());
        return Block(std::move(ret));
    }
    throw runtime_error("reshape_and_merge: the blocks are not mergeable!");
}

namespace {
thread_local bool t_avoid_mixed_sweeps = false;

void sweep_ranks(const LoopB &l, set<int> &out) {
    if (!l._sweeps.empty()) out.insert(l.rank);
    for (const Block &b : l._block_list)
        if (!b.isInstr()) sweep_ranks(b.getLoop(), out);
}
} // namespace

MixedSweepRule::MixedSweepRule(bool on) : previous(t_avoid_mixed_sweeps) { t_avoid_mixed_sweeps = on; }
bool MixedSweepRule::active() { return t_avoid_mixed_sweeps; }
MixedSweepRule::~MixedSweepRule() { t_avoid_mixed_sweeps = previous; }

bool mergeable(const Block &b1, const Block &b2, bool avoid_rank0_sweep) {
    if (b1.isInstr() || b2.isInstr()) return false;
    const LoopB &l1 = b1.getLoop();
    const LoopB &l2 = b2.getLoop();
    if (l2.isSystemOnly()) return true;
    if (avoid_rank0_sweep && l1.rank == 0 && l2.rank == 0) {
        if (l1._sweeps.empty() != l2._sweeps.empty()) return false;
    }
    if (t_avoid_mixed_sweeps) {
        set<int> ranks;
        sweep_ranks(l1, ranks);
        sweep_ranks(l2, ranks);
        if (ranks.size() > 1) return false;
    }
    if (sweeps_accessed_by_block(l1._sweeps, l2)) return false;
    if (l1.size == l2.size || (l2._reshapable && l1.size != 0 && l2.size % l1.size == 0) ||
        (l1._reshapable && l2.size != 0 && l1.size % l2.size == 0)) {
        return dp_compatible(l1, l2);
    }
    return false;
}

ostream &operator<<(ostream &out, const LoopB &b) { return out << b.pprint(); }
ostream &operator<<(ostream &out, const Block &b) { return out << b.pprint(); }

} // namespace jitk
} // namespace bohrium
