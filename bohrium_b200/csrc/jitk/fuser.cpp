// Fusers and transformers. The algorithms restate core/jitk/fuser.cpp:35-392,
// core/jitk/graph.cpp:52-365 and core/jitk/transformer.cpp:29-246 of the reference; the block
// DAG is a small adjacency structure of our own that keeps the reference's vertex order and its
// ordered (set-based) out-edge lists, so merge decisions are taken in the same order.
#include <algorithm>
#include <cassert>
#include <deque>
#include <map>
#include <numeric>
#include <stdexcept>
#include "fuser.hpp"

using namespace std;

namespace bohrium {
namespace jitk {

namespace {
template <typename C, typename T>
bool contains(const C &c, const T &v) {
    return c.find(v) != c.end();
}
} // namespace

FusionConfig::FusionConfig(const ConfigParser &config, bool avoid_rank0)
    : pre_fuser(config.defaultGet<string>("pre_fuser", "lossy")),
      fuser_list(config.defaultGetList("fuser_list", {"greedy", "collapse_redundant_axes"})),
      greedy_threshold(config.defaultGet<uint64_t>("greedy_threshold", 10000)),
      avoid_rank0_sweep(config.defaultGet<bool>("avoid_rank0_sweep", avoid_rank0)),
      avoid_mixed_sweeps(config.defaultGet<bool>("avoid_mixed_sweeps", false)),
      monolithic(config.defaultGet<bool>("monolithic", false)) {}

// ------------------------------------------------------------------------------- simplification
void simplify_instr(bh_instruction &instr) {
    if (instr.operand.empty()) return;
    {
        // Drop size-1 axes but keep at least one dimension (and never the swept axis).
        const BhIntVec shape = instr.shape();
        const int sa = instr.sweep_axis();
        size_t ndim_left = bh_opcode_is_reduction(instr.opcode) ? shape.size() - 1 : shape.size();
        for (int64_t i = static_cast<int64_t>(shape.size()) - 1; i >= 0 && ndim_left > 1; --i) {
            if (sa != i && shape[i] == 1) {
                instr.remove_axis(i);
                --ndim_left;
            }
        }
    }
    if (instr.ndim() > 1 && instr.reshapable()) {
        const BhIntVec shape = instr.shape();
        instr.reshape({shape.prod()});
    }
}

namespace {
bool fully_dp_compatible(const bh_view &writer, const bh_view &reader) {
    if (writer.isConstant() || reader.isConstant() || writer.base != reader.base) return true;
    if (writer.start != reader.start || writer.ndim != reader.ndim) return false;
    for (int64_t i = 0; i < writer.ndim; ++i)
        if (writer.stride[i] != reader.stride[i] || writer.shape[i] != reader.shape[i]) return false;
    return true;
}

bool fully_dp_compatible(const InstrPtr &a, const InstrPtr &b) {
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
        if (!fully_dp_compatible(a->operand[0], v)) return false;
    for (const bh_view &v : a->operand)
        if (!fully_dp_compatible(b->operand[0], v)) return false;
    return true;
}

bool fully_fusible(const vector<InstrPtr> &instr_list, const InstrPtr &instr) {
    if (instr_list.empty() || bh_opcode_is_system(instr->opcode)) return true;
    const BhIntVec dshape = instr->shape();
    const bool sweep = bh_opcode_is_sweep(instr->opcode);
    for (const InstrPtr &i : instr_list) {
        if (bh_opcode_is_system(i->opcode)) continue;
        if (i->shape() != dshape || !fully_dp_compatible(i, instr)) return false;
        // With the mixed-sweep rule, a group sweeps at most one axis (see MixedSweepRule).
        if (sweep && MixedSweepRule::active() && bh_opcode_is_sweep(i->opcode) && i->sweep_axis() != instr->sweep_axis())
            return false;
    }
    return true;
}
} // namespace

vector<InstrPtr> simplify_instr_list(const vector<bh_instruction *> &instr_list) {
    // Move every BH_FREE right after the last instruction that accesses its base.
    map<const bh_instruction *, vector<bh_base *>> last_access;
    map<bh_base *, const bh_instruction *> base2free;
    set<const bh_instruction *> free_instrs;
    {
        set<bh_base *> pending;
        for (auto it = instr_list.crbegin(); it != instr_list.crend(); ++it) {
            const bh_instruction *instr = *it;
            if (instr->opcode == BH_FREE) {
                free_instrs.insert(instr);
                base2free.insert(make_pair(instr->operand[0].base, instr));
                pending.insert(instr->operand[0].base);
            } else {
                vector<bh_base *> found;
                for (const bh_view &v : instr->getViews())
                    if (contains(pending, v.base) && find(found.begin(), found.end(), v.base) == found.end())
                        found.push_back(v.base);
                if (!found.empty()) {
                    sort(found.begin(), found.end());
                    last_access.insert(make_pair(instr, found));
                    for (bh_base *b : found) pending.erase(b);
                }
            }
        }
    }
    vector<InstrPtr> ret;
    for (const bh_instruction *instr : instr_list) {
        if (instr->operand.empty() || contains(free_instrs, instr)) continue;
        bh_instruction simple(*instr);
        simplify_instr(simple);
        ret.push_back(make_shared<const bh_instruction>(simple));
        auto it = last_access.find(instr);
        if (it != last_access.end()) {
            for (bh_base *b : it->second) ret.push_back(make_shared<const bh_instruction>(*base2free.at(b)));
        }
    }
    return ret;
}

vector<Block> pre_fuser_lossy(const vector<bh_instruction *> &instr_list) {
    const vector<InstrPtr> simple = simplify_instr_list(instr_list);
    vector<vector<InstrPtr>> groups;
    for (auto it = simple.begin(); it != simple.end();) {
        groups.push_back({*it});
        vector<InstrPtr> &group = groups.back();
        if (bh_opcode_is_system((*it)->opcode)) {
            // A group never starts with a system instruction (it must not dictate the shape):
            // the following instructions join it.
            ++it;
            for (; it != simple.end(); ++it) {
                if (fully_fusible(group, *it)) {
                    group.push_back(*it);
                } else {
                    break;
                }
            }
            continue;
        }
        ++it;
        for (; it != simple.end(); ++it) {
            if (fully_fusible(group, *it)) {
                group.push_back(*it);
            } else {
                break;
            }
        }
    }
    vector<Block> ret;
    for (const vector<InstrPtr> &g : groups) {
        // Groups made only of frees are attached as a free-only block of the following shape.
        size_t first = 0;
        while (first < g.size() && bh_opcode_is_system(g[first]->opcode)) ++first;
        if (first == g.size()) {
            // Only system instructions: nest them with the shape of the freed base.
            vector<InstrPtr> frees;
            for (const InstrPtr &i : g) {
                bh_instruction flat(*i);
                frees.push_back(make_shared<const bh_instruction>(flat));
            }
            ret.push_back(create_nested_block(frees, 0, frees.front()->operand[0].shape[0]));
            continue;
        }
        vector<InstrPtr> ordered;
        ordered.push_back(g[first]);
        for (size_t i = 0; i < g.size(); ++i)
            if (i != first) ordered.push_back(g[i]);
        ret.push_back(create_nested_block(ordered));
    }
    return ret;
}

vector<Block> fuser_singleton(const vector<bh_instruction *> &instr_list) {
    vector<Block> ret;
    for (const InstrPtr &instr : simplify_instr_list(instr_list)) {
        const BhIntVec shape = instr->shape();
        ret.push_back(create_nested_block(vector<InstrPtr>{instr}, 0, shape[0]));
    }
    return ret;
}

void fuser_serial(vector<Block> &block_list, bool avoid_rank0_sweep) {
    vector<Block> ret;
    for (auto it = block_list.begin(); it != block_list.end();) {
        ret.push_back(*it);
        Block &cur = ret.back();
        ++it;
        if (cur.isInstr()) continue;
        for (; it != block_list.end(); ++it) {
            if (!it->isInstr() && mergeable(cur, *it, avoid_rank0_sweep)) {
                cur = reshape_and_merge(cur.getLoop(), it->getLoop());
            } else {
                break;
            }
        }
        fuser_serial(cur.getLoop()._block_list, avoid_rank0_sweep);
    }
    block_list = ret;
}

// ------------------------------------------------------------------------------------ block DAG
namespace {

struct DAG {
    struct Vertex {
        Block block;
        set<size_t> out, in;
        bool alive = true;
    };
    vector<Vertex> v;

    size_t add(const Block &b) {
        v.push_back(Vertex{b, {}, {}, true});
        return v.size() - 1;
    }
    void add_edge(size_t a, size_t b) {
        v[a].out.insert(b);
        v[b].in.insert(a);
    }
    void remove_edge(size_t a, size_t b) {
        v[a].out.erase(b);
        v[b].in.erase(a);
    }
    void clear_vertex(size_t a) {
        for (size_t c : v[a].out) v[c].in.erase(a);
        for (size_t p : v[a].in) v[p].out.erase(a);
        v[a].out.clear();
        v[a].in.clear();
    }
    void remove_vertex(size_t a) {
        clear_vertex(a);
        v[a].alive = false;
    }
    size_t num_edges() const {
        size_t n = 0;
        for (const Vertex &x : v)
            if (x.alive) n += x.out.size();
        return n;
    }
    // Edges in vertex order, each vertex's out-edges in target order.
    vector<pair<size_t, size_t>> edges() const {
        vector<pair<size_t, size_t>> ret;
        for (size_t a = 0; a < v.size(); ++a)
            if (v[a].alive)
                for (size_t b : v[a].out) ret.emplace_back(a, b);
        return ret;
    }
    // Is `b` reachable from `a` through a path of length >= 2?
    bool long_path_exist(size_t a, size_t b) const {
        vector<char> seen(v.size(), 0);
        deque<size_t> q;
        q.push_back(a);
        seen[a] = 1;
        while (!q.empty()) {
            const size_t u = q.front();
            q.pop_front();
            for (size_t w : v[u].out) {
                if (w == b && u != a) return true;
                if (!seen[w]) {
                    seen[w] = 1;
                    q.push_back(w);
                }
            }
        }
        return false;
    }
};

DAG from_block_list(const vector<Block> &block_list) {
    DAG g;
    map<const bh_base *, set<size_t>> base2vertices;
    for (const Block &block : block_list) {
        const size_t vertex = g.add(block);
        set<size_t> connecting;
        for (const bh_base *base : block.getAllBases()) {
            set<size_t> &vs = base2vertices[base];
            connecting.insert(vs.begin(), vs.end());
            vs.insert(vertex);
        }
        for (auto it = connecting.rbegin(); it != connecting.rend(); ++it)
            if (*it != vertex && block.dependOn(g.v[*it].block)) g.add_edge(*it, vertex);
        set<size_t> connecting_freed;
        if (!block.isInstr()) {
            for (const bh_base *base : block.getLoop().getAllFrees()) {
                set<size_t> &vs = base2vertices[base];
                connecting_freed.insert(vs.begin(), vs.end());
                vs.insert(vertex);
            }
        }
        for (auto it = connecting_freed.rbegin(); it != connecting_freed.rend(); ++it)
            if (*it != vertex) g.add_edge(*it, vertex);
    }
    return g;
}

// Depth-first topological order (finish order reversed), visiting vertices and out-edges in order.
vector<Block> fill_block_list(const DAG &g) {
    vector<size_t> finished;
    vector<char> state(g.v.size(), 0);
    for (size_t s = 0; s < g.v.size(); ++s) {
        if (!g.v[s].alive || state[s]) continue;
        vector<pair<size_t, set<size_t>::const_iterator>> stack;
        state[s] = 1;
        stack.emplace_back(s, g.v[s].out.begin());
        while (!stack.empty()) {
            auto &top = stack.back();
            if (top.second != g.v[top.first].out.end()) {
                const size_t w = *top.second;
                ++top.second;
                if (!state[w]) {
                    state[w] = 1;
                    stack.emplace_back(w, g.v[w].out.begin());
                }
            } else {
                finished.push_back(top.first);
                stack.pop_back();
            }
        }
    }
    vector<Block> ret;
    for (auto it = finished.rbegin(); it != finished.rend(); ++it) ret.push_back(g.v[*it].block);
    return ret;
}

void merge_vertices(DAG &g, size_t a, size_t b, bool remove_b) {
    g.v[a].block = reshape_and_merge(g.v[a].block.getLoop(), g.v[b].block.getLoop());
    const set<size_t> children = g.v[b].out, parents = g.v[b].in;
    for (size_t c : children) g.add_edge(a, c);
    for (size_t p : parents)
        if (p != a) g.add_edge(p, a);
    if (remove_b) {
        g.remove_vertex(b);
    } else {
        g.clear_vertex(b);
    }
}

// Remove transitive edges and return the mergeable ones (core/jitk/graph.cpp:319-342).
vector<pair<size_t, size_t>> fusible_edges(DAG &g, bool avoid_rank0_sweep) {
    vector<pair<size_t, size_t>> fusibles;
    for (const auto &e : g.edges()) {
        if (g.long_path_exist(e.first, e.second)) {
            g.remove_edge(e.first, e.second);
        } else if (mergeable(g.v[e.first].block, g.v[e.second].block, avoid_rank0_sweep)) {
            fusibles.push_back(e);
        }
    }
    return fusibles;
}

void greedy(DAG &g, bool avoid_rank0_sweep) {
    while (true) {
        const auto fusibles = fusible_edges(g, avoid_rank0_sweep);
        if (fusibles.empty()) break;
        auto greatest = fusibles.front();
        uint64_t greatest_weight = merge_weight(g.v[greatest.first].block, g.v[greatest.second].block);
        for (const auto &e : fusibles) {
            const uint64_t w = merge_weight(g.v[e.first].block, g.v[e.second].block);
            if (w > greatest_weight) {
                greatest = e;
                greatest_weight = w;
            }
        }
        merge_vertices(g, greatest.first, greatest.second, true);
    }
}

// Topological traversal that greedily fuses root vertices (core/jitk/graph.hpp:63-139).
// `pick` chooses the next root from the candidate set.
// The queue either is FIFO (breadth first) or prefers reshapable roots: the last reshapable root in
// vertex order, else the smallest root (core/jitk/fuser.cpp:309-345).
struct RootQueue {
    const DAG &g;
    bool fifo;
    deque<size_t> q;
    set<size_t> all, reshapable;
    RootQueue(const DAG &dag, bool f) : g(dag), fifo(f) {}
    void push(size_t x) {
        if (fifo) {
            q.push_back(x);
        } else if (all.insert(x).second && g.v[x].block.isReshapable()) {
            reshapable.insert(x);
        }
    }
    bool empty() const { return fifo ? q.empty() : all.empty(); }
    size_t pop() {
        size_t r;
        if (fifo) {
            r = q.front();
            q.pop_front();
        } else {
            r = reshapable.empty() ? *all.begin() : *reshapable.rbegin();
            all.erase(r);
            reshapable.erase(r);
        }
        return r;
    }
};

vector<Block> topological(DAG &g, bool avoid_rank0_sweep, bool fifo_queue) {
    vector<Block> ret;
    RootQueue roots(g, fifo_queue);
    auto push = [&](size_t x) { roots.push(x); };
    auto pop = [&]() { return roots.pop(); };
    for (size_t x = 0; x < g.v.size(); ++x)
        if (g.v[x].alive && g.v[x].in.empty()) push(x);
    while (!roots.empty()) {
        const size_t vertex = pop();
        ret.push_back(g.v[vertex].block);
        Block &block = ret.back();
        for (size_t w : g.v[vertex].out)
            if (g.v[w].in.size() <= 1) push(w);
        g.clear_vertex(vertex);
        if (block.isInstr()) continue;
        vector<size_t> nonfusible;
        while (!roots.empty()) {
            const size_t x = pop();
            if (!g.v[x].block.isInstr() && mergeable(block, g.v[x].block, avoid_rank0_sweep)) {
                block = reshape_and_merge(block.getLoop(), g.v[x].block.getLoop());
                for (size_t w : g.v[x].out)
                    if (g.v[w].in.size() <= 1) push(w);
                g.clear_vertex(x);
            } else {
                nonfusible.push_back(x);
            }
        }
        for (size_t x : nonfusible) push(x);
    }
    return ret;
}

} // namespace

uint64_t merge_weight(const Block &b1, const Block &b2) {
    if (b1.isInstr() || b2.isInstr()) return 0;
    const set<bh_base *> news = b1.getLoop().getAllNews();
    const set<bh_base *> frees = b2.getLoop().getAllFrees();
    uint64_t total = 0;
    for (bh_base *b : news)
        if (contains(frees, b)) total += static_cast<uint64_t>(b->nbytes());
    return total;
}

uint64_t block_cost(const Block &block) {
    vector<const bh_base *> non_temps;
    const set<bh_base *> temps = block.isInstr() ? set<bh_base *>() : block.getLoop().getAllTemps();
    for (const InstrPtr &instr : all_instr(block))
        for (const bh_view &v : instr->getViews())
            if (!contains(temps, v.base) && find(non_temps.begin(), non_temps.end(), v.base) == non_temps.end())
                non_temps.push_back(v.base);
    uint64_t total = 0;
    for (const bh_base *b : non_temps) total += static_cast<uint64_t>(b->nbytes());
    return total;
}

void fuser_breadth_first(vector<Block> &block_list, bool avoid_rank0_sweep) {
    DAG g = from_block_list(block_list);
    vector<Block> ret = topological(g, avoid_rank0_sweep, true);
    for (Block &b : ret)
        if (!b.isInstr()) fuser_breadth_first(b.getLoop()._block_list, false);
    block_list = ret;
}

void fuser_reshapable_first(vector<Block> &block_list, bool avoid_rank0_sweep) {
    DAG g = from_block_list(block_list);
    vector<Block> ret = topological(g, avoid_rank0_sweep, false);
    for (Block &b : ret)
        if (!b.isInstr()) fuser_reshapable_first(b.getLoop()._block_list, false);
    block_list = ret;
}

void fuser_greedy(const FusionConfig &config, vector<Block> &block_list) {
    DAG g = from_block_list(block_list);
    if (g.num_edges() > config.greedy_threshold) {
        fuser_reshapable_first(block_list, config.avoid_rank0_sweep);
        return;
    }
    greedy(g, config.avoid_rank0_sweep);
    vector<Block> ret = fill_block_list(g);
    for (Block &b : ret)
        if (!b.isInstr()) fuser_greedy(config, b.getLoop()._block_list);
    block_list = ret;
}

void fuser_chosen(const FusionConfig &config, vector<Block> &block_list, const MergeChooser &chooser) {
    DAG g = from_block_list(block_list);
    if (g.num_edges() > config.greedy_threshold) {
        fuser_reshapable_first(block_list, config.avoid_rank0_sweep);
        return;
    }
    while (true) {
        const auto fusibles = fusible_edges(g, config.avoid_rank0_sweep);
        if (fusibles.empty()) break;
        vector<pair<const Block *, const Block *>> cands;
        for (const auto &e : fusibles) cands.emplace_back(&g.v[e.first].block, &g.v[e.second].block);
        const int pick = chooser(cands);
        if (pick < 0 || pick >= static_cast<int>(fusibles.size())) break;
        merge_vertices(g, fusibles[pick].first, fusibles[pick].second, true);
    }
    vector<Block> ret = fill_block_list(g);
    for (Block &b : ret)
        if (!b.isInstr()) fuser_greedy(config, b.getLoop()._block_list);
    block_list = ret;
}

// ----------------------------------------------------------------------------------- transformers
namespace {
vector<InstrPtr> swap_axis(const vector<InstrPtr> &instr_list, int64_t axis1, int64_t axis2) {
    vector<InstrPtr> ret;
    for (const InstrPtr &instr : instr_list) {
        bh_instruction tmp(*instr);
        tmp.transpose(axis1, axis2);
        ret.push_back(make_shared<bh_instruction>(tmp));
    }
    return ret;
}

vector<Block> swap_blocks(const LoopB &parent, const LoopB *child) {
    vector<Block> ret;
    for (const Block &b : parent._block_list) {
        LoopB loop;
        loop.rank = parent.rank;
        if (b.isInstr() || &b.getLoop() != child) {
            loop.size = parent.size;
            loop._block_list.push_back(b);
            loop._frees.insert(parent._frees.begin(), parent._frees.end());
        } else {
            loop.size = child->size;
            const vector<InstrPtr> t = swap_axis(all_instr(*child), parent.rank, child->rank);
            loop._block_list.push_back(create_nested_block(t, child->rank, parent.size));
            loop._frees.insert(child->_frees.begin(), child->_frees.end());
        }
        loop.metadataUpdate();
        ret.emplace_back(std::move(loop));
    }
    return ret;
}

const LoopB *find_swappable_sub_block(const LoopB &parent) {
    // Iterate the sweeps in origin order so the choice does not depend on pointer values.
    vector<InstrPtr> sweeps(parent._sweeps.begin(), parent._sweeps.end());
    sort(sweeps.begin(), sweeps.end(), [](const InstrPtr &a, const InstrPtr &b) { return a->origin_id < b->origin_id; });
    for (const InstrPtr &sweep : sweeps) {
        for (const Block &b : parent._block_list) {
            if (b.isInstr()) continue;
            for (const Block &ib : b.getLoop()._block_list)
                if (ib.isInstr() && *ib.getInstr() == *sweep) return &b.getLoop();
        }
    }
    return nullptr;
}

bool collapse_instr_axes(LoopB &loop, const int axis) {
    for (Block &block : loop._block_list) {
        if (block.isInstr()) {
            bh_instruction instr(*block.getInstr());
            const int sa = instr.sweep_axis();
            if (sa == axis || sa == axis + 1) return false;
            for (size_t i = 0; i < instr.operand.size(); ++i) {
                bh_view &view = instr.operand[i];
                if (view.isConstant()) continue;
                int ax = axis;
                if (i == 0 && bh_opcode_is_reduction(instr.opcode)) ax = sa < ax ? ax - 1 : ax;
                if (view.ndim <= ax + 1) return false;
                if (view.shape[ax + 1] * view.stride[ax + 1] != view.stride[ax]) return false;
                view.shape[ax] *= view.shape[ax + 1];
                view.stride[ax] = view.stride[ax + 1];
            }
            instr.remove_axis(axis + 1);
            block.setInstr(instr);
        } else {
            --block.getLoop().rank;
            if (!collapse_instr_axes(block.getLoop(), axis)) return false;
        }
    }
    loop.metadataUpdate();
    return true;
}

bool collapse_loop_with_child(LoopB &loop) {
    if (loop._sweeps.empty() && loop._block_list.size() == 1 && loop._reshapable) {
        Block &child = loop._block_list[0];
        if (!child.isInstr() && child.getLoop()._sweeps.empty() && child.getLoop()._reshapable) {
            loop.size *= child.getLoop().size;
            loop._frees.insert(child.getLoop()._frees.begin(), child.getLoop()._frees.end());
            auto tmp = std::move(child.getLoop()._block_list);
            loop._block_list = std::move(tmp);
            return collapse_instr_axes(loop, loop.rank);
        }
    }
    return false;
}
} // namespace

void push_reductions_inwards(vector<Block> &block_list) {
    vector<Block> list2(block_list);
    for (Block &b : list2)
        if (!b.isInstr()) push_reductions_inwards(b.getLoop()._block_list);
    vector<Block> ret;
    for (const Block &b : list2) {
        const LoopB *swappable = nullptr;
        if (!b.isInstr() && (swappable = find_swappable_sub_block(b.getLoop())) != nullptr) {
            const vector<Block> tmp = swap_blocks(b.getLoop(), swappable);
            ret.insert(ret.end(), tmp.begin(), tmp.end());
        } else {
            ret.push_back(b);
        }
    }
    block_list = ret;
}

void split_for_threading(vector<Block> &block_list, uint64_t min_threading) {
    vector<Block> ret;
    for (const Block &block : block_list) {
        if (block.isInstr() || !block.getLoop()._sweeps.empty()) {
            ret.push_back(block);
            continue;
        }
        const LoopB &loop = block.getLoop();
        uint64_t max_nelem = 0;
        for (const InstrPtr &instr : all_instr(loop)) {
            if (!instr->operand.empty())
                max_nelem = max(max_nelem, static_cast<uint64_t>(instr->operand[0].shape.prod()));
        }
        if (loop._block_list.size() > 1 && max_nelem > min_threading && parallel_ranks(loop).second < min_threading) {
            for (auto it = loop._block_list.begin(); it != loop._block_list.end(); ++it) {
                {
                    LoopB newloop{loop.rank, loop.size};
                    while (it != loop._block_list.end() && (it->isInstr() || !it->getLoop()._sweeps.empty())) {
                        newloop._block_list.push_back(*it);
                        ++it;
                    }
                    if (!newloop._block_list.empty()) {
                        newloop.metadataUpdate();
                        ret.push_back(Block(std::move(newloop)));
                    }
                }
                if (it != loop._block_list.end()) {
                    LoopB newloop{loop.rank, loop.size};
                    newloop._block_list.push_back(*it);
                    newloop.metadataUpdate();
                    ret.push_back(Block(std::move(newloop)));
                }
                ret.back().getLoop()._frees = loop._frees;
                if (it == loop._block_list.end()) break;
            }
        } else {
            ret.push_back(block);
        }
    }
    block_list = ret;
}

void collapse_redundant_axes(vector<Block> &block_list) {
    for (Block &b : block_list)
        if (!b.isInstr()) collapse_redundant_axes(b.getLoop()._block_list);
    vector<Block> ret;
    for (const Block &block : block_list) {
        if (!block.isInstr()) {
            Block b(block);
            if (collapse_loop_with_child(b.getLoop())) {
                ret.push_back(std::move(b));
            } else {
                ret.push_back(block);
            }
        } else {
            ret.push_back(block);
        }
    }
    block_list = ret;
}

// ------------------------------------------------------------------------------- kernel assembly
namespace {
vector<InstrPtr> order_sweep_by_origin_id(const set<InstrPtr> &sweep_set) {
    vector<InstrPtr> ret(sweep_set.begin(), sweep_set.end());
    sort(ret.begin(), ret.end(), [](const InstrPtr &a, const InstrPtr &b) { return a->origin_id > b->origin_id; });
    return ret;
}

bh_instruction make_identity(const InstrPtr &sweep, int64_t &origin_count) {
    bh_instruction identity(BH_IDENTITY, {sweep->operand[0]});
    identity.operand.resize(2);
    identity.operand[1].base = nullptr;
    identity.constant = sweep_identity(sweep->opcode, sweep->operand[0].base->dtype());
    identity.origin_id = origin_count++;
    identity.constructor = sweep->constructor;
    // Accumulates run serially along the swept axis: only its first element is the identity.
    if (bh_opcode_is_accumulate(sweep->opcode)) identity.operand[0].shape[sweep->sweep_axis()] = 1;
    return identity;
}

// Insert identity instructions in front of every swept sub-block (core/jitk/apply_fusion.cpp:87-129).
void add_identity_block(LoopB &loop, int64_t &origin_count) {
    vector<Block> ret;
    for (Block &block : loop._block_list) {
        if (block.isInstr()) {
            ret.push_back(block);
            continue;
        }
        add_identity_block(block.getLoop(), origin_count);
        for (const InstrPtr &sweep : order_sweep_by_origin_id(block.getLoop().getSweeps())) {
            const bh_instruction identity = make_identity(sweep, origin_count);
            if (loop.rank == -1 && sweep->operand[0].is_scalar()) {
                ret.emplace_back(identity, 0);
            } else if (loop.rank == sweep->operand[0].ndim - 1) {
                ret.emplace_back(identity, static_cast<int>(sweep->operand[0].ndim));
            } else {
                ret.push_back(create_nested_block({make_shared<const bh_instruction>(identity)}, loop.rank + 1));
            }
            bh_instruction updated{*sweep};
            updated.constructor = false;
            block.getLoop().replaceInstr(sweep, updated);
            block.getLoop().metadataUpdate();
        }
        ret.push_back(block);
    }
    loop._block_list = ret;
    loop.metadataUpdate();
}

vector<LoopB> add_identity_block(vector<Block> &block_list, int64_t &origin_count) {
    vector<LoopB> ret;
    for (Block &block : block_list) {
        add_identity_block(block.getLoop(), origin_count);
        LoopB kernel{-1, 1};
        for (const InstrPtr &sweep : order_sweep_by_origin_id(block.getLoop().getSweeps())) {
            const bh_instruction identity = make_identity(sweep, origin_count);
            if (sweep->operand[0].is_scalar()) {
                kernel._block_list.emplace_back(identity, 0);
            } else {
                kernel._block_list.push_back(create_nested_block({make_shared<const bh_instruction>(identity)}, 0));
            }
            bh_instruction updated{*sweep};
            updated.constructor = false;
            block.getLoop().replaceInstr(sweep, updated);
            block.getLoop().metadataUpdate();
        }
        kernel._block_list.push_back(block);
        kernel.metadataUpdate();
        ret.emplace_back(std::move(kernel));
    }
    return ret;
}
} // namespace

vector<Block> fuse_block_list(const vector<bh_instruction *> &instr_list, const FusionConfig &config,
                              const MergeChooser *chooser) {
    const MixedSweepRule rule(config.avoid_mixed_sweeps);
    vector<Block> block_list;
    if (config.pre_fuser == "none" || config.pre_fuser == "singleton") {
        block_list = fuser_singleton(instr_list);
    } else if (config.pre_fuser == "lossy" || config.pre_fuser == "pre_fuser_lossy") {
        block_list = pre_fuser_lossy(instr_list);
    } else {
        throw runtime_error("Unknown pre-fuser: \"" + config.pre_fuser + "\"");
    }
    for (const string &t : config.fuser_list) {
        if (t == "push_reductions_inwards") {
            push_reductions_inwards(block_list);
        } else if (t == "split_for_threading") {
            split_for_threading(block_list);
        } else if (t == "collapse_redundant_axes") {
            collapse_redundant_axes(block_list);
        } else if (t == "serial") {
            fuser_serial(block_list, config.avoid_rank0_sweep);
        } else if (t == "breadth_first") {
            fuser_breadth_first(block_list, config.avoid_rank0_sweep);
        } else if (t == "reshapable_first") {
            fuser_reshapable_first(block_list, config.avoid_rank0_sweep);
        } else if (t == "greedy") {
            fuser_greedy(config, block_list);
        } else if (t == "learned") {
            if (chooser != nullptr) {
                fuser_chosen(config, block_list, *chooser);
            } else {
                fuser_greedy(config, block_list);
            }
        } else {
            throw runtime_error("Unknown transformer: \"" + t + "\"");
        }
    }
    return block_list;
}

vector<LoopB> get_kernel_list(const vector<bh_instruction *> &instr_list, const FusionConfig &config,
                              const vector<Block> *cached_block_list, vector<Block> *block_list_out,
                              const MergeChooser *chooser) {
    int64_t origin_count = 0;
    for (bh_instruction *instr : instr_list) instr->origin_id = origin_count++;
    vector<Block> block_list =
        cached_block_list != nullptr ? *cached_block_list : fuse_block_list(instr_list, config, chooser);
    if (block_list_out != nullptr) *block_list_out = block_list;
    vector<LoopB> ret;
    if (config.avoid_rank0_sweep) {
        for (Block &b : block_list) {
            if (b.isInstr() || !b.getLoop()._sweeps.empty()) {
                ret.emplace_back(LoopB{-1, 1, {std::move(b)}});
            } else {
                LoopB kernel{-1, 1, {std::move(b)}};
                add_identity_block(kernel, origin_count);
                ret.emplace_back(std::move(kernel));
            }
        }
    } else if (config.monolithic) {
        LoopB kernel{-1, 1, std::move(block_list)};
        add_identity_block(kernel, origin_count);
        ret = {std::move(kernel)};
    } else {
        ret = add_identity_block(block_list, origin_count);
    }
    return ret;
}

} // namespace jitk
} // namespace bohrium
