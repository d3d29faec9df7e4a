// CUDA-graph replay of repeated flushes (batch mode "graph").
//
// A fingerprinted BhIR (one compiled once and executed many times) first runs through the plan
// cache as usual. From its second valid replay on, its launches -- grouped exactly as the
// "grouped" mode groups them, with the same work functions and the same scratch offsets -- are
// packed once and captured into a CUDA graph:
//   - buffers of arrays that the flush creates and frees again are parked: the graph owns them,
//     so a replay neither allocates nor frees;
//   - every other array's device buffer is looked up once and recorded; the graph is relaunched
//     only while all of them (and the scratch and counter arenas) still have those addresses,
//     otherwise it is dropped and the flush runs through the plan again;
//   - the parameter blocks of grouped launches live in a device block the graph owns.
// A replay is then one cudaGraphLaunch plus the host bookkeeping of which host copies are stale.
// The kernels are the plan's kernels, so results are bit-identical to the plain launches.
#include <cstring>
#include <map>
#include <stdexcept>
#include <cuda.h>
#include <cuda_runtime.h>
#include "engine.hpp"

using namespace std;

namespace bohrium {
namespace cuda {

namespace {
void check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw runtime_error(string("[CUDA] ") + what + ": " + cudaGetErrorString(e));
}
} // namespace

EngineCUDA::ReplayGraph::~ReplayGraph() {
    if (stream) cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    if (exec) cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(exec));
    if (graph) cudaGraphDestroy(static_cast<cudaGraph_t>(graph));
    if (params_dev) cudaFree(params_dev);
    for (void *p : parked) cudaFree(p);
}

namespace {

struct GLaunch {
    void *fn = nullptr;
    int64_t grid = 1;
    bool batched = false;
    vector<uint8_t> params;  // plain: the parameter struct; batched: items then prefix sums
    size_t items_bytes = 0;  // batched: offset of the prefix sums
    size_t dev_off = 0;      // batched: offset in the graph's parameter block
    int nitems = 0;
    int64_t total = 0;
};

} // namespace

bool EngineCUDA::graph_usable(const ReplayGraph &g) const {
    if (g.scratch != scratch || g.counters != counters || g.scan_arena != scan_arena) return false;
    for (const auto &bp : g.persistent) {
        auto it = buffers.find(bp.first);
        if (it == buffers.end() || it->second.ptr != bp.second) return false;
    }
    return true;
}

void EngineCUDA::graph_launch(ReplayGraph &g) {
    for (const auto &bp : g.persistent) {
        auto it = buffers.find(bp.first);
        if (it != buffers.end()) settle(it->second);
    }
    check(cudaGraphLaunch(static_cast<cudaGraphExec_t>(g.exec), static_cast<cudaStream_t>(_stream)), "cudaGraphLaunch");
    if (g.stale_epoch != stale_epoch) {
        for (bh_base *b : g.written) host_stale.insert(b);
        g.stale_epoch = stale_epoch;
    }
    _stats.launches += g.nlaunches;
    ++_stats.graph_replays;
}

bool EngineCUDA::build_graph(Replay &r) {
    const FlushPlan &plan = *r.plan;
    const vector<bh_base *> &bases = r.base_ids;
    const vector<bh_instruction *> &instrs = r.instrs;
    unique_ptr<ReplayGraph> g(new ReplayGraph());
    g->stream = _stream;

    // Which arrays the launches address, and which the flush frees again (flush-local).
    vector<char> used(bases.size(), 0), local(bases.size(), 0), written(bases.size(), 0);
    for (const PlanKernel &pk : plan.kernels) {
        for (const PlanUnit &pu : pk.units)
            for (int idx : pu.ptr_base)
                if (idx >= 0) used[static_cast<size_t>(idx)] = 1;
        for (int f : pk.frees) local[static_cast<size_t>(f)] = 1;
        for (int w : pk.writes) written[static_cast<size_t>(w)] = 1;
    }
    vector<void *> ptr(bases.size(), nullptr);
    for (size_t i = 0; i < bases.size(); ++i) {
        if (!used[i]) continue;
        if (local[i]) {
            const int64_t nb = bases[i]->nbytes();
            if (nb > 0) {
                void *p = nullptr;
                check(cudaMalloc(&p, static_cast<size_t>(nb)), "cudaMalloc(parked)");
                g->parked.push_back(p);
                ptr[i] = p;
            }
        } else {
            ptr[i] = getBuffer(bases[i]);
            g->persistent.emplace_back(bases[i], ptr[i]);
        }
    }
    for (size_t i = 0; i < bases.size(); ++i)
        if (written[i] && !local[i]) g->written.push_back(bases[i]);

    // The launches, grouped as run_plan groups them in "grouped" mode.
    vector<vector<const PlanUnit *>> launches;  // each entry: one plain unit or one group
    if (plan.kernels.size() < 2) {
        for (const PlanKernel &pk : plan.kernels)
            for (const PlanUnit &pu : pk.units) launches.push_back({&pu});
    } else {
        vector<vector<const PlanUnit *>> by_level(static_cast<size_t>(plan.nlevels));
        for (const PlanKernel &pk : plan.kernels)
            for (size_t j = 0; j < pk.units.size(); ++j) by_level[static_cast<size_t>(pk.level) + j].push_back(&pk.units[j]);
        for (const auto &level : by_level) {
            map<const Compiled *, vector<const PlanUnit *>> groups;
            vector<const Compiled *> order;
            for (const PlanUnit *pu : level) {
                if (!groups.count(pu->compiled)) order.push_back(pu->compiled);
                groups[pu->compiled].push_back(pu);
            }
            for (const Compiled *c : order) {
                const auto &g = groups[c];
                if (g.size() > 1 && g[0]->unit.no_batch) {
                    for (const PlanUnit *pu : g) launches.push_back({pu});
                } else {
                    launches.push_back(g);
                }
            }
        }
    }
    // Size the arenas once, then pack every launch.
    int64_t scratch_need = 0, counter_need = 1;
    for (const auto &grp : launches) {
        int64_t s = 0, c = 0;
        for (const PlanUnit *pu : grp) {
            s += grp.size() == 1 ? pu->unit.scratch_bytes() : (pu->unit.scratch_bytes() + 255) / 256 * 256;
            c += pu->unit.counters_needed();
        }
        scratch_need = max(scratch_need, s);
        counter_need = max(counter_need, c);
    }
    ensure_scratch(scratch_need);
    ensure_counters(counter_need);
    if (plan.scan_bytes > 0) ensure_scan_arena(plan.scan_bytes);
    ptr_override = &ptr;
    vector<GLaunch> gl;
    size_t dev_bytes = 0;
    try {
        for (const auto &grp : launches) {
            GLaunch L;
            const PlanUnit &proto = *grp[0];
            const size_t psize = proto.unit.fields.size() * 8;
            if (grp.size() == 1) {
                if (proto.unit.work_items() == 0) continue;
                L.fn = proto.compiled->fn;
                L.params.resize(psize);
                pack_params(proto, bases, instrs, 0, 0, L.params.data());
                L.grid = max<int64_t>(1, min<int64_t>(proto.unit.work_items(),
                                                      static_cast<int64_t>(_sm_count) * proto.compiled->occ));
            } else {
                L.batched = true;
                L.fn = proto.compiled->fn_batch;
                const size_t n = grp.size();
                L.items_bytes = (psize * n + 15) / 16 * 16;
                L.params.assign(L.items_bytes + (n + 1) * sizeof(int64_t), 0);
                int64_t *prefix = reinterpret_cast<int64_t *>(L.params.data() + L.items_bytes);
                int64_t soff = 0, coff = 0, total = 0;
                packing_grouped = true;
                for (size_t k = 0; k < n; ++k) {
                    pack_params(*grp[k], bases, instrs, soff, coff, L.params.data() + k * psize);
                    soff += (grp[k]->unit.scratch_bytes() + 255) / 256 * 256;
                    coff += grp[k]->unit.counters_needed();
                    prefix[k] = total;
                    total += grp[k]->unit.grouped_work_items();
                }
                packing_grouped = false;
                prefix[n] = total;
                if (total == 0) continue;
                L.nitems = static_cast<int>(n);
                L.total = total;
                L.grid = max<int64_t>(1, min<int64_t>(total, static_cast<int64_t>(_sm_count) * proto.compiled->occ_batch));
                L.dev_off = dev_bytes;
                dev_bytes += (L.params.size() + 255) / 256 * 256;
            }
            gl.push_back(std::move(L));
        }
    } catch (...) {
        ptr_override = nullptr;
        throw;
    }
    ptr_override = nullptr;
    g->scratch = scratch;
    g->counters = counters;
    g->scan_arena = scan_arena;
    cudaStream_t s = static_cast<cudaStream_t>(_stream);
    if (dev_bytes > 0) {
        check(cudaMalloc(&g->params_dev, dev_bytes), "cudaMalloc(graph params)");
        for (const GLaunch &L : gl)
            if (L.batched)
                check(cudaMemcpy(static_cast<uint8_t *>(g->params_dev) + L.dev_off, L.params.data(), L.params.size(),
                                 cudaMemcpyHostToDevice),
                      "cudaMemcpy(graph params)");
    }
    // Everything the graph reads exists now (uploads above were on the engine's stream).
    synchronize();
    check(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    int launch_err = 0;
    for (const GLaunch &L : gl) {
        if (L.batched) {
            void *items = static_cast<uint8_t *>(g->params_dev) + L.dev_off;
            void *prefix = static_cast<uint8_t *>(items) + L.items_bytes;
            int nitems = L.nitems;
            int64_t total = L.total;
            void *args[] = {&items, &prefix, &nitems, &total};
            launch_err = launch_raw(L.fn, L.grid, args);
        } else {
            void *args[] = {const_cast<uint8_t *>(L.params.data())};
            launch_err = launch_raw(L.fn, L.grid, args);
        }
        if (launch_err != 0) break;
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t end = cudaStreamEndCapture(s, &graph);
    if (launch_err != 0 || end != cudaSuccess || graph == nullptr) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return false;
    }
    cudaGraphExec_t exec = nullptr;
    if (cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
        cudaGraphDestroy(graph);
        cudaGetLastError();
        return false;
    }
    g->graph = graph;
    g->exec = exec;
    g->nlaunches = gl.size();
    r.graph = std::move(g);
    return true;
}

} // namespace cuda
} // namespace bohrium
