// Learned fusion: the cost model's use inside the engine.
//
// - Recording: with `record` on, every kernel of a flush runs alone between two events and its
//   feature vector (jitk::block_features) and device time are appended to `records`; the rows
//   are the training set of the cost model (bohrium_b200/costmodel.py trains it with the GPU
//   kernels of mlp.cu).
// - Choosing merges: the learned transformer (jitk::fuser_chosen) asks choose_merge() for the next
//   merge among the legal ones (mergeable(), the plain rule). Every candidate (a, b) is scored by
//   the predicted gain t(a) + t(b) - t(a merged with b), all predictions of one step computed in
//   one batched inference on the GPU; the best positive gain is merged, none stops the fuser.
// - Keeping a plan: a learned plan is tried only when its floating-point sums and products fold
//   in the same order as in the greedy plan (so every output is bit-identical to the greedy
//   form); both plans are timed on the device and the faster one stays for the structure.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <cuda_runtime.h>
#include <bh_b200.h>
#include "engine.hpp"

using namespace std;
using namespace bohrium::jitk;

namespace bohrium {
namespace cuda {

namespace {

void check_cuda(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw runtime_error(string("[CUDA] ") + what + ": " + cudaGetErrorString(e));
}

uint64_t mix(uint64_t h, uint64_t v) {
    h ^= v + 0x9E3779B97F4A7C15ULL + (h << 6) + (h >> 2);
    return h * 0xBF58476D1CE4E5B9ULL;
}

// Structural key of a block within one fusion: its loops (rank, size) and instructions (origin id).
uint64_t block_key(const Block &b) {
    if (b.isInstr()) return mix(0x1234567ULL, static_cast<uint64_t>(b.getInstr()->origin_id));
    const LoopB &l = b.getLoop();
    uint64_t h = mix(static_cast<uint64_t>(l.rank) + 77, static_cast<uint64_t>(l.size));
    for (const Block &c : l._block_list) h = mix(h, block_key(c));
    return h;
}

} // namespace

string EngineCUDA::FlushPlan::signature() const {
    string s;
    for (const PlanKernel &pk : kernels) {
        s += to_string(pk.level) + ":";
        for (const PlanUnit &pu : pk.units) s += pu.unit.name + ",";
        s += ";";
    }
    return s;
}

void EngineCUDA::load_costmodel(const string &path) {
    ifstream f(path, ios::binary);
    if (!f) throw runtime_error("cost model: cannot open " + path);
    char magic[8];
    f.read(magic, 8);
    if (!f || memcmp(magic, "BHCM0001", 8) != 0) throw runtime_error("cost model: " + path + " is not a model file");
    int32_t nf = 0, np = 0;
    f.read(reinterpret_cast<char *>(&nf), 4);
    f.read(reinterpret_cast<char *>(&np), 4);
    if (!f || nf != kCostFeatures || nf != bh_ve_cuda_costmodel_nfeatures() || np != bh_ve_cuda_costmodel_nparams())
        throw runtime_error("cost model: " + path + " has the wrong shape");
    vector<float> mean(static_cast<size_t>(nf)), sd(static_cast<size_t>(nf)), params(static_cast<size_t>(np));
    float tm = 0.f, ts = 1.f;
    f.read(reinterpret_cast<char *>(mean.data()), 4 * nf);
    f.read(reinterpret_cast<char *>(sd.data()), 4 * nf);
    f.read(reinterpret_cast<char *>(&tm), 4);
    f.read(reinterpret_cast<char *>(&ts), 4);
    f.read(reinterpret_cast<char *>(params.data()), 4 * static_cast<std::streamsize>(np));
    if (!f) throw runtime_error("cost model: " + path + " is truncated");
    if (cm == nullptr) {
        cm = bh_ve_cuda_costmodel_create(0);
        if (cm == nullptr) throw runtime_error(string("cost model: ") + bhb_last_error());
    }
    if (bh_ve_cuda_costmodel_set_params(cm, params.data()) != 0)
        throw runtime_error(string("cost model: ") + bhb_last_error());
    cm_mean = std::move(mean);
    cm_std = std::move(sd);
    cm_tmean = tm;
    cm_tstd = ts;
    // Decisions taken with another model (or none) are void.
    decided.clear();
    trials.clear();
}

void EngineCUDA::set_fusion(const string &pre_fuser, const string &fuser_list) {
    if (!pre_fuser.empty()) fusion_config.pre_fuser = pre_fuser;
    if (!fuser_list.empty()) {
        vector<string> names;
        string cur;
        for (char c : fuser_list + ",") {
            if (c == ',' || c == ' ') {
                if (!cur.empty()) names.push_back(cur);
                cur.clear();
            } else {
                cur += c;
            }
        }
        fusion_config.fuser_list = names;
    }
    synchronize();
    fuse_cache.clear();
    replays.clear();
    plans.clear();
    trials.clear();
    decided.clear();
}

size_t EngineCUDA::dump_records(const string &path) const {
    ofstream f(path, ios::binary);
    if (!f) throw runtime_error("records: cannot write " + path);
    f.write(reinterpret_cast<const char *>(records.data()), static_cast<std::streamsize>(records.size() * 4));
    return record_count();
}

void EngineCUDA::record_kernel_times(const FlushPlan &plan, const vector<bh_base *> &bases,
                                     const vector<bh_instruction *> &instrs) {
    cudaStream_t s = static_cast<cudaStream_t>(_stream);
    if (rec_e0 == nullptr) {
        cudaEvent_t a, b;
        check_cuda(cudaEventCreate(&a), "cudaEventCreate");
        check_cuda(cudaEventCreate(&b), "cudaEventCreate");
        rec_e0 = a;
        rec_e1 = b;
    }
    for (const PlanKernel &pk : plan.kernels) {
        ++_stats.kernels;
        if (!pk.units.empty()) {
            check_cuda(cudaEventRecord(static_cast<cudaEvent_t>(rec_e0), s), "cudaEventRecord");
            for (const PlanUnit &pu : pk.units) launch_plain(pu, bases, instrs);
            check_cuda(cudaEventRecord(static_cast<cudaEvent_t>(rec_e1), s), "cudaEventRecord");
            check_cuda(cudaEventSynchronize(static_cast<cudaEvent_t>(rec_e1)), "cudaEventSynchronize");
            float ms = 0.f;
            check_cuda(cudaEventElapsedTime(&ms, static_cast<cudaEvent_t>(rec_e0), static_cast<cudaEvent_t>(rec_e1)),
                       "cudaEventElapsedTime");
            records.insert(records.end(), pk.feat.begin(), pk.feat.end());
            records.push_back(ms * 1000.f);
        }
        for (int w : pk.writes) host_stale.insert(bases[static_cast<size_t>(w)]);
        for (int f : pk.frees) free_base(bases[static_cast<size_t>(f)]);
    }
}

void EngineCUDA::predict_us(const vector<CostFeatures> &rows, vector<float> &out) {
    out.assign(rows.size(), 0.f);
    if (rows.empty()) return;
    vector<float> x(rows.size() * kCostFeatures);
    for (size_t r = 0; r < rows.size(); ++r)
        for (int f = 0; f < kCostFeatures; ++f)
            x[r * kCostFeatures + static_cast<size_t>(f)] =
                (rows[r][static_cast<size_t>(f)] - cm_mean[static_cast<size_t>(f)]) / cm_std[static_cast<size_t>(f)];
    vector<float> y(rows.size());
    if (bh_ve_cuda_costmodel_predict(cm, x.data(), static_cast<int64_t>(rows.size()), y.data()) != 0)
        throw runtime_error(string("cost model: ") + bhb_last_error());
    _stats.learned_predictions += rows.size();
    for (size_t r = 0; r < rows.size(); ++r) out[r] = std::exp(y[r] * cm_tstd + cm_tmean);
}

int EngineCUDA::choose_merge(const vector<pair<const Block *, const Block *>> &cands) {
    if (cands.empty() || cm == nullptr) return -1;
    const auto t0 = chrono::steady_clock::now();
    struct Timer {  // the model's share of the learned contraction: features, inference, choice
        double &acc;
        chrono::steady_clock::time_point t0;
        ~Timer() { acc += chrono::duration<double>(chrono::steady_clock::now() - t0).count(); }
    } timer{_stats.time_learned_choose, t0};
    // Keys of every block involved and of every merged pair; predict what is not cached yet.
    vector<uint64_t> ka(cands.size()), kb(cands.size()), km(cands.size());
    vector<CostFeatures> rows;
    vector<uint64_t> pending;
    auto want = [&](uint64_t key, const Block &b) {
        if (pred_cache.count(key) || find(pending.begin(), pending.end(), key) != pending.end()) return;
        rows.push_back(block_features(b));
        pending.push_back(key);
    };
    for (size_t i = 0; i < cands.size(); ++i) {
        const Block &a = *cands[i].first, &b = *cands[i].second;
        ka[i] = block_key(a);
        kb[i] = block_key(b);
        km[i] = mix(mix(ka[i], 0xA11CEULL), kb[i]);
        want(ka[i], a);
        want(kb[i], b);
        if (!pred_cache.count(km[i]) && find(pending.begin(), pending.end(), km[i]) == pending.end()) {
            if (a.isInstr() || b.isInstr()) {
                pred_cache[km[i]] = 1e30f;  // never chosen
            } else {
                rows.push_back(block_features(reshape_and_merge(a.getLoop(), b.getLoop())));
                pending.push_back(km[i]);
            }
        }
    }
    vector<float> pred;
    predict_us(rows, pred);
    for (size_t r = 0; r < pending.size(); ++r) pred_cache[pending[r]] = pred[r];
    int best = -1;
    double best_gain = learned_min_gain_us;
    for (size_t i = 0; i < cands.size(); ++i) {
        const double gain = static_cast<double>(pred_cache[ka[i]]) + pred_cache[kb[i]] - pred_cache[km[i]];
        if (gain > best_gain) {
            best_gain = gain;
            best = static_cast<int>(i);
        }
    }
    return best;
}

bool EngineCUDA::start_trial(uint64_t key, vector<bh_instruction *> &instr_list, const vector<bh_base *> &base_ids,
                             FlushPlan &greedy) {
    const auto t0 = chrono::steady_clock::now();
    FusionConfig cfg = fusion_config;
    bool has_greedy = false;
    for (string &t : cfg.fuser_list) {
        if (t == "greedy") {
            t = "learned";
            has_greedy = true;
        }
    }
    if (!has_greedy) {
        decided.insert(key);
        return false;
    }
    pred_cache.clear();
    const vector<LoopB> kernels = get_kernel_list(instr_list, cfg, nullptr, nullptr, &chooser);
    FlushPlan learned = build_plan(kernels, base_ids);
    learned.nbases = base_ids.size();
    _stats.time_learned_fusion += chrono::duration<double>(chrono::steady_clock::now() - t0).count();
    if (learned.signature() == greedy.signature()) {
        ++_stats.learned_same;
        decided.insert(key);
        return false;
    }
    if (learned.orders != greedy.orders) {
        ++_stats.learned_order_differs;
        decided.insert(key);
        return false;
    }
    ++_stats.learned_trials;
    Trial &t = trials[key];
    t.greedy = std::move(greedy);
    t.learned = std::move(learned);
    return true;
}

void EngineCUDA::run_trial(uint64_t key, Trial &t, const vector<bh_base *> &bases, const vector<bh_instruction *> &instrs) {
    // Greedy first, then alternate; each run timed alone on the engine's stream.
    const bool use_learned = t.t_learned.size() < t.t_greedy.size();
    const FlushPlan &plan = use_learned ? t.learned : t.greedy;
    cudaStream_t s = static_cast<cudaStream_t>(_stream);
    if (rec_e0 == nullptr) {
        cudaEvent_t a, b;
        check_cuda(cudaEventCreate(&a), "cudaEventCreate");
        check_cuda(cudaEventCreate(&b), "cudaEventCreate");
        rec_e0 = a;
        rec_e1 = b;
    }
    float ms = 0.f;
    // The autotuner's variant rotation would distort the comparison: trials use the variants in
    // place, and tuning resumes once the plan is chosen.
    const bool tune = autotune;
    autotune = false;
    if (batch_mode == "graph") {
        // Replays will run as a CUDA graph without launch gaps: compare device busy time.
        busy_timing = true;
        busy_used = 0;
        run_plan(plan, bases, instrs);
        busy_timing = false;
        ms = static_cast<float>(busy_ms());
    } else {
        check_cuda(cudaEventRecord(static_cast<cudaEvent_t>(rec_e0), s), "cudaEventRecord");
        run_plan(plan, bases, instrs);
        check_cuda(cudaEventRecord(static_cast<cudaEvent_t>(rec_e1), s), "cudaEventRecord");
        check_cuda(cudaEventSynchronize(static_cast<cudaEvent_t>(rec_e1)), "cudaEventSynchronize");
        check_cuda(cudaEventElapsedTime(&ms, static_cast<cudaEvent_t>(rec_e0), static_cast<cudaEvent_t>(rec_e1)),
                   "cudaEventElapsedTime");
    }
    autotune = tune;
    (use_learned ? t.t_learned : t.t_greedy).push_back(ms);
    const size_t runs = static_cast<size_t>(max(learned_runs, 1));
    if (t.t_greedy.size() >= runs && t.t_learned.size() >= runs) {
        const double g = *min_element(t.t_greedy.begin(), t.t_greedy.end());
        const double l = *min_element(t.t_learned.begin(), t.t_learned.end());
        if (l < g * (1.0 - learned_margin)) {
            ++_stats.learned_kept;
            plans[key] = std::move(t.learned);
        } else {
            ++_stats.greedy_kept;
            plans[key] = std::move(t.greedy);
        }
        decided.insert(key);
        trials.erase(key);
    }
}

} // namespace cuda
} // namespace bohrium
