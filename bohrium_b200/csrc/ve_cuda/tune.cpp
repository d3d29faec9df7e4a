// Autotuning of launch shapes: register caps.
//
// A kernel with large work (at least `tune_min_elements` elements) is compiled a few more times
// with NVRTC's --maxrregcount below its natural register count (more resident CTAs per SM,
// possibly at the cost of spills), and its first plain launches rotate through the variants,
// each timed alone with CUDA events. After two timings of every variant the fastest one is kept
// for that source, and the choice is written to the kernel cache directory (tune.txt) so that
// later processes start with it. All variants come from the same source and the same options
// but the register cap (FMA contraction off), so they compute bit-identical results.
#include <algorithm>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <cuda.h>
#include <cuda_runtime.h>
#include "engine.hpp"

using namespace std;

namespace bohrium {
namespace cuda {

namespace {
void check_rt(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw runtime_error(string("[CUDA] ") + what + ": " + cudaGetErrorString(e));
}
uint64_t source_hash(const string &s) {
    uint64_t h = 1469598103934665603ULL;
    for (unsigned char c : s) {
        h ^= c;
        h *= 1099511628211ULL;
    }
    return h;
}
} // namespace

void EngineCUDA::load_tune_choices() {
    if (cache_dir.empty()) return;
    ifstream in(cache_dir + "/tune.txt");
    string hex_hash;
    int cap = 0;
    while (in >> hex_hash >> cap) tune_choices[stoull(hex_hash, nullptr, 16)] = cap;
}

void EngineCUDA::save_tune_choice(uint64_t hash, int maxrreg) {
    tune_choices[hash] = maxrreg;
    if (cache_dir.empty()) return;
    ofstream out(cache_dir + "/tune.txt", ios::app);
    out << hex << hash << " " << dec << maxrreg << "\n";
}

bool EngineCUDA::tune_launch(Compiled &c, const LaunchUnit &u, int64_t work, void **args) {
    const uint64_t h = source_hash(c.source);
    if (!c.tuning) {
        c.tuning = true;
        const int regs = c.variants[0].regs;
        for (int cap : {128, 96, 80, 64, 48, 40, 32}) {
            if (cap >= regs || c.variants.size() >= 4) continue;
            c.variants.push_back(load_variant(cubin_for(c.name, c.source, cap), c.name, cap));
        }
        if (c.variants.size() == 1) {
            c.tuned = true;
            save_tune_choice(h, 0);
            return false;
        }
    }
    // The variant with the fewest timings runs next.
    size_t k = 0;
    for (size_t i = 1; i < c.variants.size(); ++i)
        if (c.variants[i].ms.size() < c.variants[k].ms.size()) k = i;
    Compiled::Variant &v = c.variants[k];
    if (rec_e0 == nullptr) {
        cudaEvent_t a, b;
        check_rt(cudaEventCreate(&a), "cudaEventCreate");
        check_rt(cudaEventCreate(&b), "cudaEventCreate");
        rec_e0 = a;
        rec_e1 = b;
    }
    cudaStream_t s = static_cast<cudaStream_t>(_stream);
    const int64_t grid = max<int64_t>(1, min<int64_t>(work, static_cast<int64_t>(_sm_count) * v.occ));
    check_rt(cudaEventRecord(static_cast<cudaEvent_t>(rec_e0), s), "cudaEventRecord");
    if (launch_raw(v.fn, grid, args) != 0) throw runtime_error("cuLaunchKernel (tuning) failed for " + u.name);
    check_rt(cudaEventRecord(static_cast<cudaEvent_t>(rec_e1), s), "cudaEventRecord");
    check_rt(cudaEventSynchronize(static_cast<cudaEvent_t>(rec_e1)), "cudaEventSynchronize");
    float ms = 0.f;
    check_rt(cudaEventElapsedTime(&ms, static_cast<cudaEvent_t>(rec_e0), static_cast<cudaEvent_t>(rec_e1)),
             "cudaEventElapsedTime");
    v.ms.push_back(ms);
    ++_stats.tune_launches;
    bool done = true;
    for (const Compiled::Variant &x : c.variants) done = done && x.ms.size() >= 2;
    if (done) {
        size_t best = 0;
        float best_ms = *min_element(c.variants[0].ms.begin(), c.variants[0].ms.end());
        for (size_t i = 1; i < c.variants.size(); ++i) {
            const float m = *min_element(c.variants[i].ms.begin(), c.variants[i].ms.end());
            if (m < best_ms * 0.98f) {  // a cap has to win clearly
                best = i;
                best_ms = m;
            }
        }
        c.chosen = static_cast<int>(best);
        const Compiled::Variant &b = c.variants[best];
        c.fn = b.fn;
        c.fn_batch = b.fn_batch;
        c.occ = b.occ;
        c.occ_batch = b.occ_batch;
        c.tuned = true;
        ++_stats.tuned_kernels;
        if (b.maxrreg > 0) ++_stats.tuned_capped;
        save_tune_choice(h, b.maxrreg);
    }
    return true;
}

} // namespace cuda
} // namespace bohrium
