// Autotuning of launch shapes: register caps, inner-loop unrolling and CTAs per SM.
//
// A kernel with large work (at least `tune_min_elements` elements) is compiled a few more times:
// with NVRTC's --maxrregcount below its natural register count (more resident CTAs per SM,
// possibly at the cost of spills) and, where the source marks its element loop, with that loop
// unrolled 2 or 4 times (more loads in flight per thread); and its plain launch is also tried with
// half the CTAs per SM that fit, and with one (a smaller persistent grid: less contention on
// shared counters and L2 sets, longer runs per CTA). Its first plain launches rotate through
// the variants, each timed alone with CUDA events. After three timings of every variant the fastest
// one is kept for that source, and the choice is written to the kernel cache directory
// (tune.txt) so that later processes start with it. Register caps and unrolling change neither
// the operations nor their order on any value (FMA contraction is off), so every variant
// computes bit-identical results.
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

const char kUnrollMarker[] = "/*@unroll@*/";
constexpr size_t kTuneSamples = 3;  // timed launches per variant (the fastest counts)

void EngineCUDA::load_tune_choices() {
    if (cache_dir.empty()) return;
    ifstream in(cache_dir + "/tune.txt");
    string line;
    while (getline(in, line)) {
        stringstream ss(line);
        string hex_hash;
        TuneChoice c;
        if (!(ss >> hex_hash >> c.maxrreg >> c.unroll)) continue;
        if (!(ss >> c.ctas)) c.ctas = 0;
        tune_choices[stoull(hex_hash, nullptr, 16)] = c;
    }
}

void EngineCUDA::save_tune_choice(uint64_t hash, int maxrreg, int unroll, int ctas) {
    tune_choices[hash] = TuneChoice{maxrreg, unroll, ctas};
    if (cache_dir.empty()) return;
    ofstream out(cache_dir + "/tune.txt", ios::app);
    out << hex << hash << " " << dec << maxrreg << " " << unroll << " " << ctas << "\n";
}

EngineCUDA::Compiled::Variant EngineCUDA::make_variant(const Compiled &c, int maxrreg, int unroll) {
    string src = c.source;
    if (unroll > 0) {
        const string pragma = "#pragma unroll " + to_string(unroll);
        for (size_t pos = src.find(kUnrollMarker); pos != string::npos; pos = src.find(kUnrollMarker, pos))
            src.replace(pos, sizeof(kUnrollMarker) - 1, pragma);
    }
    Compiled::Variant v = load_variant(cubin_for(c.name, src, maxrreg), c.name, maxrreg, dynamic_shared_bytes(c.source));
    v.unroll = unroll;
    return v;
}

void EngineCUDA::ensure_variants(Compiled &c) {
    if (!c.tuning) {
        c.tuning = true;
        const int regs = c.variants[0].regs;
        vector<int> caps;
        for (int cap : {128, 96, 80, 64, 48, 40, 32})
            if (cap < regs && caps.size() < 2) caps.push_back(cap);
        for (int cap : caps) c.variants.push_back(make_variant(c, cap, 0));
        if (c.source.find(kUnrollMarker) != string::npos) {
            for (int unroll : {2, 4}) c.variants.push_back(make_variant(c, 0, unroll));
            if (!caps.empty()) c.variants.push_back(make_variant(c, caps.back(), 4));
        }
        // Launch shape: fewer resident CTAs per SM than fit (the same code, a smaller grid).
        const int occ = c.variants[0].occ;
        for (int ctas : {occ / 2, 1}) {
            if (ctas < 1 || ctas >= occ) continue;
            Compiled::Variant v = c.variants[0];
            v.ms.clear();
            v.ms_batch.clear();
            v.ctas = ctas;
            bool dup = false;
            for (const Compiled::Variant &x : c.variants) dup = dup || (x.maxrreg == 0 && x.unroll == 0 && x.ctas == ctas);
            if (!dup) c.variants.push_back(v);
        }
    }
}

namespace {
// Time one launch of `fn` alone on `stream` (milliseconds).
float time_launch(EngineCUDA &e, void *&e0, void *&e1, void *stream, void *fn, int64_t grid, void **args,
                  int (EngineCUDA::*launch)(void *, int64_t, void **)) {
    if (e0 == nullptr) {
        cudaEvent_t a, b;
        check_rt(cudaEventCreate(&a), "cudaEventCreate");
        check_rt(cudaEventCreate(&b), "cudaEventCreate");
        e0 = a;
        e1 = b;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    check_rt(cudaEventRecord(static_cast<cudaEvent_t>(e0), s), "cudaEventRecord");
    if ((e.*launch)(fn, grid, args) != 0) throw runtime_error("cuLaunchKernel failed while tuning");
    check_rt(cudaEventRecord(static_cast<cudaEvent_t>(e1), s), "cudaEventRecord");
    check_rt(cudaEventSynchronize(static_cast<cudaEvent_t>(e1)), "cudaEventSynchronize");
    float ms = 0.f;
    check_rt(cudaEventElapsedTime(&ms, static_cast<cudaEvent_t>(e0), static_cast<cudaEvent_t>(e1)), "cudaEventElapsedTime");
    return ms;
}
} // namespace

bool EngineCUDA::tune_batch_launch(Compiled &c, int64_t total, void **args) {
    ensure_variants(c);
    if (c.variants.size() == 1) {
        c.tuned_batch = true;
        return false;
    }
    size_t k = 0;
    for (size_t i = 1; i < c.variants.size(); ++i)
        if (c.variants[i].ms_batch.size() < c.variants[k].ms_batch.size()) k = i;
    Compiled::Variant &v = c.variants[k];
    const int64_t grid = max<int64_t>(1, min<int64_t>(total, static_cast<int64_t>(_sm_count) * v.occ_batch));
    v.ms_batch.push_back(time_launch(*this, rec_e0, rec_e1, _stream, v.fn_batch, grid, args, &EngineCUDA::launch_raw));
    ++_stats.tune_launches;
    bool done = true;
    for (const Compiled::Variant &x : c.variants) done = done && x.ms_batch.size() >= kTuneSamples;
    if (done) {
        size_t best = 0;
        float best_ms = *min_element(c.variants[0].ms_batch.begin(), c.variants[0].ms_batch.end());
        for (size_t i = 1; i < c.variants.size(); ++i) {
            const float m = *min_element(c.variants[i].ms_batch.begin(), c.variants[i].ms_batch.end());
            if (m < best_ms * 0.98f) {
                best = i;
                best_ms = m;
            }
        }
        c.chosen_batch = static_cast<int>(best);
        c.fn_batch = c.variants[best].fn_batch;
        c.occ_batch = c.variants[best].occ_batch;
        c.tuned_batch = true;
    }
    return true;
}

bool EngineCUDA::tune_launch(Compiled &c, const LaunchUnit &u, int64_t work, void **args) {
    const uint64_t h = source_hash(c.source);
    ensure_variants(c);
    if (c.variants.size() == 1) {
        c.tuned = true;
        save_tune_choice(h, 0, 0, 0);
        return false;
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
    const int64_t grid = max<int64_t>(1, min<int64_t>(work, static_cast<int64_t>(_sm_count) * v.ctas_per_sm()));
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
    for (const Compiled::Variant &x : c.variants) done = done && x.ms.size() >= kTuneSamples;
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
        c.occ = b.ctas_per_sm();
        if (!c.tuned_batch) {
            c.fn_batch = b.fn_batch;
            c.occ_batch = b.occ_batch;
        }
        c.tuned = true;
        ++_stats.tuned_kernels;
        if (b.maxrreg > 0 || b.unroll > 0 || b.ctas > 0) ++_stats.tuned_capped;
        save_tune_choice(h, b.maxrreg, b.unroll, b.ctas);
    }
    return true;
}

} // namespace cuda
} // namespace bohrium
