// B200 vector engine: memory, compilation, launching and the flush loop.
#include <algorithm>
#include <atomic>
#include <thread>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <sys/stat.h>
#include <unistd.h>
#include <cuda.h>
#include <cuda_runtime.h>
#include <nvrtc.h>
#include <bh_b200.h>
#include <bohrium/bh_main_memory.hpp>
#include "engine.hpp"

using namespace std;
using namespace bohrium::jitk;

namespace bohrium {
namespace cuda {

// ---------------------------------------------------------------------------------- errors
namespace {
void check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw runtime_error(string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}
void check_nvrtc(nvrtcResult r, const char *what) {
    if (r != NVRTC_SUCCESS) throw runtime_error(string("NVRTC error in ") + what + ": " + nvrtcGetErrorString(r));
}
double seconds_since(chrono::steady_clock::time_point t0) {
    return chrono::duration<double>(chrono::steady_clock::now() - t0).count();
}
uint64_t fnv1a(const void *data, size_t n, uint64_t h = 1469598103934665603ULL) {
    const unsigned char *p = static_cast<const unsigned char *>(data);
    for (size_t i = 0; i < n; ++i) {
        h ^= p[i];
        h *= 1099511628211ULL;
    }
    return h;
}
// Cheap 64-bit mixing for structural hashes.
struct Hasher {
    uint64_t h = 0x9E3779B97F4A7C15ULL;
    void add(uint64_t v) {
        v ^= v >> 33;
        v *= 0xff51afd7ed558ccdULL;
        v ^= v >> 33;
        h = (h ^ v) * 0x100000001b3ULL + 0x9E3779B97F4A7C15ULL;
    }
};
} // namespace

// Driver entry points, fetched through the runtime so the library loads without libcuda.so
// (the machine that builds it has no GPU driver).
struct DeviceApi {
    CUresult (*cuModuleLoadData)(CUmodule *, const void *) = nullptr;
    CUresult (*cuModuleUnload)(CUmodule) = nullptr;
    CUresult (*cuModuleGetFunction)(CUfunction *, CUmodule, const char *) = nullptr;
    CUresult (*cuLaunchKernel)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                               CUstream, void **, void **) = nullptr;
    CUresult (*cuLaunchKernelEx)(const CUlaunchConfig *, CUfunction, void **, void **) = nullptr;
    CUresult (*cuOccupancyMaxActiveBlocksPerMultiprocessor)(int *, CUfunction, int, size_t) = nullptr;
    CUresult (*cuGetErrorString)(CUresult, const char **) = nullptr;
    CUresult (*cuFuncGetAttribute)(int *, CUfunction_attribute, CUfunction) = nullptr;
    CUresult (*cuFuncSetAttribute)(CUfunction, CUfunction_attribute, int) = nullptr;
    CUresult (*cuTensorMapEncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                       const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                       CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill) = nullptr;

    template <typename F>
    void get(const char *name, F &fp) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        check(cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q), name);
        if (p == nullptr || q != cudaDriverEntryPointSuccess) throw runtime_error(string("driver symbol not found: ") + name);
        fp = reinterpret_cast<F>(p);
    }
    DeviceApi() {
        get("cuModuleLoadData", cuModuleLoadData);
        get("cuModuleUnload", cuModuleUnload);
        get("cuModuleGetFunction", cuModuleGetFunction);
        get("cuLaunchKernel", cuLaunchKernel);
        get("cuLaunchKernelEx", cuLaunchKernelEx);
        get("cuOccupancyMaxActiveBlocksPerMultiprocessor", cuOccupancyMaxActiveBlocksPerMultiprocessor);
        get("cuGetErrorString", cuGetErrorString);
        get("cuFuncGetAttribute", cuFuncGetAttribute);
        get("cuFuncSetAttribute", cuFuncSetAttribute);
        get("cuTensorMapEncodeTiled", cuTensorMapEncodeTiled);
    }
    void ck(CUresult r, const char *what) const {
        if (r != CUDA_SUCCESS) {
            const char *s = "?";
            if (cuGetErrorString) cuGetErrorString(r, &s);
            throw runtime_error(string("CUDA driver error in ") + what + ": " + s);
        }
    }
};

// ------------------------------------------------------------------------------------- engine
EngineCUDA::EngineCUDA(component::ComponentVE &c) : comp(c) {
    const ConfigParser &cfg = comp.config;
    prof = cfg.defaultGet<bool>("prof", false);
    verbose = cfg.defaultGet<bool>("verbose", false);
    fmad = cfg.defaultGet<bool>("fmad", false);
    fma_contract = cfg.defaultGet<bool>("fma_contract", true);
    batch_mode = cfg.defaultGet<string>("batch", "off");
    cg_opt.bounds_check = cfg.defaultGet<bool>("bounds_check", false);
    cg_opt.flat_v = cfg.defaultGet<int>("elements_per_thread", 4);
    cg_opt.preload_heavy = cfg.defaultGet<bool>("preload_heavy", true);
    cg_opt.interleave = cfg.defaultGet<int>("interleave", 1);
    cg_opt.tile2d = cfg.defaultGet<bool>("tile2d", true);
    cg_opt.vector_access = cfg.defaultGet<bool>("vector_access", true);
    cg_opt.scan_single_pass = cfg.defaultGet<bool>("scan_single_pass", false);
    cg_opt.scan_windows = cfg.defaultGet<bool>("scan_windows", false);
    cg_opt.stage_bulk = cfg.defaultGet<bool>("stage_bulk", true);
    cg_opt.scan_prefetch = cfg.defaultGet<bool>("scan_prefetch", true);
    pdl = cfg.defaultGet<bool>("pdl", true);
    cg_opt.scan_spin_cap = cfg.defaultGet<int64_t>("scan_spin_cap", int64_t{1} << 22);
    // The GPU reduces over the outermost axis natively, so sweeps may fuse with maps at rank 0.
    fusion_config = jitk::FusionConfig(cfg, false);
    cache_dir = cfg.defaultGet<string>("cache_dir", "");
    if (cache_dir == "NONE") cache_dir.clear();
    _device = cfg.defaultGet<int>("device_number", 0);
    learned_on = cfg.defaultGet<bool>("learned", false);
    learned_runs = cfg.defaultGet<int>("learned_runs", 3);
    learned_margin = cfg.defaultGet<double>("learned_margin", 0.03);
    record = cfg.defaultGet<bool>("record", false);
    chooser = [this](const vector<pair<const Block *, const Block *>> &cands) { return choose_merge(cands); };

    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        throw runtime_error("Error: no devices supporting CUDA");
    }
    check(cudaSetDevice(_device), "cudaSetDevice");
    check(cudaFree(nullptr), "context init");
    cudaDeviceProp prop;
    check(cudaGetDeviceProperties(&prop, _device), "cudaGetDeviceProperties");
    _sm_count = prop.multiProcessorCount;
    api.reset(new DeviceApi());
    cudaStream_t s;
    check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
    _stream = s;
    eager_upload = cfg.defaultGet<bool>("eager_upload", true);
    if (eager_upload) {
        cudaStream_t cs;
        check(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "cudaStreamCreate(copy)");
        _copy_stream = cs;
    }
    // Keep freed device memory in the pool (exact reuse across flushes).
    cudaMemPool_t pool;
    check(cudaDeviceGetDefaultMemPool(&pool, _device), "cudaDeviceGetDefaultMemPool");
    uint64_t threshold = UINT64_MAX;
    const int64_t limit_pct = cfg.defaultGet<int64_t>("malloc_cache_limit", 90);
    if (limit_pct < 0 || limit_pct > 100) throw runtime_error("config: `malloc_cache_limit` must be between 0 and 100");
    threshold = static_cast<uint64_t>(static_cast<double>(prop.totalGlobalMem) * (limit_pct / 100.0));
    check(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold), "cudaMemPoolSetAttribute");
    ensure_counters(4096);
    check(cudaMalloc(&err_record, sizeof(unsigned long long)), "cudaMalloc(err)");
    check(cudaMemset(err_record, 0, sizeof(unsigned long long)), "cudaMemset(err)");
    if (!cache_dir.empty()) mkdir(cache_dir.c_str(), 0755);
    autotune = cfg.defaultGet<bool>("autotune", true);
    tune_min_elements = cfg.defaultGet<int64_t>("autotune_min_elements", 1 << 20);
    load_tune_choices();
    const string model = cfg.defaultGet<string>("costmodel", "");
    if (!model.empty() && model != "NONE") load_costmodel(model);
}

EngineCUDA::~EngineCUDA() {
    try {
        if (_copy_stream) cudaStreamSynchronize(static_cast<cudaStream_t>(_copy_stream));
        cudaStreamSynchronize(static_cast<cudaStream_t>(_stream));
        // Replays own CUDA graphs and device memory, and a graph's clean-up synchronises the
        // engine's stream: release them while that stream still exists (members are destroyed
        // only after this body has destroyed it).
        replays.clear();
        for (auto &kv : buffers) {
            if (kv.second.arrival) cudaEventDestroy(static_cast<cudaEvent_t>(kv.second.arrival));
            if (kv.second.ptr) cudaFree(kv.second.ptr);
        }
        for (void *e : spare_events) cudaEventDestroy(static_cast<cudaEvent_t>(e));
        if (_copy_stream) cudaStreamDestroy(static_cast<cudaStream_t>(_copy_stream));
        if (scratch) cudaFree(scratch);
        if (counters) cudaFree(counters);
        if (staging_dev) cudaFree(staging_dev);
        if (scan_arena) cudaFree(scan_arena);
        if (staging_host) cudaFreeHost(staging_host);
        for (void *p : staging_retired) cudaFreeHost(p);
        for (void *e : busy_events) cudaEventDestroy(static_cast<cudaEvent_t>(e));
        if (staging_event) cudaEventDestroy(static_cast<cudaEvent_t>(staging_event));
        if (err_record) cudaFree(err_record);
        if (rec_e0) cudaEventDestroy(static_cast<cudaEvent_t>(rec_e0));
        if (rec_e1) cudaEventDestroy(static_cast<cudaEvent_t>(rec_e1));
        if (cm) bh_ve_cuda_costmodel_destroy(cm);
        cudaStreamDestroy(static_cast<cudaStream_t>(_stream));
    } catch (...) {
    }
}

void EngineCUDA::synchronize() { check(cudaStreamSynchronize(static_cast<cudaStream_t>(_stream)), "cudaStreamSynchronize"); }

void EngineCUDA::synchronize_all() {
    if (_copy_stream)
        check(cudaStreamSynchronize(static_cast<cudaStream_t>(_copy_stream)), "cudaStreamSynchronize(copy)");
    synchronize();
    check_tma_record();
}

// A kernel whose TMA copies (TILE2D tiles, bulk-staged stencil rows) did not complete within its
// bounded wait records that in the error record (top bits 11) and skips the rest of its work. Read
// at synchronisation points only, so that flushes stay asynchronous.
void EngineCUDA::check_tma_record() {
    if (!tma_check_pending) return;
    tma_check_pending = false;
    unsigned long long v = 0;
    check(cudaMemcpy(&v, err_record, sizeof(v), cudaMemcpyDeviceToHost), "cudaMemcpy(err)");
    if ((v >> 62) == 3ULL) {
        check(cudaMemset(err_record, 0, sizeof(v)), "cudaMemset(err)");
        throw runtime_error("a kernel gave up waiting for a TMA copy (CTA " +
                            to_string(v & 0xffffffffULL) + "); its outputs are incomplete");
    }
}

// ------------------------------------------------------------------------------------- memory
void EngineCUDA::copyToDevice(bh_base *base) {
    if (buffers.count(base)) return;
    DevBuf b;
    b.nbytes = base->nbytes();
    if (b.nbytes > 0) {
        check(inject_alloc_failures > 0 ? (--inject_alloc_failures, cudaErrorMemoryAllocation)
                                        : cudaMallocAsync(&b.ptr, static_cast<size_t>(b.nbytes), static_cast<cudaStream_t>(_stream)),
              "cudaMallocAsync");
        if (base->getDataPtr() != nullptr) {
            check(cudaMemcpyAsync(b.ptr, base->getDataPtr(), static_cast<size_t>(b.nbytes), cudaMemcpyHostToDevice,
                                  static_cast<cudaStream_t>(_stream)),
                  "cudaMemcpyAsync(H2D)");
            _stats.bytes_h2d += static_cast<uint64_t>(b.nbytes);
        }
    }
    buffers[base] = b;
    ++buffer_epoch;
}

void *EngineCUDA::getBuffer(bh_base *base) {
    auto it = buffers.find(base);
    if (it == buffers.end()) {
        copyToDevice(base);
        it = buffers.find(base);
    }
    settle(it->second);
    return it->second.ptr;
}

void EngineCUDA::settle(DevBuf &b) {
    if (b.arrival == nullptr) return;
    check(cudaStreamWaitEvent(static_cast<cudaStream_t>(_stream), static_cast<cudaEvent_t>(b.arrival), 0),
          "cudaStreamWaitEvent(upload)");
    spare_events.push_back(b.arrival);
    b.arrival = nullptr;
}

void EngineCUDA::eager_copy(bh_base *base) {
    cudaStream_t cs = static_cast<cudaStream_t>(_copy_stream);
    DevBuf b;
    b.nbytes = base->nbytes();
    // Allocated on the copy stream: the pool only hands out memory whose earlier uses are done.
    check(inject_alloc_failures > 0 ? (--inject_alloc_failures, cudaErrorMemoryAllocation)
                                    : cudaMallocAsync(&b.ptr, static_cast<size_t>(b.nbytes), cs),
          "cudaMallocAsync(upload)");
    check(cudaMemcpyAsync(b.ptr, base->getDataPtr(), static_cast<size_t>(b.nbytes), cudaMemcpyHostToDevice, cs),
          "cudaMemcpyAsync(H2D upload)");
    cudaEvent_t e;
    if (spare_events.empty()) {
        check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate(upload)");
    } else {
        e = static_cast<cudaEvent_t>(spare_events.back());
        spare_events.pop_back();
    }
    check(cudaEventRecord(e, cs), "cudaEventRecord(upload)");
    b.arrival = e;
    buffers[base] = b;
    _stats.bytes_h2d += static_cast<uint64_t>(b.nbytes);
    ++_stats.eager_uploads;
    ++buffer_epoch;
}

void EngineCUDA::delBuffer(bh_base *base) {
    auto it = buffers.find(base);
    if (it == buffers.end()) return;
    settle(it->second);
    if (it->second.ptr) {
        if (it->second.external) {
            synchronize();
            cudaFree(it->second.ptr);
        } else {
            check(cudaFreeAsync(it->second.ptr, static_cast<cudaStream_t>(_stream)), "cudaFreeAsync");
        }
    }
    buffers.erase(it);
    if (host_stale.erase(base)) ++stale_epoch;
    ++buffer_epoch;
}

void EngineCUDA::free_base(bh_base *base) {
    delBuffer(base);
    void *p = base->getDataPtr();
    if (p == nullptr) return;
    ++buffer_epoch;
    auto it = pinned.find(p);
    if (it != pinned.end()) {
        // Copies from page-locked memory are asynchronous: wait before releasing it.
        synchronize();
        cudaFreeHost(p);
        pinned.erase(it);
        base->resetDataPtr(nullptr);
    } else {
        // Copies from pageable memory are staged before cudaMemcpyAsync returns.
        bh_data_free(base);
    }
}

void *EngineCUDA::host_alloc(int64_t nbytes) {
    void *p = nullptr;
    check(cudaMallocHost(&p, static_cast<size_t>(max<int64_t>(nbytes, 1))), "cudaMallocHost");
    pinned.insert(p);
    return p;
}

void EngineCUDA::record_execute_begin() {
    if (!ev_begin) {
        cudaEvent_t a, b;
        check(cudaEventCreate(&a), "cudaEventCreate");
        check(cudaEventCreate(&b), "cudaEventCreate");
        ev_begin = a;
        ev_end = b;
    }
    check(cudaEventRecord(static_cast<cudaEvent_t>(ev_begin), static_cast<cudaStream_t>(_stream)), "cudaEventRecord");
}

void EngineCUDA::record_execute_end() {
    check(cudaEventRecord(static_cast<cudaEvent_t>(ev_end), static_cast<cudaStream_t>(_stream)), "cudaEventRecord");
}

double EngineCUDA::last_execute_ms() {
    if (!ev_begin) return 0.0;
    check(cudaEventSynchronize(static_cast<cudaEvent_t>(ev_end)), "cudaEventSynchronize");
    float ms = 0;
    check(cudaEventElapsedTime(&ms, static_cast<cudaEvent_t>(ev_begin), static_cast<cudaEvent_t>(ev_end)),
          "cudaEventElapsedTime");
    return ms;
}

void EngineCUDA::timer_start() {
    if (!tm_begin) {
        cudaEvent_t a, b;
        check(cudaEventCreate(&a), "cudaEventCreate");
        check(cudaEventCreate(&b), "cudaEventCreate");
        tm_begin = a;
        tm_end = b;
    }
    check(cudaEventRecord(static_cast<cudaEvent_t>(tm_begin), static_cast<cudaStream_t>(_stream)), "cudaEventRecord");
}

double EngineCUDA::timer_stop_ms() {
    if (!tm_begin) return 0.0;
    check(cudaEventRecord(static_cast<cudaEvent_t>(tm_end), static_cast<cudaStream_t>(_stream)), "cudaEventRecord");
    check(cudaEventSynchronize(static_cast<cudaEvent_t>(tm_end)), "cudaEventSynchronize");
    float ms = 0;
    check(cudaEventElapsedTime(&ms, static_cast<cudaEvent_t>(tm_begin), static_cast<cudaEvent_t>(tm_end)),
          "cudaEventElapsedTime");
    return ms;
}

void EngineCUDA::copyToHost(const set<bh_base *> &bases, bool evict) {
    bool any = false;
    for (bh_base *base : bases) {
        auto it = buffers.find(base);
        if (it == buffers.end()) continue;
        settle(it->second);
        if (host_stale.count(base) || base->getDataPtr() == nullptr) {
            if (base->getDataPtr() == nullptr) ++buffer_epoch;
            bh_data_malloc(base);
            if (it->second.nbytes > 0) {
                check(cudaMemcpyAsync(base->getDataPtr(), it->second.ptr, static_cast<size_t>(it->second.nbytes),
                                      cudaMemcpyDeviceToHost, static_cast<cudaStream_t>(_stream)),
                      "cudaMemcpyAsync(D2H)");
                _stats.bytes_d2h += static_cast<uint64_t>(it->second.nbytes);
                any = true;
            }
            if (host_stale.erase(base)) ++stale_epoch;
        }
    }
    if (any) {
        synchronize();
        check_tma_record();
    }
    if (evict)
        for (bh_base *base : bases) delBuffer(base);
}

void EngineCUDA::copyAllBasesToHost() {
    set<bh_base *> all;
    for (auto &kv : buffers) all.insert(kv.first);
    copyToHost(all, true);
}

void *EngineCUDA::getMemoryPointer(bh_base &base, bool copy2host, bool force_alloc, bool nullify) {
    ++buffer_epoch;
    if (copy2host) {
        // The caller may write to the host data: the host copy becomes the master copy.
        copyToHost({&base}, true);
        if (force_alloc) bh_data_malloc(&base);
        void *ret = base.getDataPtr();
        if (nullify) base.resetDataPtr(nullptr);
        return ret;
    }
    return getBuffer(&base);
}

void EngineCUDA::setMemoryPointer(bh_base *base, bool host_ptr, void *mem) {
    ++buffer_epoch;
    if (host_ptr) {
        delBuffer(base);
        if (base->getDataPtr() != nullptr && base->getDataPtr() != mem) bh_data_free(base);
        base->resetDataPtr(mem);
        if (eager_upload && mem != nullptr && base->nbytes() > 0 && pinned.count(mem)) eager_copy(base);
    } else {
        // Kernels load whole elements (16 bytes at once for complex128): an address that is not a
        // multiple of the element size would be a misaligned access on the device.
        const int64_t esize = bh_type_size(base->dtype());
        if (mem != nullptr && reinterpret_cast<uintptr_t>(mem) % static_cast<uintptr_t>(esize) != 0)
            throw runtime_error("setMemoryPointer(): device pointer is not aligned to the element size (" +
                                to_string(esize) + " bytes)");
        delBuffer(base);
        DevBuf b;
        b.ptr = mem;
        b.nbytes = base->nbytes();
        b.external = true;
        buffers[base] = b;
        host_stale.insert(base);
    }
}

void *EngineCUDA::ensure_scratch(int64_t bytes) {
    if (bytes <= scratch_bytes) return scratch;
    const int64_t nb = max<int64_t>(bytes, max<int64_t>(scratch_bytes * 2, 1 << 20));
    if (scratch) check(cudaFreeAsync(scratch, static_cast<cudaStream_t>(_stream)), "cudaFreeAsync(scratch)");
    check(cudaMallocAsync(&scratch, static_cast<size_t>(nb), static_cast<cudaStream_t>(_stream)), "cudaMallocAsync(scratch)");
    scratch_bytes = nb;
    return scratch;
}

void *EngineCUDA::ensure_scan_arena(int64_t bytes) {
    if (bytes <= scan_arena_bytes) return scan_arena;
    const int64_t nb = max<int64_t>(bytes, max<int64_t>(scan_arena_bytes * 2, 1 << 16));
    if (scan_arena) check(cudaFreeAsync(scan_arena, static_cast<cudaStream_t>(_stream)), "cudaFreeAsync(scan)");
    check(cudaMallocAsync(&scan_arena, static_cast<size_t>(nb), static_cast<cudaStream_t>(_stream)), "cudaMallocAsync(scan)");
    scan_arena_bytes = nb;
    return scan_arena;
}

unsigned int *EngineCUDA::ensure_counters(int64_t n) {
    if (n <= counter_capacity) return counters;
    const int64_t nc = max<int64_t>(n, counter_capacity * 2);
    cudaStream_t s = static_cast<cudaStream_t>(_stream);
    if (counters) check(cudaFreeAsync(counters, s), "cudaFreeAsync(counters)");
    check(cudaMallocAsync(&counters, static_cast<size_t>(nc) * sizeof(unsigned int), s), "cudaMallocAsync(counters)");
    check(cudaMemsetAsync(counters, 0, static_cast<size_t>(nc) * sizeof(unsigned int), s), "cudaMemsetAsync(counters)");
    counter_capacity = nc;
    return counters;
}

// ------------------------------------------------------------------------------- compilation
namespace {

vector<string> nvrtc_options(bool fmad, int maxrreg = 0) {
    vector<string> o = {"-arch=sm_100a", "-std=c++17", fmad ? "--fmad=true" : "--fmad=false", "-lineinfo"};
    if (maxrreg > 0) o.push_back("--maxrregcount=" + to_string(maxrreg));
    return o;
}

// NVRTC compilation of one source to a cubin (thread-safe: one program per call). Returns the
// compiler log through `error` on failure.
bool nvrtc_cubin(const string &name, const string &source, const vector<string> &opts, vector<char> &cubin,
                 string &error) {
    nvrtcProgram prog;
    if (nvrtcCreateProgram(&prog, source.c_str(), (name + ".cu").c_str(), 0, nullptr, nullptr) != NVRTC_SUCCESS) {
        error = "nvrtcCreateProgram failed for " + name;
        return false;
    }
    vector<const char *> copts;
    for (const string &o : opts) copts.push_back(o.c_str());
    const nvrtcResult r = nvrtcCompileProgram(prog, static_cast<int>(copts.size()), copts.data());
    if (r != NVRTC_SUCCESS) {
        size_t logsz = 0;
        nvrtcGetProgramLogSize(prog, &logsz);
        string log(logsz, '\0');
        nvrtcGetProgramLog(prog, &log[0]);
        nvrtcDestroyProgram(&prog);
        error = "NVRTC compilation of " + name + " failed:\n" + log + "\n--- source ---\n" + source;
        return false;
    }
    size_t n = 0;
    nvrtcGetCUBINSize(prog, &n);
    cubin.resize(n);
    const bool ok = nvrtcGetCUBIN(prog, cubin.data()) == NVRTC_SUCCESS;
    nvrtcDestroyProgram(&prog);
    if (!ok) error = "nvrtcGetCUBIN failed for " + name;
    return ok;
}

} // namespace

string EngineCUDA::disk_cache_path(const string &source, int maxrreg) const {
    if (cache_dir.empty()) return "";
    int nvrtc_major = 0, nvrtc_minor = 0;
    nvrtcVersion(&nvrtc_major, &nvrtc_minor);
    string key = source;
    for (const string &o : nvrtc_options(fmad, maxrreg)) key += o;
    key += to_string(nvrtc_major) + "." + to_string(nvrtc_minor);
    stringstream ss;
    ss << cache_dir << "/" << hex << fnv1a(key.data(), key.size()) << ".cubin";
    return ss.str();
}

void EngineCUDA::precompile(const vector<const LaunchUnit *> &units) {
    // Sources that are neither loaded, nor compiled ahead, nor in the disk cache.
    vector<const LaunchUnit *> todo;
    set<uint64_t> seen;
    for (const LaunchUnit *u : units) {
        const uint64_t h = fnv1a(u->source.data(), u->source.size());
        if (functions.count(h) || ahead.count(h) || !seen.insert(h).second) continue;
        const string path = disk_cache_path(u->source);
        if (!path.empty() && access(path.c_str(), R_OK) == 0) continue;  // checked when it is loaded
        todo.push_back(u);
    }
    if (todo.size() < 2 || inject_nvrtc_failures > 0) return;  // an injected failure hits the serial path
    const auto t0 = chrono::steady_clock::now();
    const vector<string> opts = nvrtc_options(fmad);
    vector<vector<char>> cubins(todo.size());
    vector<string> errors(todo.size());
    atomic<size_t> next{0};
    const size_t nthreads = min<size_t>(todo.size(), max(1u, min(16u, thread::hardware_concurrency())));
    vector<thread> pool;
    for (size_t t = 0; t < nthreads; ++t) {
        pool.emplace_back([&]() {
            for (size_t i = next++; i < todo.size(); i = next++)
                nvrtc_cubin(todo[i]->name, todo[i]->source, opts, cubins[i], errors[i]);
        });
    }
    for (thread &th : pool) th.join();
    for (size_t i = 0; i < todo.size(); ++i) {
        if (!errors[i].empty()) throw runtime_error(errors[i]);
        ahead[fnv1a(todo[i]->source.data(), todo[i]->source.size())] = std::move(cubins[i]);
    }
    _stats.time_compile += seconds_since(t0);
    _stats.parallel_compiles += todo.size();
}

// Kernel cache files: an 8-byte tag, the cubin's size and its FNV-1a hash, then the cubin. A file
// that is short, has another tag or fails the hash (a truncated write, a stale format, a damaged
// disk) is deleted and the kernel recompiled: its bytes never reach the driver.
namespace {
const char kCacheTag[8] = {'B', 'H', 'C', 'U', 'B', 'I', 'N', '1'};
}

bool EngineCUDA::read_cache_file(const string &path, vector<char> &cubin) {
    ifstream in(path, ios::binary);
    if (!in) return false;
    vector<char> all((istreambuf_iterator<char>(in)), istreambuf_iterator<char>());
    cubin.clear();
    uint64_t n = 0, h = 0;
    bool ok = all.size() >= 24 && memcmp(all.data(), kCacheTag, 8) == 0;
    if (ok) {
        memcpy(&n, all.data() + 8, 8);
        memcpy(&h, all.data() + 16, 8);
        ok = n > 0 && all.size() == 24 + n && fnv1a(all.data() + 24, n) == h;
    }
    if (!ok) {
        ++_stats.disk_cache_rejected;
        unlink(path.c_str());
        return false;
    }
    cubin.assign(all.begin() + 24, all.end());
    return true;
}

void EngineCUDA::write_cache_file(const string &path, const vector<char> &cubin) {
    if (path.empty()) return;
    const string tmp = path + ".tmp" + to_string(getpid());
    {
        ofstream out(tmp, ios::binary);
        const uint64_t n = cubin.size(), h = fnv1a(cubin.data(), cubin.size());
        out.write(kCacheTag, 8);
        out.write(reinterpret_cast<const char *>(&n), 8);
        out.write(reinterpret_cast<const char *>(&h), 8);
        out.write(cubin.data(), static_cast<streamsize>(cubin.size()));
        if (!out) {
            out.close();
            unlink(tmp.c_str());
            return;
        }
    }
    rename(tmp.c_str(), path.c_str());
}

bool EngineCUDA::compile_cubin(const string &name, const string &source, const vector<string> &opts,
                               vector<char> &cubin, string &error) {
    if (inject_nvrtc_failures > 0) {
        --inject_nvrtc_failures;
        error = "NVRTC compilation of " + name + " failed: injected failure";
        return false;
    }
    return nvrtc_cubin(name, source, opts, cubin, error);
}

vector<char> EngineCUDA::cubin_for(const string &name, const string &source, int maxrreg) {
    vector<char> cubin;
    const string path = disk_cache_path(source, maxrreg);
    if (!path.empty() && read_cache_file(path, cubin)) {
        ++_stats.disk_cache_hits;
        return cubin;
    }
    string error;
    if (!compile_cubin(name, source, nvrtc_options(fmad, maxrreg), cubin, error)) throw runtime_error(error);
    write_cache_file(path, cubin);
    return cubin;
}

// Dynamic shared memory a kernel source asks for: the value of its "// bh_dynamic_shared_bytes: N"
// line (0 without one). Only the plain kernel uses it; the grouped-launch wrapper does not.
int EngineCUDA::dynamic_shared_bytes(const string &source) {
    const string key = "// bh_dynamic_shared_bytes: ";
    const size_t at = source.find(key);
    return at == string::npos ? 0 : atoi(source.c_str() + at + key.size());
}

unsigned EngineCUDA::shared_bytes_of(void *fn) const {
    auto it = fn_shared.find(fn);
    return it == fn_shared.end() ? 0u : it->second;
}

EngineCUDA::Compiled::Variant EngineCUDA::load_variant(const vector<char> &cubin, const string &name, int maxrreg,
                                                       int dyn_smem) {
    CUmodule mod;
    api->ck(api->cuModuleLoadData(&mod, cubin.data()), "cuModuleLoadData");
    Compiled::Variant v;
    CUfunction f, fb;
    api->ck(api->cuModuleGetFunction(&f, mod, name.c_str()), "cuModuleGetFunction");
    api->ck(api->cuModuleGetFunction(&fb, mod, (name + "_batch").c_str()), "cuModuleGetFunction(batch)");
    v.fn = reinterpret_cast<void *>(f);
    v.fn_batch = reinterpret_cast<void *>(fb);
    if (dyn_smem > 0) {
        api->ck(api->cuFuncSetAttribute(f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, dyn_smem),
                "cuFuncSetAttribute(dynamic shared memory)");
        fn_shared[v.fn] = static_cast<unsigned>(dyn_smem);
    }
    api->ck(api->cuOccupancyMaxActiveBlocksPerMultiprocessor(&v.occ, f, kThreads, static_cast<size_t>(dyn_smem)),
            "cuOccupancy");
    api->ck(api->cuOccupancyMaxActiveBlocksPerMultiprocessor(&v.occ_batch, fb, kThreads, 0), "cuOccupancy");
    api->ck(api->cuFuncGetAttribute(&v.regs, CU_FUNC_ATTRIBUTE_NUM_REGS, f), "cuFuncGetAttribute");
    v.occ = max(v.occ, 1);
    v.occ_batch = max(v.occ_batch, 1);
    v.maxrreg = maxrreg;
    return v;
}

EngineCUDA::Compiled *EngineCUDA::compiled_for(const LaunchUnit &u) {
    const uint64_t h = fnv1a(u.source.data(), u.source.size());
    auto it = functions.find(h);
    if (it != functions.end()) {
        ++_stats.kernel_cache_hits;
        return &it->second;
    }
    ++_stats.kernel_cache_misses;
    const auto t0 = chrono::steady_clock::now();
    vector<char> cubin;
    auto pre = ahead.find(h);
    if (pre != ahead.end()) {
        cubin = std::move(pre->second);
        ahead.erase(pre);
        write_cache_file(disk_cache_path(u.source), cubin);
    } else {
        cubin = cubin_for(u.name, u.source, 0);
    }
    Compiled c;
    c.name = u.name;
    c.source = u.source;
    c.variants.push_back(load_variant(cubin, u.name, 0, dynamic_shared_bytes(u.source)));
    // A register cap chosen by an earlier tuning run of this source.
    auto tc = tune_choices.find(h);
    if (tc != tune_choices.end()) {
        c.tuned = true;
        if (tc->second.maxrreg > 0 || tc->second.unroll > 0) {
            c.variants.push_back(make_variant(c, tc->second.maxrreg, tc->second.unroll));
            c.chosen = 1;
        }
        c.variants.back().ctas = tc->second.ctas;
    }
    const Compiled::Variant &v = c.variants[static_cast<size_t>(c.chosen)];
    c.fn = v.fn;
    c.fn_batch = v.fn_batch;
    c.occ = v.ctas_per_sm();
    c.occ_batch = v.occ_batch;
    _stats.time_compile += seconds_since(t0);
    if (verbose) cerr << "[ve_cuda] compiled " << u.name << "\n" << u.source << endl;
    return &functions.emplace(h, std::move(c)).first->second;
}

// ------------------------------------------------------------------------------------ launch
// Scratch bytes a unit needs for its partials.
static int64_t unit_scratch(const LaunchUnit &u) { return u.scratch_bytes(); }

// The TMA tensor map of a TILE2D view (see ParamField::TMAP): base `b` at device address `p` as a
// 2-D array of rows of tm_ld elements, boxes of tm_box_x x tm_box_y elements, with the 128-byte
// swizzle when asked. Writes the 128-byte map to `out` and returns true, or returns false (the
// unit then runs without TMA) when the view does not fit: a TMA copy needs 16-byte aligned base,
// rows and start column, and the view must lie inside whole rows of the map without wrapping to
// the next row.
bool EngineCUDA::encode_tile_map(const ParamField &f, const bh_base *b, void *p, uint8_t *out) {
    const int64_t esize = bh_type_size(b->dtype());
    const int64_t ld = f.tm_ld, start = f.i64;
    if (ld <= 0 || start < 0 || p == nullptr) return false;
    const int64_t nrows = b->nelem() / ld;
    const int64_t ocol = start % ld, orow = start / ld;
    if ((ld * esize) % 16 != 0 || (ocol * esize) % 16 != 0 || reinterpret_cast<uintptr_t>(p) % 16 != 0) return false;
    if (ocol + f.tm_xspan > ld || orow + f.tm_yspan > nrows || ld >= (int64_t{1} << 31) || nrows >= (int64_t{1} << 31))
        return false;
    CUtensorMapDataType dt;
    switch (b->dtype()) {
        case bh_type::FLOAT32: dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT32; break;
        case bh_type::FLOAT64: dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT64; break;
        case bh_type::INT32: dt = CU_TENSOR_MAP_DATA_TYPE_INT32; break;
        case bh_type::UINT32: dt = CU_TENSOR_MAP_DATA_TYPE_UINT32; break;
        case bh_type::INT64: dt = CU_TENSOR_MAP_DATA_TYPE_INT64; break;
        case bh_type::UINT64: dt = CU_TENSOR_MAP_DATA_TYPE_UINT64; break;
        default: return false;
    }
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(ld), static_cast<cuuint64_t>(nrows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld * esize)};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(f.tm_box_x), static_cast<cuuint32_t>(f.tm_box_y)};
    const cuuint32_t estr[2] = {1u, 1u};
    CUtensorMap map;
    if (api->cuTensorMapEncodeTiled(&map, dt, 2, p, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                    f.tm_swizzle ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                                    CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    static_assert(sizeof(CUtensorMap) == 128, "CUtensorMap is 128 bytes");
    memcpy(out, &map, sizeof(map));
    return true;
}

void EngineCUDA::pack_params(const PlanUnit &pu, const vector<bh_base *> &bases,
                             const vector<bh_instruction *> &instrs, int64_t scratch_off, int64_t counter_idx,
                             uint8_t *out) {
    const LaunchUnit &u = pu.unit;
    memset(out, 0, u.fields.size() * 8);
    bool tma_ok = !packing_grouped;
    for (size_t i = 0; i < u.fields.size(); ++i) {
        const ParamField &f = u.fields[i];
        uint8_t *slot = out + i * 8;
        switch (f.kind) {
            case ParamField::TMAP: {
                // All 16 slots are written with the first one; a grouped launch gets no map.
                if (f.part != 0 || !tma_ok) break;
                const int idx = pu.ptr_base[i];
                bh_base *b = idx >= 0 ? bases[static_cast<size_t>(idx)] : f.base;
                void *p = ptr_override != nullptr && idx >= 0 && (*ptr_override)[static_cast<size_t>(idx)] != nullptr
                              ? (*ptr_override)[static_cast<size_t>(idx)]
                              : getBuffer(b);
                tma_ok = encode_tile_map(f, b, p, slot);
                break;
            }
            case ParamField::TMA_OK: {
                const int64_t v = tma_ok ? 1 : 0;
                memcpy(slot, &v, 8);
                if (tma_ok) {
                    tma_check_pending = true;
                    ++_stats.tma_units;
                }
                break;
            }
            case ParamField::PTR: {
                const int idx = pu.ptr_base[i];
                bh_base *b = idx >= 0 ? bases[static_cast<size_t>(idx)] : f.base;
                void *p = ptr_override != nullptr && idx >= 0 && (*ptr_override)[static_cast<size_t>(idx)] != nullptr
                              ? (*ptr_override)[static_cast<size_t>(idx)]
                              : getBuffer(b);
                memcpy(slot, &p, 8);
                break;
            }
            case ParamField::I64: memcpy(slot, &f.i64, 8); break;
            case ParamField::CONST: {
                const bh_constant &c =
                    f.origin >= 0 && f.origin < static_cast<int64_t>(instrs.size()) ? instrs[f.origin]->constant : f.c;
                memcpy(slot, reinterpret_cast<const uint8_t *>(&c.value) + 8 * f.part,
                       static_cast<size_t>(min<int64_t>(bh_type_size(f.c.type), 8)));
                break;
            }
            case ParamField::R123_START:
            case ParamField::R123_KEY: {
                const bh_constant &c =
                    f.origin >= 0 && f.origin < static_cast<int64_t>(instrs.size()) ? instrs[f.origin]->constant : f.c;
                const uint64_t v = f.kind == ParamField::R123_START ? c.value.r123.start : c.value.r123.key;
                memcpy(slot, &v, 8);
                break;
            }
            case ParamField::SCRATCH: {
                void *p = f.i64 == -1              ? static_cast<void *>(err_record)
                          : u.sched == Sched::SCAN1D ? static_cast<void *>(static_cast<uint8_t *>(scan_arena) + u.scan_offset)
                                                     : static_cast<void *>(static_cast<uint8_t *>(scratch) + scratch_off);
                memcpy(slot, &p, 8);
                break;
            }
            case ParamField::COUNTER: {
                void *p = counters + counter_idx + f.off;
                memcpy(slot, &p, 8);
                break;
            }
        }
    }
}

void EngineCUDA::busy_begin() {
    if (!busy_timing) return;
    while (busy_events.size() < busy_used + 2) {
        cudaEvent_t e;
        check(cudaEventCreate(&e), "cudaEventCreate");
        busy_events.push_back(e);
    }
    check(cudaEventRecord(static_cast<cudaEvent_t>(busy_events[busy_used]), static_cast<cudaStream_t>(_stream)),
          "cudaEventRecord");
}

void EngineCUDA::busy_end() {
    if (!busy_timing) return;
    check(cudaEventRecord(static_cast<cudaEvent_t>(busy_events[busy_used + 1]), static_cast<cudaStream_t>(_stream)),
          "cudaEventRecord");
    busy_used += 2;
}

double EngineCUDA::busy_ms() {
    synchronize();
    double total = 0;
    for (size_t i = 0; i + 1 < busy_used; i += 2) {
        float ms = 0;
        check(cudaEventElapsedTime(&ms, static_cast<cudaEvent_t>(busy_events[i]),
                                   static_cast<cudaEvent_t>(busy_events[i + 1])),
              "cudaEventElapsedTime");
        total += ms;
    }
    busy_used = 0;
    return total;
}

void EngineCUDA::record_begin(UnitRecord &r, void *&e0) {
    if (!prof) return;
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, static_cast<cudaStream_t>(_stream));
    e0 = e;
    (void)r;
}

void EngineCUDA::record_end(UnitRecord &r, void *e0) {
    if (!prof) return;
    cudaEvent_t e1;
    cudaEventCreate(&e1);
    cudaEventRecord(e1, static_cast<cudaStream_t>(_stream));
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&r.ms, static_cast<cudaEvent_t>(e0), e1);
    cudaEventDestroy(static_cast<cudaEvent_t>(e0));
    cudaEventDestroy(e1);
    _stats.records.push_back(r);
}

void EngineCUDA::launch_plain(const PlanUnit &pu, const vector<bh_base *> &bases,
                              const vector<bh_instruction *> &instrs) {
    const LaunchUnit &u = pu.unit;
    const int64_t work = u.work_items();
    if (work == 0) return;
    ensure_scratch(unit_scratch(u));
    ensure_counters(max<int64_t>(u.counters_needed(), 1));
    vector<uint8_t> params(u.fields.size() * 8);
    pack_params(pu, bases, instrs, 0, 0, params.data());
    const int64_t resident = static_cast<int64_t>(_sm_count) * pu.compiled->occ;
    const int64_t grid = max<int64_t>(1, min<int64_t>(work, resident));
    void *args[] = {params.data()};
    if (autotune && !pu.compiled->tuned && u.elements >= tune_min_elements && !prof && !record &&
        tune_launch(*pu.compiled, u, work, args)) {
        ++_stats.launches;
        return;
    }
    UnitRecord rec{u.name, u.sched, u.elements, u.algorithmic_bytes, 1, 0.f};
    void *e0 = nullptr;
    record_begin(rec, e0);
    busy_begin();
    launch_dependent(pu.compiled->fn, grid, args, "cuLaunchKernel");
    busy_end();
    record_end(rec, e0);
    ++_stats.launches;
    if (u.sched == Sched::SERIAL) ++_stats.serial_units;
}

// A launch of the engine's own kernels on its stream with programmatic stream serialization (when
// `pdl` is on): the kernel may start while the one before it finishes, and waits in
// bh_grid_dependency() until that one's writes are visible.
void EngineCUDA::launch_dependent(void *fn, int64_t grid, void **args, const char *what) {
    const unsigned smem = static_cast<unsigned>(shared_bytes_of(fn));
    if (!pdl) {
        api->ck(api->cuLaunchKernel(reinterpret_cast<CUfunction>(fn), static_cast<unsigned>(grid), 1, 1, kThreads, 1, 1,
                                    smem, static_cast<CUstream>(_stream), args, nullptr),
                what);
        return;
    }
    CUlaunchAttribute attr[1];
    memset(attr, 0, sizeof(attr));
    attr[0].id = CU_LAUNCH_ATTRIBUTE_PROGRAMMATIC_STREAM_SERIALIZATION;
    attr[0].value.programmaticStreamSerializationAllowed = 1;
    CUlaunchConfig cfg;
    memset(&cfg, 0, sizeof(cfg));
    cfg.gridDimX = static_cast<unsigned>(grid);
    cfg.gridDimY = cfg.gridDimZ = 1;
    cfg.blockDimX = kThreads;
    cfg.blockDimY = cfg.blockDimZ = 1;
    cfg.sharedMemBytes = smem;
    cfg.hStream = static_cast<CUstream>(_stream);
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    api->ck(api->cuLaunchKernelEx(&cfg, reinterpret_cast<CUfunction>(fn), args, nullptr), what);
}

int EngineCUDA::launch_raw(void *fn, int64_t grid, void **args) {
    return static_cast<int>(api->cuLaunchKernel(reinterpret_cast<CUfunction>(fn), static_cast<unsigned>(grid), 1, 1,
                                                kThreads, 1, 1, shared_bytes_of(fn), static_cast<CUstream>(_stream),
                                                args, nullptr));
}

EngineCUDA::PackCache::~PackCache() {
    if (dev) cudaFree(dev);  // waits for the launches that read it
}

void EngineCUDA::launch_batched(const vector<const PlanUnit *> &group, const vector<bh_base *> &bases,
                                const vector<bh_instruction *> &instrs, PackCache *cache) {
    const PlanUnit &proto = *group[0];
    const size_t psize = proto.unit.fields.size() * 8;
    const size_t n = group.size();
    // Per-item scratch and counters.
    int64_t scratch_total = 0, counter_total = 0;
    vector<int64_t> scratch_off(n), counter_off(n);
    for (size_t k = 0; k < n; ++k) {
        scratch_off[k] = scratch_total;
        scratch_total += (unit_scratch(group[k]->unit) + 255) / 256 * 256;
        counter_off[k] = counter_total;
        counter_total += group[k]->unit.counters_needed();
    }
    ensure_scratch(scratch_total);
    ensure_counters(max<int64_t>(counter_total, 1));
    // Items (parameter structs) followed by the prefix sums of their work counts.
    const size_t items_bytes = (psize * n + 15) / 16 * 16;
    const size_t bytes = items_bytes + (n + 1) * sizeof(int64_t);
    uint8_t *dev = nullptr;
    int64_t total = 0;
    if (cache && cache->dev && cache->n == n && cache->bytes == bytes && cache->epoch == buffer_epoch &&
        cache->scratch == scratch && cache->counters == counters && cache->scan_arena == scan_arena) {
        // The same items as last time, already on the device.
        dev = cache->dev;
        total = cache->total;
        ++_stats.pack_reuses;
    } else {
        uint8_t *host = staging_alloc(bytes);
        int64_t *prefix = reinterpret_cast<int64_t *>(host + items_bytes);
        packing_grouped = true;  // tensor maps need the plain kernel's parameter space
        for (size_t k = 0; k < n; ++k) {
            pack_params(*group[k], bases, instrs, scratch_off[k], counter_off[k], host + k * psize);
            prefix[k] = total;
            total += group[k]->unit.grouped_work_items();
        }
        packing_grouped = false;
        prefix[n] = total;
        if (total == 0) return;
        if (cache) {
            if (cache->capacity < bytes) {
                if (cache->dev) {
                    synchronize();
                    check(cudaFree(cache->dev), "cudaFree(pack cache)");
                    cache->dev = nullptr;
                }
                void *p = nullptr;
                check(cudaMalloc(&p, bytes), "cudaMalloc(pack cache)");
                cache->dev = static_cast<uint8_t *>(p);
                cache->capacity = bytes;
            }
            dev = cache->dev;
            cache->n = n;
            cache->bytes = bytes;
            cache->items_bytes = items_bytes;
            cache->total = total;
            cache->epoch = buffer_epoch;  // after any buffer the packing allocated
            cache->scratch = scratch;
            cache->counters = counters;
            cache->scan_arena = scan_arena;
        } else {
            dev = device_staging(bytes);
        }
        check(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, static_cast<cudaStream_t>(_stream)),
              "cudaMemcpyAsync(batch items)");
        if (!staging_event) {
            cudaEvent_t e;
            check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
            staging_event = e;
        }
        check(cudaEventRecord(static_cast<cudaEvent_t>(staging_event), static_cast<cudaStream_t>(_stream)),
              "cudaEventRecord(staging)");
    }
    if (total == 0) return;
    void *items_ptr = dev;
    void *prefix_ptr = dev + items_bytes;
    int nitems = static_cast<int>(n);
    void *args[] = {&items_ptr, &prefix_ptr, &nitems, &total};
    const int64_t resident = static_cast<int64_t>(_sm_count) * proto.compiled->occ_batch;
    const int64_t grid = max<int64_t>(1, min<int64_t>(total, resident));
    UnitRecord rec{proto.unit.name + "_batch", proto.unit.sched, 0, 0, static_cast<int>(n), 0.f};
    for (const PlanUnit *pu : group) {
        rec.elements += pu->unit.elements;
        rec.bytes += pu->unit.algorithmic_bytes;
    }
    if (autotune && !proto.compiled->tuned_batch && rec.elements >= tune_min_elements && !prof && !record &&
        tune_batch_launch(*proto.compiled, total, args)) {
        ++_stats.launches;
        ++_stats.grouped_launches;
        return;
    }
    void *e0 = nullptr;
    record_begin(rec, e0);
    busy_begin();
    launch_dependent(proto.compiled->fn_batch, grid, args, "cuLaunchKernel(batch)");
    busy_end();
    record_end(rec, e0);
    ++_stats.launches;
    ++_stats.grouped_launches;
}

uint8_t *EngineCUDA::staging_alloc(size_t bytes) {
    // Host staging lives for the whole flush; it is recycled once the previous flush's copies ended.
    if (staging_used + bytes > staging_capacity) {
        // Keep old blocks alive until the stream has consumed them.
        synchronize();
        for (void *p : staging_retired) cudaFreeHost(p);
        staging_retired.clear();
        if (staging_host) staging_retired.push_back(staging_host);
        staging_capacity = max<size_t>(bytes * 2, max<size_t>(staging_capacity * 2, 1 << 20));
        void *p = nullptr;
        check(cudaMallocHost(&p, staging_capacity), "cudaMallocHost(staging)");
        staging_host = static_cast<uint8_t *>(p);
        staging_used = 0;
        if (staging_dev) check(cudaFreeAsync(staging_dev, static_cast<cudaStream_t>(_stream)), "cudaFreeAsync");
        check(cudaMallocAsync(reinterpret_cast<void **>(&staging_dev), staging_capacity,
                              static_cast<cudaStream_t>(_stream)),
              "cudaMallocAsync(staging)");
    }
    uint8_t *p = staging_host + staging_used;
    last_staging_offset = staging_used;
    staging_used += (bytes + 255) / 256 * 256;
    return p;
}

uint8_t *EngineCUDA::device_staging(size_t) { return staging_dev + last_staging_offset; }

void EngineCUDA::check_error_record() {
    if (!cg_opt.bounds_check) return;
    unsigned long long v = 0;
    check(cudaMemcpyAsync(&v, err_record, sizeof(v), cudaMemcpyDeviceToHost, static_cast<cudaStream_t>(_stream)),
          "cudaMemcpyAsync(err)");
    synchronize();
    if (v != 0) {
        check(cudaMemset(err_record, 0, sizeof(v)), "cudaMemset(err)");
        last_error_index = v & 0x7fffffffffffffffULL;
        throw runtime_error("bounds check: a generated kernel indexed element " + to_string(last_error_index) +
                            " outside its array");
    }
}

// ------------------------------------------------------------------------------- fuse cache
namespace {
// Structural hash of an instruction list: opcodes, sweep axes, the constant slot, constructor
// flags, and for every view its base (numbered by first appearance), dtype, size, start (unless
// sliding), shape and stride. `base_ids` receives the bases in first-appearance order.
uint64_t hash_instr_list(const vector<bh_instruction *> &instr_list, vector<bh_base *> &base_ids, bool &sliding) {
    Hasher h;
    unordered_map<const bh_base *, uint64_t> ids;
    sliding = false;
    for (const bh_instruction *instr : instr_list) {
        h.add(static_cast<uint64_t>(instr->opcode));
        h.add(static_cast<uint64_t>(instr->sweep_axis()));
        h.add(instr->constructor ? 1 : 0);
        for (const bh_view &v : instr->operand) {
            if (v.isConstant()) {
                h.add(0xC0115747ULL);
                continue;
            }
            auto it = ids.find(v.base);
            uint64_t id;
            if (it == ids.end()) {
                id = ids.size();
                ids[v.base] = id;
                base_ids.push_back(v.base);
            } else {
                id = it->second;
            }
            h.add(id);
            h.add(static_cast<uint64_t>(v.base->dtype()));
            h.add(static_cast<uint64_t>(v.base->nelem()));
            if (v.hasSlide()) {
                sliding = true;
            } else {
                h.add(static_cast<uint64_t>(v.start));
            }
            h.add(static_cast<uint64_t>(v.ndim));
            for (int64_t d = 0; d < v.ndim; ++d) {
                h.add(static_cast<uint64_t>(v.shape[d]));
                h.add(static_cast<uint64_t>(v.stride[d]));
            }
        }
    }
    h.add(instr_list.size());
    return h.h;
}

void rebase(Block &block, const map<bh_base *, bh_base *> &cached2new,
            const unordered_map<int64_t, const bh_instruction *> &origin) {
    if (block.isInstr()) {
        bh_instruction instr(*block.getInstr());
        auto it = origin.find(instr.origin_id);
        if (it == origin.end()) throw runtime_error("fuse cache: unknown origin id");
        const bh_instruction *o = it->second;
        for (size_t i = 0; i < instr.operand.size(); ++i) {
            bh_view &v = instr.operand[i];
            if (v.isConstant()) {
                if (!bh_opcode_is_sweep(instr.opcode)) instr.constant = o->constant;
            } else {
                if (v.hasSlide()) v.start = o->operand[i].start;
                v.base = cached2new.at(v.base);
            }
        }
        instr.constructor = o->constructor;
        block.setInstr(instr);
    } else {
        LoopB &loop = block.getLoop();
        for (Block &b : loop._block_list) rebase(b, cached2new, origin);
        set<bh_base *> frees;
        for (bh_base *b : loop._frees) frees.insert(cached2new.at(b));
        loop._frees = std::move(frees);
        loop.metadataUpdate();
    }
}
} // namespace

vector<LoopB> EngineCUDA::kernels_for(vector<bh_instruction *> &instr_list, uint64_t key,
                                      const vector<bh_base *> &base_ids) {
    const auto t0 = chrono::steady_clock::now();
    vector<LoopB> kernels;
    auto it = fuse_cache.find(key);
    if (it != fuse_cache.end() && it->second.base_ids.size() == base_ids.size()) {
        ++_stats.fuse_cache_hits;
        map<bh_base *, bh_base *> cached2new;
        for (size_t i = 0; i < base_ids.size(); ++i) cached2new[it->second.base_ids[i]] = base_ids[i];
        unordered_map<int64_t, const bh_instruction *> origin;
        for (const bh_instruction *i : instr_list) origin[i->origin_id] = i;
        vector<Block> blocks = it->second.block_list;
        for (Block &b : blocks) rebase(b, cached2new, origin);
        kernels = get_kernel_list(instr_list, fusion_config, &blocks);
    } else {
        ++_stats.fuse_cache_misses;
        vector<Block> blocks;
        kernels = get_kernel_list(instr_list, fusion_config, nullptr, &blocks, chooser ? &chooser : nullptr);
        fuse_cache[key] = FusePayload{std::move(blocks), base_ids};
    }
    _stats.time_fusion += seconds_since(t0);
    return kernels;
}

// One pass over the flushed list (core/jitk/instruction.cpp:580-593 and engine.cpp:338-351 of the
// reference, fused): drop BH_NONE/BH_TALLY, free bases that are freed without being computed, set
// the constructor flags (first use is as an output and the base has neither device nor host data),
// number instructions (origin ids) and bases (first appearance), and hash the structure.
uint64_t EngineCUDA::prepare(vector<bh_instruction> &list, vector<bh_instruction *> &out, vector<bh_base *> &base_ids,
                             bool &sliding, Replay *replay) {
    Hasher h;
    unordered_map<const bh_base *, uint32_t> ids;
    ids.reserve(list.size() * 2 + 16);
    out.reserve(list.size());
    sliding = false;
    vector<bh_base *> dead;
    for (bh_instruction &instr : list) {
        if (instr.opcode == BH_NONE || instr.opcode == BH_TALLY) continue;
        if (instr.opcode == BH_FREE && !ids.count(instr.operand[0].base)) {
            dead.push_back(instr.operand[0].base);
            continue;
        }
        instr.origin_id = static_cast<int64_t>(out.size());
        instr.constructor = false;
        h.add(static_cast<uint64_t>(instr.opcode));
        h.add(static_cast<uint64_t>(instr.sweep_axis()));
        for (size_t o = 0; o < instr.operand.size(); ++o) {
            const bh_view &v = instr.operand[o];
            if (v.isConstant()) {
                h.add(0xC0115747ULL);
                continue;
            }
            auto it = ids.find(v.base);
            uint64_t id;
            if (it == ids.end()) {
                id = ids.size();
                ids.emplace(v.base, static_cast<uint32_t>(id));
                base_ids.push_back(v.base);
                if (o == 0 && instr.opcode != BH_FREE) {
                    instr.constructor = !buffers.count(v.base) && v.base->getDataPtr() == nullptr;
                    if (replay) replay->first_outputs.emplace_back(v.base, instr.constructor);
                }
            } else {
                id = it->second;
            }
            h.add(id);
            h.add(static_cast<uint64_t>(v.base->dtype()));
            h.add(static_cast<uint64_t>(v.base->nelem()));
            if (v.hasSlide()) {
                sliding = true;
            } else {
                h.add(static_cast<uint64_t>(v.start));
            }
            h.add(static_cast<uint64_t>(v.ndim));
            for (int64_t d = 0; d < v.ndim; ++d) {
                h.add(static_cast<uint64_t>(v.shape[d]));
                h.add(static_cast<uint64_t>(v.stride[d]));
            }
        }
        h.add(instr.constructor ? 1 : 0);
        out.push_back(&instr);
    }
    h.add(out.size());
    for (bh_base *b : dead) free_base(b);
    if (replay) replay->dead = std::move(dead);
    return h.h;
}

bool EngineCUDA::replay_valid(const Replay &r) const {
    for (const auto &fo : r.first_outputs) {
        const bool fresh = !buffers.count(fo.first) && fo.first->getDataPtr() == nullptr;
        if (fresh != fo.second) return false;
    }
    return true;
}

void EngineCUDA::setConstructorFlag(vector<bh_instruction *> &instr_list) {
    // Arrays already on the device or with host data are not constructed by this flush.
    set<const bh_base *> constructed;
    for (auto &kv : buffers) constructed.insert(kv.first);
    for (bh_instruction *instr : instr_list) {
        instr->constructor = false;
        for (size_t o = 0; o < instr->operand.size(); ++o) {
            const bh_view &v = instr->operand[o];
            if (v.isConstant()) continue;
            if (o == 0 && !constructed.count(v.base) && v.base->getDataPtr() == nullptr) instr->constructor = true;
            constructed.insert(v.base);
        }
    }
}

// -------------------------------------------------------------------------------- flush plans
EngineCUDA::FlushPlan EngineCUDA::build_plan(const vector<LoopB> &kernels, const vector<bh_base *> &base_ids) {
    FlushPlan plan;
    unordered_map<const bh_base *, int> index;
    for (size_t i = 0; i < base_ids.size(); ++i) index[base_ids[i]] = static_cast<int>(i);
    auto idx = [&](const bh_base *b) -> int {
        auto it = index.find(b);
        return it == index.end() ? -1 : it->second;
    };
    // Dependency levels: a kernel runs after every earlier kernel it shares a written base with.
    vector<int> last_write_level(base_ids.size(), -1), last_read_level(base_ids.size(), -1);
    // Lower every kernel first so that all new sources compile in parallel.
    vector<vector<LaunchUnit>> lowered(kernels.size());
    vector<int> folded_into(kernels.size(), -1);
    {
        const auto tc = chrono::steady_clock::now();
        vector<const LaunchUnit *> all;
        for (size_t k = 0; k < kernels.size(); ++k) {
            if (kernels[k].isSystemOnly()) continue;
            lowered[k] = lower_kernel(kernels[k], cg_opt);
        }
        // Small dependent order-free reductions run in the tail of the kernel before them. Not
        // while recording per-kernel timings, whose features describe one kernel each.
        if (!record) folded_into = fuse_tails(kernels, lowered, cg_opt);
        for (size_t k = 0; k < kernels.size(); ++k)
            for (const LaunchUnit &u : lowered[k]) all.push_back(&u);
        _stats.time_codegen += seconds_since(tc);
        precompile(all);
    }
    // Register temporaries: arrays this flush creates that no unit addresses in memory. They never
    // get a buffer or host data, so their writes and frees need no bookkeeping and make no
    // dependencies between kernels.
    vector<char> in_memory(base_ids.size(), 0), created(base_ids.size(), 0);
    for (const vector<LaunchUnit> &units : lowered)
        for (const LaunchUnit &u : units)
            for (const ParamField &f : u.fields)
                if ((f.kind == ParamField::PTR || f.kind == ParamField::TMAP) && f.base != nullptr) {
                    const int b = idx(f.base);
                    if (b >= 0) in_memory[static_cast<size_t>(b)] = 1;
                }
    for (const LoopB &kernel : kernels)
        for (const InstrPtr &instr : all_instr(kernel))
            if (instr->constructor && !instr->operand.empty() && !instr->operand[0].isConstant()) {
                const int b = idx(instr->operand[0].base);
                if (b >= 0) created[static_cast<size_t>(b)] = 1;
            }
    auto register_temp = [&](int b) { return created[static_cast<size_t>(b)] && !in_memory[static_cast<size_t>(b)]; };
    for (size_t kidx = 0; kidx < kernels.size(); ++kidx) {
        if (folded_into[kidx] >= 0) continue;  // runs in the tail of an earlier kernel
        const LoopB &kernel = kernels[kidx];
        // The kernels this plan kernel runs: itself and any folded into its tail.
        vector<const LoopB *> parts{&kernel};
        for (size_t j = kidx + 1; j < kernels.size(); ++j)
            if (folded_into[j] == static_cast<int>(kidx)) parts.push_back(&kernels[j]);
        PlanKernel pk;
        if (!kernel.isSystemOnly()) {
            vector<LaunchUnit> &units = lowered[kidx];
            int64_t scan_need = 0;
            for (LaunchUnit &u : units) {
                if (u.sched != Sched::SCAN1D) continue;
                u.scan_offset = plan.scan_bytes;
                scan_need = max<int64_t>(scan_need, (u.scan_bytes + 255) / 256 * 256);
            }
            plan.scan_bytes += scan_need;
            for (LaunchUnit &u : units) {
                PlanUnit pu;
                pu.compiled = compiled_for(u);
                pu.ptr_base.assign(u.fields.size(), -1);
                for (size_t f = 0; f < u.fields.size(); ++f)
                    if (u.fields[f].kind == ParamField::PTR || u.fields[f].kind == ParamField::TMAP)
                        pu.ptr_base[f] = idx(u.fields[f].base);
                pu.unit = std::move(u);
                pk.units.push_back(std::move(pu));
            }
        }
        set<int> reads, writes;
        for (const LoopB *part : parts) {
            for (const InstrPtr &instr : all_instr(*part)) {
                for (size_t o = 0; o < instr->operand.size(); ++o) {
                    const bh_view &v = instr->operand[o];
                    if (v.isConstant()) continue;
                    const int b = idx(v.base);
                    if (b < 0 || register_temp(b)) continue;
                    if (o == 0) {
                        writes.insert(b);
                    } else {
                        reads.insert(b);
                    }
                }
            }
            for (bh_base *f : part->getAllFrees()) {
                const int b = idx(f);
                if (b >= 0 && !register_temp(b)) {
                    pk.frees.push_back(b);
                    writes.insert(b);
                }
            }
        }
        pk.writes.assign(writes.begin(), writes.end());
        // Features of every kernel, whether recording is on or not: a plan built before recording
        // is switched on is reused by the recorded executions (computing them only when recording
        // left those kernels with all-zero features).
        if (!pk.units.empty()) pk.feat = jitk::block_features(kernel);
        // Summation order of the floating-point sums and products: "seq" (one thread folds in
        // index order) unless a unit reduces the sweep across threads.
        for (const LoopB *part : parts)
        for (const InstrPtr &instr : all_instr(*part)) {
            if (!bh_opcode_is_sweep(instr->opcode)) continue;
            const bh_opcode op = instr->opcode;
            if (op != BH_ADD_REDUCE && op != BH_MULTIPLY_REDUCE && op != BH_ADD_ACCUMULATE &&
                op != BH_MULTIPLY_ACCUMULATE)
                continue;
            const bh_type t = instr->operand[0].base->dtype();
            if (t != bh_type::FLOAT32 && t != bh_type::FLOAT64 && t != bh_type::COMPLEX64 && t != bh_type::COMPLEX128)
                continue;
            plan.orders[instr->origin_id] = "seq";
        }
        for (const PlanUnit &pu : pk.units)
            for (const auto &ro : pu.unit.red_orders)
                if (plan.orders.count(ro.first)) plan.orders[ro.first] = ro.second;
        int level = 0;
        for (int b : reads) level = max(level, last_write_level[b] + 1);
        for (int b : writes) level = max(level, max(last_write_level[b], last_read_level[b]) + 1);
        pk.level = level;
        const int end_level = level + max<int>(static_cast<int>(pk.units.size()), 1) - 1;
        for (int b : reads) last_read_level[b] = max(last_read_level[b], end_level);
        for (int b : writes) last_write_level[b] = max(last_write_level[b], end_level);
        plan.nlevels = max(plan.nlevels, end_level + 1);
        plan.kernels.push_back(std::move(pk));
    }
    return plan;
}

void EngineCUDA::run_plan(const FlushPlan &plan, const vector<bh_base *> &bases, const vector<bh_instruction *> &instrs,
                          Replay *replay) {
    if (plan.scan_bytes > 0) ensure_scan_arena(plan.scan_bytes);
    if (record) {
        record_kernel_times(plan, bases, instrs);
        return;
    }
    // A replay whose writes are all still in host_stale (nothing was removed from it since its
    // last run) need not insert them again.
    const bool stale_known = replay != nullptr && replay->stale_after == stale_epoch;
    if (batch_mode == "off" || plan.kernels.size() < 2) {
        for (const PlanKernel &pk : plan.kernels) {
            ++_stats.kernels;
            for (const PlanUnit &pu : pk.units) launch_plain(pu, bases, instrs);
            if (!stale_known)
                for (int w : pk.writes) host_stale.insert(bases[static_cast<size_t>(w)]);
            for (int f : pk.frees) free_base(bases[static_cast<size_t>(f)]);
        }
        if (replay) replay->stale_after = stale_epoch;
        return;
    }
    // Grouped execution: level by level, units of the same compiled kernel run as one launch.
    vector<vector<const PlanUnit *>> by_level(static_cast<size_t>(plan.nlevels));
    vector<vector<const PlanKernel *>> kernels_by_end(static_cast<size_t>(plan.nlevels));
    for (const PlanKernel &pk : plan.kernels) {
        ++_stats.kernels;
        for (size_t j = 0; j < pk.units.size(); ++j) by_level[pk.level + j].push_back(&pk.units[j]);
        kernels_by_end[pk.level + max<size_t>(pk.units.size(), 1) - 1].push_back(&pk);
    }
    for (size_t lv = 0; lv < by_level.size(); ++lv) {
        map<const Compiled *, vector<const PlanUnit *>> groups;
        vector<const Compiled *> order;
        for (const PlanUnit *pu : by_level[lv]) {
            if (!groups.count(pu->compiled)) order.push_back(pu->compiled);
            groups[pu->compiled].push_back(pu);
        }
        for (const Compiled *c : order) {
            const auto &g = groups[c];
            if (g.size() == 1 || g[0]->unit.no_batch) {
                for (const PlanUnit *pu : g) launch_plain(*pu, bases, instrs);
            } else {
                PackCache *pc = nullptr;
                if (replay) {
                    unique_ptr<PackCache> &slot = replay->packs[{lv, c}];
                    if (!slot) slot.reset(new PackCache());
                    pc = slot.get();
                }
                launch_batched(g, bases, instrs, pc);
            }
        }
        for (const PlanKernel *pk : kernels_by_end[lv]) {
            if (!stale_known)
                for (int w : pk->writes) host_stale.insert(bases[static_cast<size_t>(w)]);
            for (int f : pk->frees) free_base(bases[static_cast<size_t>(f)]);
        }
    }
    if (replay) replay->stale_after = stale_epoch;
}

void EngineCUDA::handleExecution(BhIR *bhir) {
    const auto t0 = chrono::steady_clock::now();
    // A repeated, unmodified BhIR replays its plan without scanning the instruction list.
    const uint64_t fingerprint = bhir == cur_ir ? cur_hints.fingerprint : 0;
    if (fingerprint != 0) {
        auto rit = replays.find(fingerprint);
        // A graph replay whose arrays and host copies are untouched since its last launch needs
        // no checks at all.
        const bool graph_mode = batch_mode == "graph" && !prof && !record;
        // No buffer or host pointer changed since a replay that changed none itself: its checks
        // would find what they found then.
        const bool same_state = rit != replays.end() && rit->second.checked_epoch == buffer_epoch;
        const bool unchanged = same_state && graph_mode && rit->second.graph;
        if (rit != replays.end() && (same_state || replay_valid(rit->second))) {
            Replay &r = rit->second;
            for (bh_base *b : r.dead) free_base(b);
            const auto t1 = chrono::steady_clock::now();
            _stats.time_prepare += chrono::duration<double>(t1 - t0).count();
            if (graph_mode) {
                if (r.graph && !unchanged && !graph_usable(*r.graph)) r.graph.reset();
                if (!r.graph && !r.graph_failed && r.valid_runs >= 1 && !build_graph(r)) r.graph_failed = true;
                ++r.valid_runs;
                if (r.graph) {
                    ++_stats.plan_cache_hits;
                    ++_stats.replays;
                    graph_launch(*r.graph);
                    _stats.time_launch += seconds_since(t1);
                    copyToHost(bhir->_syncs, false);
                    check_error_record();
                    r.checked_epoch = buffer_epoch;
                    _stats.time_exec_host += seconds_since(t0);
                    return;
                }
            }
            if (staging_used > 0 && staging_event)
                check(cudaEventSynchronize(static_cast<cudaEvent_t>(staging_event)), "cudaEventSynchronize(staging)");
            staging_used = 0;
            ++_stats.plan_cache_hits;
            ++_stats.replays;
            const uint64_t epoch0 = buffer_epoch;
            run_plan(*r.plan, r.base_ids, r.instrs, &r);
            r.checked_epoch = buffer_epoch == epoch0 ? buffer_epoch : 0;
            _stats.time_launch += seconds_since(t1);
            copyToHost(bhir->_syncs, false);
            check_error_record();
            _stats.time_exec_host += seconds_since(t0);
            return;
        }
    }
    vector<bh_instruction *> instr_list;
    vector<bh_base *> base_ids;
    bool sliding = false;
    Replay replay;
    if (fma_contract) {
        auto holds_nothing = [this](const bh_base *b) {
            return b->getDataPtr() == nullptr && !buffers.count(const_cast<bh_base *>(b));
        };
        _stats.fma_contractions +=
            static_cast<uint64_t>(contract_multiply_add(bhir->instr_list, bhir->_syncs, holds_nothing));
    }
    const uint64_t key = prepare(bhir->instr_list, instr_list, base_ids, sliding, fingerprint ? &replay : nullptr);
    const auto t1 = chrono::steady_clock::now();
    _stats.time_prepare += chrono::duration<double>(t1 - t0).count();
    if (staging_used > 0 && staging_event) {
        // The previous flush's parameter copies must have left the staging area before reuse.
        check(cudaEventSynchronize(static_cast<cudaEvent_t>(staging_event)), "cudaEventSynchronize(staging)");
    }
    staging_used = 0;
    auto it = sliding ? plans.end() : plans.find(key);
    auto tit = sliding ? trials.end() : trials.find(key);
    if (it != plans.end() && it->second.nbases == base_ids.size()) {
        ++_stats.plan_cache_hits;
        run_plan(it->second, base_ids, instr_list);
    } else if (tit != trials.end() && tit->second.greedy.nbases == base_ids.size()) {
        ++_stats.plan_cache_hits;
        run_trial(key, tit->second, base_ids, instr_list);
    } else {
        ++_stats.plan_cache_misses;
        const vector<LoopB> kernels = kernels_for(instr_list, key, base_ids);
        FlushPlan plan = build_plan(kernels, base_ids);
        plan.nbases = base_ids.size();
        if (!sliding && learned_on && cm != nullptr && !decided.count(key) &&
            start_trial(key, instr_list, base_ids, plan)) {
            run_trial(key, trials.at(key), base_ids, instr_list);
        } else {
            run_plan(plan, base_ids, instr_list);
            if (!sliding) plans[key] = std::move(plan);
        }
    }
    if (fingerprint != 0 && !sliding) {
        auto pit = plans.find(key);
        if (pit != plans.end()) {
            replay.plan = &pit->second;
            replay.base_ids = base_ids;
            replay.instr_copy.reserve(instr_list.size());
            for (const bh_instruction *i : instr_list) replay.instr_copy.push_back(*i);
            for (bh_instruction &i : replay.instr_copy) replay.instrs.push_back(&i);
            replays[fingerprint] = std::move(replay);
        }
    }
    const auto t2 = chrono::steady_clock::now();
    _stats.time_launch += chrono::duration<double>(t2 - t1).count();
    copyToHost(bhir->_syncs, false);
    check_error_record();
    _stats.time_exec_host += seconds_since(t0);
}

void EngineCUDA::handleExtmethod(BhIR *bhir) {
    // Only a list that contains extension methods needs splitting (and copying).
    bool any = false;
    if (!(bhir == cur_ir && cur_hints.plain) && (!comp.extmethods.empty() || !comp.child_extmethods.empty())) {
        for (const bh_instruction &instr : bhir->instr_list) {
            if (comp.extmethods.count(instr.opcode) || comp.child_extmethods.count(instr.opcode)) {
                any = true;
                break;
            }
        }
    }
    if (!any) return;
    // The list is rewritten below: its registered fingerprint no longer describes it.
    if (bhir == cur_ir) cur_hints.fingerprint = 0;
    bh_ir_hints_clear(bhir);
    vector<bh_instruction> instr_list;
    for (bh_instruction &instr : bhir->instr_list) {
        auto ext = comp.extmethods.find(instr.opcode);
        auto childext = comp.child_extmethods.find(instr.opcode);
        if (ext != comp.extmethods.end() || childext != comp.child_extmethods.end()) {
            BhIR b(std::move(instr_list), bhir->getSyncs());
            handleExecution(&b);
            instr_list.clear();
            if (ext != comp.extmethods.end()) {
                bh_ve_cuda_ext_context ctx;
                ctx.version = 1;
                ctx.engine = this;
                ctx.stream = _stream;
                ctx.device_pointer = [](void *e, bh_base *b) { return static_cast<EngineCUDA *>(e)->getBuffer(b); };
                ctx.written = [](void *e, bh_base *b) { static_cast<EngineCUDA *>(e)->mark_device_written(b); };
                ext->second.execute(&instr, &ctx);
                if (!instr.operand.empty() && !instr.operand[0].isConstant()) mark_device_written(instr.operand[0].base);
            } else {
                set<bh_base *> bases = instr.get_bases();
                copyToHost(bases, true);
                vector<bh_instruction> child_list{instr};
                BhIR cb(std::move(child_list), bhir->getSyncs());
                comp.child.execute(&cb);
            }
        } else {
            instr_list.push_back(instr);
        }
    }
    bhir->instr_list = std::move(instr_list);
}

namespace {
// Slide views between repeats of flush-and-repeat (include/bohrium/jitk/engines/dyn_view.hpp:21-67).
void slide_views(BhIR *bhir) {
    for (bh_instruction &instr : bhir->instr_list) {
        for (bh_view &view : instr.operand) {
            if (!view.hasSlide()) continue;
            for (const bh_slide_dim &dim : view.slides.dims) {
                if (dim.step_delay == 1 || (view.slides.iteration_counter % dim.step_delay == dim.step_delay - 1)) {
                    if (dim.stride) {
                        int64_t change = dim.offset_change * dim.stride;
                        const int64_t max_rel_idx = dim.stride * dim.shape;
                        int64_t rel_idx = view.start % (dim.stride * dim.shape);
                        rel_idx += change;
                        if (rel_idx < 0) {
                            change += max_rel_idx;
                        } else if (rel_idx >= max_rel_idx) {
                            change -= max_rel_idx;
                        }
                        view.start += change;
                        auto it = view.slides.resets.find(dim.rank);
                        if (it != view.slides.resets.end()) {
                            const int64_t reset_at = it->second.first;
                            int64_t &changes_since_reset = it->second.second;
                            changes_since_reset += change;
                            if (view.slides.iteration_counter > 0 &&
                                (view.slides.iteration_counter / dim.step_delay) % reset_at == reset_at - 1) {
                                view.start -= changes_since_reset;
                                changes_since_reset = 0;
                                view.shape[dim.rank] -= reset_at * dim.shape_change;
                            }
                        }
                    }
                    view.shape[dim.rank] += dim.shape_change;
                    if (view.shape[dim.rank] < 0) view.shape[dim.rank] = 0;
                }
            }
            view.slides.iteration_counter += 1;
        }
    }
}
} // namespace

// ------------------------------------------------------------------------------------- user kernels
namespace {
// The integers after "<option>:" in a user-kernel parameter string such as
// "global_work_size: 20 5; local_work_size: 1 1": digits separated by spaces, tabs, newlines or
// commas, up to the first other character. Empty when the option is absent or a number does not
// fit. The same reading as the reference's OpenCL engine (ve/opencl/engine_opencl.cpp:588-608).
vector<int64_t> param_integers(const string &option, const string &param) {
    const size_t at = param.find(option + ":");
    if (at == string::npos) return {};
    vector<int64_t> out;
    string tok;
    auto flush_tok = [&]() {
        if (tok.empty()) return true;
        if (tok.size() > 18) return false;
        out.push_back(stoll(tok));
        tok.clear();
        return true;
    };
    for (size_t i = at + option.size() + 1; i < param.size(); ++i) {
        const char ch = param[i];
        if (ch >= '0' && ch <= '9') {
            tok += ch;
        } else if (ch == ' ' || ch == '\t' || ch == '\n' || ch == '\r' || ch == ',') {
            if (!flush_tok()) return {};
        } else {
            break;
        }
    }
    if (!flush_tok()) return {};
    return out;
}
} // namespace

string EngineCUDA::userKernel(const string &kernel, vector<bh_view> &operands, const string &param) {
    for (const bh_view &op : operands)
        if (op.isConstant()) return "[UserKernel] fatal error - operands cannot be constants";
    const vector<int64_t> global = param_integers("global_work_size", param);
    const vector<int64_t> local = param_integers("local_work_size", param);
    if (global.size() != local.size())
        return "[CUDA] userKernel-param dimension of global_work_size and local_work_size must be the same";
    if (global.empty() || global.size() > 3) return "[CUDA] userKernel-param maximum of three dimensions!";
    // Dimension d of the work sizes is CUDA's x, y, z: a block of local_work_size threads, and
    // global_work_size / local_work_size blocks (a whole number, as OpenCL 1.x requires).
    unsigned grid[3] = {1, 1, 1}, block[3] = {1, 1, 1};
    const int64_t max_block[3] = {1024, 1024, 64}, max_grid[3] = {2147483647, 65535, 65535};
    int64_t threads = 1;
    for (size_t d = 0; d < global.size(); ++d) {
        if (local[d] <= 0 || global[d] <= 0 || global[d] % local[d] != 0)
            return "[CUDA] userKernel-param global_work_size must be a positive multiple of local_work_size";
        if (local[d] > max_block[d] || global[d] / local[d] > max_grid[d])
            return "[CUDA] userKernel-param work size beyond the device's block or grid limits";
        block[d] = static_cast<unsigned>(local[d]);
        grid[d] = static_cast<unsigned>(global[d] / local[d]);
        threads *= local[d];
    }
    if (threads > 1024) return "[CUDA] userKernel-param local_work_size has more than 1024 threads";

    const uint64_t h = fnv1a(kernel.data(), kernel.size());
    void *fn = nullptr;
    auto it = user_functions.find(h);
    if (it != user_functions.end()) {
        fn = it->second;
    } else {
        const auto t0 = chrono::steady_clock::now();
        vector<char> cubin;
        try {
            cubin = cubin_for("bh_user_kernel", kernel, 0);
        } catch (const exception &e) {
            return string("[CUDA] userKernel compilation failed: ") + e.what();
        }
        CUmodule mod;
        CUfunction f;
        if (api->cuModuleLoadData(&mod, cubin.data()) != CUDA_SUCCESS) return "[CUDA] userKernel: cuModuleLoadData failed";
        if (api->cuModuleGetFunction(&f, mod, "execute") != CUDA_SUCCESS) {
            api->cuModuleUnload(mod);
            return "[CUDA] userKernel: the source defines no extern \"C\" __global__ function named execute";
        }
        fn = reinterpret_cast<void *>(f);
        user_functions[h] = fn;
        _stats.time_compile += seconds_since(t0);
    }
    // One device pointer per operand: the start of its base array, as the reference's engines
    // pass whole buffers (ve/opencl/engine_opencl.cpp:628-630, ve/openmp/engine_openmp.cpp:503-506).
    vector<void *> ptrs(operands.size()), args(operands.size());
    for (size_t i = 0; i < operands.size(); ++i) {
        ptrs[i] = getBuffer(operands[i].base);
        args[i] = &ptrs[i];
    }
    const auto t0 = chrono::steady_clock::now();
    const CUresult r = api->cuLaunchKernel(reinterpret_cast<CUfunction>(fn), grid[0], grid[1], grid[2], block[0], block[1],
                                           block[2], 0, reinterpret_cast<CUstream>(_stream),
                                           args.empty() ? nullptr : args.data(), nullptr);
    if (r != CUDA_SUCCESS) {
        const char *msg = "?";
        api->cuGetErrorString(r, &msg);
        return string("[CUDA] userKernel launch failed: ") + msg;
    }
    ++_stats.launches;
    synchronize();
    _stats.time_exec_host += seconds_since(t0);
    for (const bh_view &op : operands) mark_device_written(op.base);
    return "";
}

void EngineCUDA::execute(BhIR *bhir) {
    ++_stats.flushes;
    cur_ir = bhir;
    cur_hints = bh_ir_hints_get(bhir);
    bh_base *cond = bhir->getRepeatCondition();
    for (uint64_t i = 0; i < bhir->getNRepeats(); ++i) {
        handleExtmethod(bhir);
        handleExecution(bhir);
        if (cond != nullptr) {
            copyToHost({cond}, false);
            if (cond->getDataPtr() != nullptr && !static_cast<bool *>(cond->getDataPtr())[0]) break;
        }
        if (!cur_hints.plain) slide_views(bhir);  // a plain list has no sliding views
    }
}

// ------------------------------------------------------------------------------------ reports
string EngineCUDA::info() const {
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, _device);
    int nv_major = 0, nv_minor = 0;
    nvrtcVersion(&nv_major, &nv_minor);
    stringstream ss;
    ss << "----\nCUDA (B200 engine):\n";
    ss << "  Device: " << prop.name << " (SM " << prop.major << "." << prop.minor << ", " << prop.multiProcessorCount
       << " SMs)\n";
    ss << "  Memory: " << prop.totalGlobalMem / 1024 / 1024 << " MB\n";
    ss << "  JIT: NVRTC " << nv_major << "." << nv_minor << " -arch=sm_100a" << (fmad ? "" : " --fmad=false") << "\n";
    ss << "  Cache dir: " << (cache_dir.empty() ? "NONE" : cache_dir) << "\n";
    ss << "  Batch mode: " << batch_mode << "\n";
    return ss.str();
}

string EngineCUDA::statistics() const {
    stringstream ss;
    ss << "flushes: " << _stats.flushes << "\nkernels: " << _stats.kernels << "\nlaunches: " << _stats.launches
       << "\ngrouped_launches: " << _stats.grouped_launches << "\ngraph_replays: " << _stats.graph_replays
       << "\nserial_units: " << _stats.serial_units << "\nfuse_cache_hits: " << _stats.fuse_cache_hits
       << "\nfuse_cache_misses: " << _stats.fuse_cache_misses << "\nkernel_cache_hits: " << _stats.kernel_cache_hits
       << "\nkernel_cache_misses: " << _stats.kernel_cache_misses << "\ndisk_cache_hits: " << _stats.disk_cache_hits
       << "\ndisk_cache_rejected: " << _stats.disk_cache_rejected
       << "\nfma_contractions: " << _stats.fma_contractions << "\neager_uploads: " << _stats.eager_uploads
       << "\ntma_units: " << _stats.tma_units << "\npack_reuses: " << _stats.pack_reuses
       << "\nbytes_h2d: " << _stats.bytes_h2d << "\nbytes_d2h: " << _stats.bytes_d2h
       << "\ntime_fusion: " << _stats.time_fusion << "\ntime_codegen: " << _stats.time_codegen
       << "\ntime_compile: " << _stats.time_compile << "\nparallel_compiles: " << _stats.parallel_compiles
       << "\ntuned_kernels: " << _stats.tuned_kernels << "\ntuned_capped: " << _stats.tuned_capped
       << "\ntune_launches: " << _stats.tune_launches
       << "\ntime_exec_host: " << _stats.time_exec_host
       << "\ntime_prepare: " << _stats.time_prepare << "\ntime_launch: " << _stats.time_launch
       << "\nplan_cache_hits: " << _stats.plan_cache_hits << "\nplan_cache_misses: " << _stats.plan_cache_misses
       << "\nreplays: " << _stats.replays << "\nlearned_trials: " << _stats.learned_trials
       << "\nlearned_kept: " << _stats.learned_kept << "\ngreedy_kept: " << _stats.greedy_kept
       << "\nlearned_same_plan: " << _stats.learned_same << "\nlearned_order_differs: " << _stats.learned_order_differs
       << "\nlearned_predictions: " << _stats.learned_predictions
       << "\ntime_learned_fusion: " << _stats.time_learned_fusion
       << "\ntime_learned_choose: " << _stats.time_learned_choose << "\nrecords: " << record_count() << "\n";
    if (!_stats.records.empty()) {
        ss << "units:\n";
        for (const UnitRecord &r : _stats.records)
            ss << "  - {name: " << r.name << ", sched: " << sched_name(r.sched) << ", elements: " << r.elements
               << ", bytes: " << r.bytes << ", ms: " << r.ms << "}\n";
    }
    return ss.str();
}

void EngineCUDA::resetStatistics() { _stats = Stats(); }

} // namespace cuda
} // namespace bohrium
