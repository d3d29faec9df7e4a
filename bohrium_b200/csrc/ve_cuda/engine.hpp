// The B200 vector engine: executes flushed BhIR on one GPU.
//
// Replaces EngineCUDA + EngineGPU of the reference (ve/cuda/engine_cuda.{hpp,cpp},
// include/bohrium/jitk/engines/engine_gpu.hpp). Differences by design:
//  - kernels are compiled in-process with NVRTC for sm_100a (no nvcc fork), cached in memory
//    and on disk, and launched asynchronously on one stream (no synchronisation per launch);
//  - every fused block runs on the GPU (no CPU offload), see codegen.hpp;
//  - device buffers come from the stream-ordered allocator pool and stay valid after a sync
//    (lazy host sync: the host copy is refreshed, the device copy is not evicted);
//  - optional batching: independent launches of the same compiled kernel run as one grouped
//    launch, and repeated flushes can be replayed as CUDA graphs (see batch.hpp).
#pragma once

#include <chrono>
#include <cstdint>
#include <map>
#include <memory>
#include <set>
#include <string>
#include <unordered_map>
#include <vector>
#include <bohrium/bh_component.hpp>
#include "../jitk/fuser.hpp"
#include "codegen.hpp"

namespace bohrium {
namespace cuda {

struct DeviceApi; // driver entry points (engine.cpp)

// Per-launch-unit timing record (device time measured with CUDA events when profiling).
struct UnitRecord {
    std::string name;
    Sched sched;
    int64_t elements = 0;
    int64_t bytes = 0;
    int n_instr = 0;
    float ms = 0.f;
};

struct Stats {
    uint64_t flushes = 0, kernels = 0, launches = 0, grouped_launches = 0, graph_replays = 0;
    uint64_t fuse_cache_hits = 0, fuse_cache_misses = 0;
    uint64_t plan_cache_hits = 0, plan_cache_misses = 0;
    uint64_t kernel_cache_hits = 0, kernel_cache_misses = 0, disk_cache_hits = 0;
    uint64_t bytes_h2d = 0, bytes_d2h = 0;
    uint64_t serial_units = 0;
    double time_fusion = 0, time_codegen = 0, time_compile = 0, time_exec_host = 0;
    std::vector<UnitRecord> records; // filled when profiling
};

class EngineCUDA {
public:
    explicit EngineCUDA(component::ComponentVE &comp);
    ~EngineCUDA();

    void execute(BhIR *bhir);                  // the repeat loop of one flush
    void handleExecution(BhIR *bhir);          // one pass over the instruction list
    void handleExtmethod(BhIR *bhir);          // split around extension methods

    // Memory interface (ComponentImpl methods are thin wrappers).
    void *getMemoryPointer(bh_base &base, bool copy2host, bool force_alloc, bool nullify);
    void setMemoryPointer(bh_base *base, bool host_ptr, void *mem);
    void copyToHost(const std::set<bh_base *> &bases, bool evict);
    void copyAllBasesToHost();
    void *getBuffer(bh_base *base); // device pointer (allocated/uploaded on demand)
    void delBuffer(bh_base *base);
    void synchronize();

    // Page-locked host memory that the engine frees (cudaFreeHost) when its base is freed.
    void *host_alloc(int64_t nbytes);
    // Events around the last execute() on the engine's stream.
    void record_execute_begin();
    void record_execute_end();
    double last_execute_ms();

    std::string info() const;
    std::string statistics() const;
    void resetStatistics();
    Stats &stats() { return _stats; }
    void *stream() const { return _stream; }
    int smCount() const { return _sm_count; }

    // Launch a compiled unit with the given host-side parameter bytes.
    void launch(const LaunchUnit &u, const std::vector<uint8_t> &params, const std::string *tag = nullptr);
    // Build the parameter bytes of a unit for the current buffers.
    std::vector<uint8_t> pack_params(const LaunchUnit &u);
    // Compiled function for a unit (compiles on first use).
    void *function_for(const LaunchUnit &u);

    // Configuration
    bool prof = false;
    bool verbose = false;
    CodegenOptions cg_opt;
    jitk::FusionConfig fusion_config;
    std::string batch_mode = "off"; // off | grouped | graph
    bool fmad = false;
    std::string cache_dir;
    uint64_t last_error_index = 0;

private:
    component::ComponentVE &comp;
    std::unique_ptr<DeviceApi> api;
    void *_stream = nullptr;
    int _device = 0;
    int _sm_count = 148;
    Stats _stats;

    struct DevBuf {
        void *ptr = nullptr;
        int64_t nbytes = 0;
        bool external = false; // adopted from setMemoryPointer(host_ptr=false)
    };
    std::unordered_map<bh_base *, DevBuf> buffers;
    std::set<bh_base *> host_stale; // device copy newer than the host copy
    std::set<void *> pinned;        // host blocks from host_alloc()
    void *ev_begin = nullptr, *ev_end = nullptr;

    // Kernel cache: source hash -> function
    std::unordered_map<uint64_t, void *> functions;
    std::unordered_map<void *, int> occupancy; // function -> resident CTAs per SM

    // Scratch arena for grid reductions and the error record.
    void *scratch = nullptr;
    int64_t scratch_bytes = 0;
    unsigned int *counters = nullptr;
    unsigned long long *err_record = nullptr;
    void *ensure_scratch(int64_t bytes);

    // Fuse cache: instruction-list hash -> block list and base order
    struct FusePayload {
        std::vector<jitk::Block> block_list;
        std::vector<bh_base *> base_ids;
    };
    std::unordered_map<uint64_t, FusePayload> fuse_cache;

    void copyToDevice(bh_base *base);
    void setConstructorFlag(std::vector<bh_instruction *> &instr_list);
    std::vector<jitk::LoopB> kernels_for(std::vector<bh_instruction *> &instr_list);
    void run_kernels(const std::vector<jitk::LoopB> &kernels);
    void free_base(bh_base *base);
    void check_error_record();
};

} // namespace cuda
} // namespace bohrium
