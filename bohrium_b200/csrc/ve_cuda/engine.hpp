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
    uint64_t plan_cache_hits = 0, plan_cache_misses = 0, replays = 0;
    uint64_t kernel_cache_hits = 0, kernel_cache_misses = 0, disk_cache_hits = 0;
    uint64_t bytes_h2d = 0, bytes_d2h = 0;
    uint64_t serial_units = 0;
    double time_fusion = 0, time_codegen = 0, time_compile = 0, time_exec_host = 0;
    double time_prepare = 0, time_launch = 0; // host time: list clean-up + hashing, plan execution
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
    // Events on the engine's stream around an arbitrary region (device time of everything launched
    // between the two calls).
    void timer_start();
    double timer_stop_ms();

    std::string info() const;
    std::string statistics() const;
    void resetStatistics();
    Stats &stats() { return _stats; }
    void *stream() const { return _stream; }
    int smCount() const { return _sm_count; }

    // A compiled unit: the plain kernel, its batched twin and their resident CTAs per SM.
    struct Compiled {
        void *fn = nullptr, *fn_batch = nullptr;
        int occ = 1, occ_batch = 1;
    };
    // Compiled kernels of a unit (NVRTC on first use, then the in-memory or disk cache).
    Compiled *compiled_for(const LaunchUnit &u);

    // Merge chooser used when the fuser list contains "learned" (set by the cost model).
    jitk::MergeChooser chooser;

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
    void *ev_begin = nullptr, *ev_end = nullptr, *tm_begin = nullptr, *tm_end = nullptr;

    // Kernel cache: source hash -> compiled kernels
    std::unordered_map<uint64_t, Compiled> functions;

    // Scratch arena for grid reductions (tile partials), their completion counters and the error
    // record of bounds-checked kernels.
    void *scratch = nullptr;
    int64_t scratch_bytes = 0;
    unsigned int *counters = nullptr;
    int64_t counter_capacity = 0;
    unsigned long long *err_record = nullptr;
    void *ensure_scratch(int64_t bytes);
    unsigned int *ensure_counters(int64_t n);

    // Page-locked staging of batched-launch parameter blocks (recycled per flush).
    uint8_t *staging_host = nullptr, *staging_dev = nullptr;
    size_t staging_capacity = 0, staging_used = 0, last_staging_offset = 0;
    std::vector<void *> staging_retired;
    void *staging_event = nullptr;
    uint8_t *staging_alloc(size_t bytes);
    uint8_t *device_staging(size_t bytes);

    // Flush plans: for a repeated instruction list (same structure, new bases/constants) the
    // compiled launch units are reused and only their parameters are packed again.
    struct PlanUnit {
        LaunchUnit unit;
        Compiled *compiled = nullptr;
        std::vector<int> ptr_base; // per field: index of the base in flush order (PTR fields)
    };
    struct PlanKernel {
        std::vector<PlanUnit> units;
        std::vector<int> frees, writes;
        int level = 0; // dependency level of the first unit
    };
    struct FlushPlan {
        std::vector<PlanKernel> kernels;
        int nlevels = 0;
        size_t nbases = 0;
    };
    std::unordered_map<uint64_t, FlushPlan> plans;
    // Replay of a fingerprinted BhIR (BhIR::_fingerprint): the plan, the bases in flush order,
    // the bases freed without being computed, and the bases whose constructor flag the plan
    // assumed (first used as an output) with that flag. A replay only has to re-check those flags.
    struct Replay {
        const FlushPlan *plan = nullptr;
        std::vector<bh_base *> base_ids, dead;
        std::vector<std::pair<bh_base *, bool>> first_outputs;
        // The flush's own instructions (by origin id): plans are shared between flushes of the
        // same structure, so constants and Random123 start/key must come from this flush.
        std::vector<bh_instruction> instr_copy;
        std::vector<bh_instruction *> instrs;
    };
    std::unordered_map<uint64_t, Replay> replays;
    bool replay_valid(const Replay &r) const;
    FlushPlan build_plan(const std::vector<jitk::LoopB> &kernels, const std::vector<bh_base *> &base_ids);
    void run_plan(const FlushPlan &plan, const std::vector<bh_base *> &bases, const std::vector<bh_instruction *> &instrs);
    void pack_params(const PlanUnit &pu, const std::vector<bh_base *> &bases, const std::vector<bh_instruction *> &instrs,
                     int64_t scratch_off, int64_t counter_idx, uint8_t *out);
    void launch_plain(const PlanUnit &pu, const std::vector<bh_base *> &bases, const std::vector<bh_instruction *> &instrs);
    void launch_batched(const std::vector<const PlanUnit *> &group, const std::vector<bh_base *> &bases,
                        const std::vector<bh_instruction *> &instrs);
    void record_begin(UnitRecord &r, void *&e0);
    void record_end(UnitRecord &r, void *e0);

    // Fuse cache: instruction-list hash -> block list and base order
    struct FusePayload {
        std::vector<jitk::Block> block_list;
        std::vector<bh_base *> base_ids;
    };
    std::unordered_map<uint64_t, FusePayload> fuse_cache;

    void copyToDevice(bh_base *base);
    void setConstructorFlag(std::vector<bh_instruction *> &instr_list);
    uint64_t prepare(std::vector<bh_instruction> &list, std::vector<bh_instruction *> &out,
                     std::vector<bh_base *> &base_ids, bool &sliding, Replay *replay = nullptr);
    std::vector<jitk::LoopB> kernels_for(std::vector<bh_instruction *> &instr_list, uint64_t key,
                                         const std::vector<bh_base *> &base_ids);
    void free_base(bh_base *base);
    void check_error_record();
};

} // namespace cuda
} // namespace bohrium
