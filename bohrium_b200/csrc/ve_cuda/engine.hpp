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
#include <unordered_set>
#include <vector>
#include <bohrium/bh_component.hpp>
#include "../jitk/costmodel.hpp"
#include "../jitk/fuser.hpp"
#include "codegen.hpp"

struct bh_costmodel; // the cost model's network (mlp.cu)

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
    uint64_t kernel_cache_hits = 0, kernel_cache_misses = 0, disk_cache_hits = 0, disk_cache_rejected = 0;
    uint64_t fma_contractions = 0, eager_uploads = 0, tma_units = 0, pack_reuses = 0;
    uint64_t bytes_h2d = 0, bytes_d2h = 0;
    uint64_t serial_units = 0;
    // learned fusion: structures tried with both plans, kept learned / kept greedy, learned plan
    // identical to the greedy one, learned plan rejected because a reduction order differed
    uint64_t learned_trials = 0, learned_kept = 0, greedy_kept = 0, learned_same = 0, learned_order_differs = 0;
    uint64_t learned_predictions = 0;
    uint64_t parallel_compiles = 0; // sources compiled ahead in parallel
    uint64_t tuned_kernels = 0, tuned_capped = 0, tune_launches = 0;
    double time_learned_fusion = 0; // learned plans: contraction, lowering and compilation
    double time_learned_choose = 0; // of which the cost model's merge choices (features + inference)
    double time_fusion = 0, time_codegen = 0, time_compile = 0, time_exec_host = 0;
    double time_prepare = 0, time_launch = 0; // host time: list clean-up + hashing, plan execution
    std::vector<UnitRecord> records; // filled when profiling
};

class EngineCUDA {
public:
    explicit EngineCUDA(component::ComponentVE &comp);
    ~EngineCUDA();

    void execute(BhIR *bhir);                  // the repeat loop of one flush
    const BhIR *cur_ir = nullptr;              // the BhIR execute() runs and its registered hints
    BhIRHints cur_hints;
    // Host-side fault injection for tests ("CUDA: inject nvrtc N" / "CUDA: inject alloc N"): the
    // next N kernel compilations fail as NVRTC failures, the next N array allocations as
    // cudaErrorMemoryAllocation, without calling NVRTC or the allocator.
    int inject_nvrtc_failures = 0, inject_alloc_failures = 0;
    // TILE2D tensor maps: encoded per plain launch (grouped launches run those units without TMA).
    bool packing_grouped = false;
    bool tma_check_pending = false;  // a TMA unit ran since the error record was last read
    bool encode_tile_map(const ParamField &f, const bh_base *b, void *p, uint8_t *out);
    void check_tma_record();
    void handleExecution(BhIR *bhir);          // one pass over the instruction list
    void handleExtmethod(BhIR *bhir);          // split around extension methods
    // ComponentImpl::userKernel with tag "cuda": compile `kernel` with NVRTC, run its
    // `extern "C" __global__ void execute(...)` with one device pointer per operand base, on a grid
    // given by `param` ("global_work_size: ...; local_work_size: ..."), and wait for it. Returns ""
    // on success, else the error text.
    std::string userKernel(const std::string &kernel, std::vector<bh_view> &operands, const std::string &param);

    // Memory interface (ComponentImpl methods are thin wrappers).
    void *getMemoryPointer(bh_base &base, bool copy2host, bool force_alloc, bool nullify);
    void setMemoryPointer(bh_base *base, bool host_ptr, void *mem);
    void copyToHost(const std::set<bh_base *> &bases, bool evict);
    void copyAllBasesToHost();
    void *getBuffer(bh_base *base); // device pointer (allocated/uploaded on demand)
    void mark_device_written(bh_base *base) { host_stale.insert(base); }
    void delBuffer(bh_base *base);
    void synchronize_all();  // the engine stream and the copy stream of eager uploads
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
        void *fn = nullptr, *fn_batch = nullptr; // the variant in use
        int occ = 1, occ_batch = 1;
        // Autotuning (tune.cpp): register-capped variants of the same source, timed on their
        // first launches; the fastest becomes fn/fn_batch. Variants compute identical results.
        struct Variant {
            void *fn = nullptr, *fn_batch = nullptr;
            int occ = 1, occ_batch = 1, maxrreg = 0, unroll = 0, regs = 0;
            int ctas = 0;  // CTAs per SM of the plain launch (0: as many as fit)
            std::vector<float> ms, ms_batch;
            int ctas_per_sm() const { return ctas > 0 && ctas < occ ? ctas : occ; }
        };
        std::vector<Variant> variants; // [0]: the default compilation
        std::string name, source;
        bool tuned = false, tuning = false, tuned_batch = false;
        int chosen = 0, chosen_batch = 0; // fn_batch/occ_batch come from variants[chosen_batch]
    };
    // Compiled kernels of a unit (NVRTC on first use, then the in-memory or disk cache).
    Compiled *compiled_for(const LaunchUnit &u);

    // Merge chooser used when the fuser list contains "learned" (set by the cost model).
    jitk::MergeChooser chooser;

    // Learned fusion (learned.cpp). With a cost model loaded and `learned_on`, a flush structure
    // seen for the first time also gets a learned plan (greedy contraction ordered by the model's
    // predicted gain, every merge still legal by mergeable()). The learned plan is tried only when
    // it folds every floating-point sum and product in the same order as the greedy plan (so its
    // results are bit-identical); both plans are then timed on the device `learned_runs` times and
    // the faster one is kept for that structure.
    bool learned_on = false;
    bool record = false;           // record (features, device microseconds) of every kernel run
    int learned_runs = 3;
    double learned_margin = 0.03; // the learned plan is kept when at least this much faster
    double learned_min_gain_us = 0.0;
    // Load a model file written by bohrium_b200/costmodel.py (CostModel.save); throws on error.
    void load_costmodel(const std::string &path);
    bool has_costmodel() const { return cm != nullptr; }
    // Replace the pre-fuser and transformer list (comma-separated names) and forget every plan.
    void set_fusion(const std::string &pre_fuser, const std::string &fuser_list);
    // Write the recorded rows (float32: features then microseconds); returns the row count.
    size_t dump_records(const std::string &path) const;
    void clear_records() { records.clear(); }
    size_t record_count() const { return records.size() / (jitk::kCostFeatures + 1); }

    // Configuration
    bool prof = false;
    bool verbose = false;
    CodegenOptions cg_opt;
    jitk::FusionConfig fusion_config;
    std::string batch_mode = "off"; // off | grouped | graph
    bool fmad = false;
    bool fma_contract = true; // multiply-add contraction on the bytecode (contract.cpp)
    bool autotune = true;            // tune register caps of kernels with large work
    int64_t tune_min_elements = 1 << 20;
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
        bool external = false;    // adopted from setMemoryPointer(host_ptr=false)
        void *arrival = nullptr;  // cudaEvent_t of an eager upload the engine's stream has not waited for
    };
    // Eager uploads: page-locked host data handed over with setMemoryPointer(host_ptr=true) is
    // copied at once on a copy stream of its own, so that the copy overlaps kernels on the
    // engine's stream that do not read it. The engine's stream waits for the copy (settle) before
    // anything on it uses the buffer.
    bool eager_upload = true;
    void *_copy_stream = nullptr;
    std::vector<void *> spare_events;
    void eager_copy(bh_base *base);
    void settle(DevBuf &b);
    std::unordered_map<bh_base *, DevBuf> buffers;
    std::unordered_set<bh_base *> host_stale; // device copy newer than the host copy
    std::set<void *> pinned;        // host blocks from host_alloc()
    void *ev_begin = nullptr, *ev_end = nullptr, *tm_begin = nullptr, *tm_end = nullptr;

    // Kernel cache: source hash -> compiled kernels; cubins compiled ahead of loading
    std::unordered_map<uint64_t, Compiled> functions;
    std::unordered_map<uint64_t, std::vector<char>> ahead;
    std::unordered_map<uint64_t, void *> user_functions; // user-kernel source hash -> its execute()
    std::string disk_cache_path(const std::string &source, int maxrreg = 0) const; // "" without a cache dir
    Compiled::Variant load_variant(const std::vector<char> &cubin, const std::string &name, int maxrreg,
                                   int dyn_smem = 0);
    // Dynamic shared memory of the plain kernels that need it (by CUfunction), used by every launch.
    std::unordered_map<void *, unsigned> fn_shared;
    unsigned shared_bytes_of(void *fn) const;
    static int dynamic_shared_bytes(const std::string &source);
    std::vector<char> cubin_for(const std::string &name, const std::string &source, int maxrreg);
    bool read_cache_file(const std::string &path, std::vector<char> &cubin); // false (and deleted) unless intact
    void write_cache_file(const std::string &path, const std::vector<char> &cubin);
    bool compile_cubin(const std::string &name, const std::string &source, const std::vector<std::string> &opts,
                       std::vector<char> &cubin, std::string &error);
    // Autotuning of plain launches (tune.cpp)
    bool tune_launch(Compiled &c, const LaunchUnit &u, int64_t work, void **args);
    bool tune_batch_launch(Compiled &c, int64_t total, void **args);
    void ensure_variants(Compiled &c);
    struct TuneChoice {
        int maxrreg = 0, unroll = 0, ctas = 0;  // 0: the default
    };
    std::map<uint64_t, TuneChoice> tune_choices; // source hash -> the variant chosen by an earlier run
    void load_tune_choices();
    void save_tune_choice(uint64_t hash, int maxrreg, int unroll, int ctas);
    Compiled::Variant make_variant(const Compiled &c, int maxrreg, int unroll);
    // NVRTC-compile the sources of `units` that are not cached yet, in parallel host threads.
    void precompile(const std::vector<const LaunchUnit *> &units);

    // Scratch arena for grid reductions (tile partials), their completion counters and the error
    // record of bounds-checked kernels.
    void *scratch = nullptr;
    int64_t scratch_bytes = 0;
    unsigned int *counters = nullptr;
    int64_t counter_capacity = 0;
    unsigned long long *err_record = nullptr;
    // SCAN1D chunk totals and carries: regions assigned per plan, kept across the scan's launches.
    void *scan_arena = nullptr;
    int64_t scan_arena_bytes = 0;
    void *ensure_scan_arena(int64_t bytes);
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
        jitk::CostFeatures feat{}; // cost-model features (when recording or learning)
    };
    struct FlushPlan {
        std::vector<PlanKernel> kernels;
        int nlevels = 0;
        size_t nbases = 0;
        // Summation order of every floating-point ADD/MULTIPLY sweep, by origin id.
        std::map<int64_t, std::string> orders;
        int64_t scan_bytes = 0; // scan arena the plan's SCAN1D units need
        std::string signature() const; // kernel names by level (plans with equal signatures match)
    };
    std::unordered_map<uint64_t, FlushPlan> plans;
    // Replay of a fingerprinted BhIR (BhIRHints::fingerprint): the plan, the bases in flush order,
    // the bases freed without being computed, and the bases whose constructor flag the plan
    // assumed (first used as an output) with that flag. A replay only has to re-check those flags.
    // A replay's CUDA graph (batch mode "graph", graph.cpp).
    struct ReplayGraph {
        void *graph = nullptr, *exec = nullptr; // cudaGraph_t, cudaGraphExec_t
        void *params_dev = nullptr;             // parameter blocks of grouped launches
        void *stream = nullptr;
        std::vector<void *> parked;             // buffers of arrays the flush creates and frees
        std::vector<std::pair<bh_base *, void *>> persistent; // other arrays and their buffers
        std::vector<bh_base *> written;         // arrays whose host copy a replay makes stale
        void *scratch = nullptr, *scan_arena = nullptr;
        unsigned int *counters = nullptr;
        size_t nlaunches = 0;
        uint64_t stale_epoch = 0; // host_stale already holds `written` while stale_epoch matches
        ~ReplayGraph();
    };
    // The parameter blocks of one grouped launch of a replay, kept on the device: a later replay
    // launches them again without packing or copying while no buffer changed (buffer_epoch) and
    // the scratch, counter and scan arenas are where they were.
    struct PackCache {
        uint64_t epoch = 0;
        const void *scratch = nullptr, *counters = nullptr, *scan_arena = nullptr;
        uint8_t *dev = nullptr;  // items, then the prefix sums of their work counts
        size_t capacity = 0, bytes = 0, items_bytes = 0, n = 0;
        int64_t total = 0;
        PackCache() = default;
        PackCache(const PackCache &) = delete;
        PackCache &operator=(const PackCache &) = delete;
        ~PackCache();
    };
    struct Replay {
        const FlushPlan *plan = nullptr;
        std::vector<bh_base *> base_ids, dead;
        std::vector<std::pair<bh_base *, bool>> first_outputs;
        // The flush's own instructions (by origin id): plans are shared between flushes of the
        // same structure, so constants and Random123 start/key must come from this flush.
        std::vector<bh_instruction> instr_copy;
        std::vector<bh_instruction *> instrs;
        std::unique_ptr<ReplayGraph> graph;
        bool graph_failed = false;
        int valid_runs = 0;
        uint64_t checked_epoch = 0; // buffer_epoch after the last replay that changed no buffer
        uint64_t stale_after = 0;   // stale_epoch after the last replay (its writes are in host_stale)
        std::map<std::pair<size_t, const Compiled *>, std::unique_ptr<PackCache>> packs; // by level, kernel
    };
    // Bumped on every change of a device buffer or a host data pointer, and on every removal from
    // host_stale; a graph replay that sees both unchanged skips its checks.
    uint64_t buffer_epoch = 1, stale_epoch = 1;
    const std::vector<void *> *ptr_override = nullptr; // per base index: buffer to pack instead
    bool graph_usable(const ReplayGraph &g) const;
    void graph_launch(ReplayGraph &g);
    bool build_graph(Replay &r);
    int launch_raw(void *fn, int64_t grid, void **args); // cuLaunchKernel on the engine's stream
    void launch_dependent(void *fn, int64_t grid, void **args, const char *what); // with PDL when `pdl`
    bool pdl = true; // programmatic dependent launch of plain and grouped launches
    std::unordered_map<uint64_t, Replay> replays;
    bool replay_valid(const Replay &r) const;

    // Learned fusion state (learned.cpp).
    bh_costmodel *cm = nullptr;
    std::vector<float> cm_mean, cm_std;
    float cm_tmean = 0.f, cm_tstd = 1.f;
    std::vector<float> records;
    void *rec_e0 = nullptr, *rec_e1 = nullptr;
    struct Trial {
        FlushPlan greedy, learned;
        std::vector<double> t_greedy, t_learned;
    };
    std::unordered_map<uint64_t, Trial> trials;
    std::set<uint64_t> decided; // structures whose plan choice is final
    std::unordered_map<uint64_t, float> pred_cache; // block key -> predicted microseconds
    int choose_merge(const std::vector<std::pair<const jitk::Block *, const jitk::Block *>> &cands);
    void predict_us(const std::vector<jitk::CostFeatures> &rows, std::vector<float> &out);
    // The learned plan for a structure whose greedy plan was just built; true when a trial starts.
    bool start_trial(uint64_t key, std::vector<bh_instruction *> &instr_list, const std::vector<bh_base *> &base_ids,
                     FlushPlan &greedy);
    void run_trial(uint64_t key, Trial &t, const std::vector<bh_base *> &bases,
                   const std::vector<bh_instruction *> &instrs);
    void record_kernel_times(const FlushPlan &plan, const std::vector<bh_base *> &bases,
                             const std::vector<bh_instruction *> &instrs);
    FlushPlan build_plan(const std::vector<jitk::LoopB> &kernels, const std::vector<bh_base *> &base_ids);
    void run_plan(const FlushPlan &plan, const std::vector<bh_base *> &bases, const std::vector<bh_instruction *> &instrs,
                  Replay *replay = nullptr);
    void pack_params(const PlanUnit &pu, const std::vector<bh_base *> &bases, const std::vector<bh_instruction *> &instrs,
                     int64_t scratch_off, int64_t counter_idx, uint8_t *out);
    void launch_plain(const PlanUnit &pu, const std::vector<bh_base *> &bases, const std::vector<bh_instruction *> &instrs);
    void launch_batched(const std::vector<const PlanUnit *> &group, const std::vector<bh_base *> &bases,
                        const std::vector<bh_instruction *> &instrs, PackCache *cache = nullptr);
    void record_begin(UnitRecord &r, void *&e0);
    void record_end(UnitRecord &r, void *e0);
    // While set, every launch is bracketed by a pair of events from this pool (device busy time
    // of a learned-fusion trial in graph mode, where launch gaps disappear in the replay).
    std::vector<void *> busy_events;
    size_t busy_used = 0;
    bool busy_timing = false;
    void busy_begin();
    void busy_end();
    double busy_ms();

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
