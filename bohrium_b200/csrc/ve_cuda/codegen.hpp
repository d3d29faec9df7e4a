// Lowering of fused kernels (jitk::LoopB, rank -1) to sm_100a CUDA source.
//
// The reference emits one generic SIMT loop nest per kernel (core/jitk/engines/engine.cpp:84-336,
// ve/cuda/engine_cuda.cpp:243-274) with fixed 128-thread blocks, hard-coded loop sizes and a CPU
// offload for blocks that sweep their outermost axis (include/bohrium/jitk/engines/engine_gpu.hpp:
// 140-142). Here every fused loop nest is lowered to one of a few launch schedules:
//
//   FLAT          the leading parallel ranks form a (rows x cols) index space processed by a
//                 grid-stride persistent kernel, V elements per thread along the innermost
//                 parallel rank; deeper ranks are serial loops inside the thread.
//   GRID_REDUCE   a 1-D nest that reduces its only axis (maps fused with sum/max/... to a scalar):
//                 fixed tiles of TILE = 256 x 8 elements, a per-tile CTA tree, then the last CTA
//                 folds the tile partials in tile order. The summation order depends only on the
//                 element count, never on the grid size, so batched and plain launches agree bit
//                 for bit.
//   SPLIT_REDUCE  a FLAT nest with few parallel points whose innermost threaded loop holds one
//                 swept sub-loop (axis reductions such as max over the rows of a 2-D array): the
//                 swept axis is cut into chunks so that ~600K threads work at once; each thread folds
//                 its chunk in order, and the last CTA of each 256-point block folds the chunk
//                 partials in chunk order (deterministic) and runs the instructions that follow.
//   LANE_REDUCE   the SPLIT_REDUCE structure when the swept axis is contiguous and there are
//                 enough points: C (power of two <= 256, from the shapes) lanes of one CTA share a
//                 point, lane c folds elements c, c+C, ... (coalesced), and a fixed shuffle tree
//                 combines the lanes; one pass, no scratch. With one point axis, a CTA per point
//                 and a stencil group among its read-only views (views of one base that differ by
//                 whole rows and a few columns), each CTA walks a range of rows and stages the
//                 group's rows in a shared-memory ring with cp.async, one row ahead.
//   OUTER_REDUCE  a nest that reduces its outermost axis into an array: threads own the output
//                 elements (the inner parallel ranks) and loop over the reduced axis.
//   SCAN1D        a 1-D nest with one accumulate (cumulative sum/product) among elementwise
//                 instructions: three units -- chunk totals, one-CTA exclusive scan of the totals,
//                 re-scan with the carry -- each with a fixed block scan (order set by the length).
//                 With scan_windows, A and C run one group of 2048 chunks at a time (C repeating
//                 B's steps for its group), so the re-scan reads the group's inputs from L2.
//   SERIAL        anything else: one thread runs the nest in program order (always correct).
//   TILE2D        a 2-D map that reads arrays through transposed views (unit stride along the outer
//                 rank): tiles of (128 bytes / element) rows x 64 columns; each transposed view's
//                 tile is one box of its base array, loaded by TMA (cp.async.bulk.tensor.2d, 128-byte
//                 swizzle) into a shared-memory ring ahead of the compute, so both the box reads and
//                 the output rows are contiguous; a read-only row-wise view beside them is staged
//                 the same way (one box of its rows). Grouped launches and views the tensor maps
//                 cannot describe take the same tiles with plain loads.
//
// Loop sizes, view offsets/strides and constants are kernel parameters. The source also fixes a
// few choices derived from the sizes (lanes per point, tiles per work item, iterations per lane,
// the stencil ring), so arrays of different sizes may get different kernels; code whose fast path
// assumes a layout (the stencil staging) checks it at launch and falls back otherwise.
#pragma once

#include <cstdint>
#include <functional>
#include <set>
#include <string>
#include <vector>
#include "../jitk/block.hpp"

namespace bohrium {
namespace cuda {

enum class Sched { FLAT, GRID_REDUCE, SPLIT_REDUCE, LANE_REDUCE, OUTER_REDUCE, SCAN1D, SERIAL, TILE2D };

// Engine-internal opcodes made by contract_multiply_add() (contract.cpp), operands (out, a, b, c):
//   BH_X_FMA   out = a*b + c      BH_X_FMS   out = a*b - c      BH_X_FNMA  out = c - a*b
// each with one rounding. At most the multiplier b and the addend c are constants; when both are,
// the instruction's constant is complex of the same precision, (multiplier, addend). Negative ids
// never collide with the Bohrium bytecode or with extension methods (ids above BH_MAX_OPCODE_ID),
// and the instructions never leave the engine's own flush.
constexpr bh_opcode BH_X_FMA = -1001, BH_X_FMS = -1002, BH_X_FNMA = -1003;
bool is_fma_opcode(bh_opcode op);
// Rewrites, in place, every float32/float64 `MUL t, a, b` whose only use is one input of the next
// instruction touching t, an ADD or SUBTRACT, after which t is freed (within 64 instructions each,
// t not synced, a and b not written in between): the ADD becomes the fused instruction, the MUL
// becomes BH_NONE, and FREEs of a or b in between move to just after the ADD. Returns the number
// of contractions.
// `holds_nothing(t)`, when given, says that no data is held for the product's array t (no device
// buffer, no host data): t's FREE is then dropped as well.
int contract_multiply_add(std::vector<bh_instruction> &list, const std::set<bh_base *> &syncs,
                          const std::function<bool(const bh_base *)> &holds_nothing = nullptr);
const char *sched_name(Sched s);

constexpr int kThreads = 256;      // threads per CTA for every schedule
constexpr int kReduceV = 8;        // elements per thread per tile in GRID_REDUCE
constexpr int64_t kReduceTile = kThreads * kReduceV;
constexpr int64_t kScanChunk = 4096; // elements per chunk in SCAN1D

// One 8-byte slot (or two for 16-byte constants) of the kernel parameter struct.
struct ParamField {
    enum Kind { PTR, I64, CONST, R123_START, R123_KEY, SCRATCH, COUNTER, TMAP, TMA_OK } kind;
    bh_base *base = nullptr; // PTR
    int64_t i64 = 0;         // I64
    bh_constant c{};         // CONST / R123_*
    int64_t origin = -1;     // CONST / R123_*: origin id of the instruction holding the constant
    int part = 0;            // CONST: which 8 bytes of the constant (1: the imaginary part of a complex128)
    int64_t off = 0;         // COUNTER: index offset in the unit's counters
    // TMAP: one of the 16 slots (`part`) of a TMA tensor map of `base`, which the engine encodes at
    // launch: a 2-D tiled map of the base seen as rows of `tm_ld` elements (as many whole rows as
    // it holds), boxes of tm_box_x (along a row) x tm_box_y elements, with the 128-byte swizzle
    // when `tm_swizzle`. `i64` is the start of the view the map serves; the view covers tm_xspan
    // elements along a row from its start and tm_yspan rows.
    int64_t tm_ld = 0, tm_box_x = 0, tm_box_y = 0, tm_xspan = 0, tm_yspan = 0;
    bool tm_swizzle = false;
    // TMA_OK: 1 when the engine encoded every tensor map of the unit for a plain launch and each
    // view lies inside its map with 16-byte aligned rows and start; 0 otherwise (grouped launches,
    // unaligned views), which selects the unit's code path without TMA.
};

struct LaunchUnit {
    std::string name;   // kernel function name (derived from the source hash)
    std::string source; // complete CUDA source
    Sched sched = Sched::FLAT;
    int V = 1;          // elements per thread along the innermost parallel rank (FLAT)
    std::vector<ParamField> fields;
    int64_t rows = 1, cols = 1; // FLAT / OUTER_REDUCE index space; GRID_REDUCE/SCAN1D: cols = length
    int nred = 0;               // GRID_REDUCE / SPLIT_REDUCE: number of reductions
    int64_t scratch_bytes_per_tile = 0; // GRID_REDUCE: bytes of partials per tile (all reductions)
    int slot_bytes = 8;         // GRID_REDUCE / SPLIT_REDUCE: bytes of one partial (16 with complex128)
    int64_t chunks = 1;         // SPLIT_REDUCE: chunks of the swept axis; LANE_REDUCE: lanes per point;
                                // GRID_REDUCE: tiles per work item; SCAN1D: work items of the phase
    int64_t batch_chunks = 0;   // GRID_REDUCE: tiles per work item in a grouped launch (0: chunks)
    int64_t scan_bytes = 0;     // SCAN1D: its chunk totals and carries and group totals and carries
    int64_t scan_offset = 0;    // SCAN1D: offset of scan_bytes in the scan arena (set by the plan)
    bool scan_gate = false;     // SCAN1D carry unit: one completion counter
    bool single_pass = false;   // SCAN1D in one pass (lower_scan1d_single): chunks = chunk count
    bool no_batch = false;      // always launched alone (its CTAs wait on one another's results)
    // The parameter members and the device code (without the kernel wrappers) of the source;
    // body_core is empty for sources with wrappers of their own.
    std::string params_decl, body_core;
    // GRID_REDUCE of a small array with order-free reductions only: body_core also defines
    // bh_tail(p), the whole reduction run by one CTA (threads fold strided elements, then one
    // block tree), which another unit's kernel can run in its tail (see fuse_tails).
    bool tail_capable = false;
    // This unit's kernel runs a folded reduction's bh_tail in the CTA that finishes last; the
    // completion counter follows the unit's own counters.
    bool tail = false;
    int64_t work_items() const;
    int64_t grouped_work_items() const; // work items when launched grouped (batch_chunks)
    int64_t scratch_bytes() const;   // partials in the scratch arena
    int64_t counters_needed() const; // completion counters

    // Bytes of arrays read/written by this unit (algorithmic, temporaries excluded).
    int64_t algorithmic_bytes = 0;
    int64_t elements = 0;

    // Summation order of the sweeps this unit reduces across threads, by origin id: "tree:<n>"
    // (GRID_REDUCE) or "split:<chunks>:<chunk length>:<n>" (SPLIT_REDUCE). Every other sweep is
    // folded by one thread in index order ("seq"), whatever the schedule.
    std::vector<std::pair<int64_t, std::string>> red_orders;
};

struct CodegenOptions {
    bool bounds_check = false; // emit index checks that record violations instead of accessing
    int flat_v = 4;            // elements per thread in FLAT
    bool preload_heavy = true;  // preload the inputs of heavy (arithmetic-bound) element bodies too
    int interleave = 1;         // GRID_REDUCE: elements of a heavy body written side by side (1 or 2)
    bool tile2d = true;         // TILE2D for maps over transposed views (else FLAT)
    bool vector_access = true;  // FLAT: 4 consecutive elements per thread, moved as 128-bit words
    bool scan_single_pass = false; // SCAN1D as one pass with look-back (else three units; see lower_scan1d_single)
    bool scan_windows = false;     // SCAN1D units A and C one group of chunks at a time (see lower_scan1d)
    bool stage_bulk = true;        // LANE_REDUCE stencil rows staged by TMA bulk copies (else cp.async)
    bool scan_prefetch = true;     // SCAN1D streaming units read their inputs from a TMA-filled ring
    int64_t scan_spin_cap = int64_t{1} << 22; // polls per look-back wait (negative: give up at once)
};

// Lower one kernel (as produced by jitk::get_kernel_list) into launch units executed in order.
std::vector<LaunchUnit> lower_kernel(const jitk::LoopB &kernel, const CodegenOptions &opt);

// Tail fusion over a flush's lowered kernels (`lowered[k]`: the units of kernel k, empty for
// system-only kernels). A kernel j that is one tail-capable GRID_REDUCE (a small array, order-
// free reductions: max, min, logical, bitwise, integer sums and products -- typically the second
// level of a 2-D max) is folded into its producer k, the last earlier kernel that writes an array
// j reads, when j commutes with every kernel between them and k's last unit is a FLAT /
// GRID_REDUCE / SPLIT_REDUCE / LANE_REDUCE / OUTER_REDUCE unit: every CTA runs the first unit's
// work, and the CTA that arrives last on an acquire-release completion counter runs the
// reduction. Kernel j's unit list is emptied. Returns, per kernel, the kernel it was folded into
// (-1: none).
std::vector<int> fuse_tails(const std::vector<jitk::LoopB> &kernels, std::vector<std::vector<LaunchUnit>> &lowered,
                            const CodegenOptions &opt);

// CUDA element type name (the "long long" family is used for 64-bit integers).
std::string cuda_type(bh_type t);

} // namespace cuda
} // namespace bohrium
