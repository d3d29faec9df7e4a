// Kernel source generation; see codegen.hpp for the schedules.
//
// Operation semantics (one C statement per bytecode, NumPy rules for signed integer division and
// remainder, reductions as `acc = acc op x`, accumulates as `out[i] = out[i-1] op in[i]`) follow
// core/jitk/instruction.cpp:58-544 of the reference; temporaries and scalar replacement of
// reduction outputs follow core/jitk/engines/engine.cpp:84-249.
#include <algorithm>
#include <cassert>
#include <cstring>
#include <functional>
#include <map>
#include <regex>
#include <set>
#include <sstream>
#include <stdexcept>
#include "codegen.hpp"

using namespace std;
using bohrium::jitk::Block;
using bohrium::jitk::InstrPtr;
using bohrium::jitk::LoopB;

namespace bohrium {
namespace cuda {

const char *sched_name(Sched s) {
    switch (s) {
        case Sched::FLAT: return "flat";
        case Sched::GRID_REDUCE: return "grid_reduce";
        case Sched::SPLIT_REDUCE: return "split_reduce";
        case Sched::LANE_REDUCE: return "lane_reduce";
        case Sched::OUTER_REDUCE: return "outer_reduce";
        case Sched::SCAN1D: return "scan1d";
        case Sched::SERIAL: return "serial";
        case Sched::TILE2D: return "tile2d";
    }
    return "?";
}

int64_t LaunchUnit::work_items() const {
    switch (sched) {
        case Sched::FLAT: {
            const int64_t per = static_cast<int64_t>(kThreads) * V;
            return rows * ((cols + per - 1) / per);
        }
        case Sched::GRID_REDUCE: {
            const int64_t tiles = (cols + kReduceTile - 1) / kReduceTile;
            return (tiles + chunks - 1) / chunks;  // chunks: tiles per work item
        }
        case Sched::SPLIT_REDUCE: return (rows * cols + kThreads - 1) / kThreads * chunks;
        case Sched::LANE_REDUCE: {
            const int64_t per = kThreads / chunks;
            return (rows * cols + per - 1) / per;
        }
        case Sched::OUTER_REDUCE: return (rows * cols + kThreads - 1) / kThreads;
        case Sched::SCAN1D: return chunks;  // chunks: work items of the phase
        case Sched::SERIAL: return 1;
        case Sched::TILE2D: return (rows + V - 1) / V * ((cols + 63) / 64);  // V: rows per tile
    }
    return 1;
}

int64_t LaunchUnit::grouped_work_items() const {
    if (sched == Sched::GRID_REDUCE && batch_chunks > 0 && batch_chunks != chunks) {
        const int64_t tiles = (cols + kReduceTile - 1) / kReduceTile;
        return (tiles + batch_chunks - 1) / batch_chunks;
    }
    return work_items();
}

int64_t LaunchUnit::scratch_bytes() const {
    if (sched == Sched::GRID_REDUCE) return (cols + kReduceTile - 1) / kReduceTile * scratch_bytes_per_tile;
    if (sched == Sched::SPLIT_REDUCE) return slot_bytes * static_cast<int64_t>(nred) * chunks * rows * cols;
    if (sched == Sched::SCAN1D) return 0;  // totals/carries live in the engine's scan arena
    return 0;
}

int64_t LaunchUnit::counters_needed() const {
    int64_t own = 0;
    if (sched == Sched::SCAN1D && single_pass) {
        // chunk, thread-sum, warp-total and group flags (one spare), ticket, CTAs that left, abort
        const int64_t ngroups = (chunks + kThreads * 8 - 1) / (kThreads * 8);
        own = chunks + (chunks + 7) / 8 + (chunks + 255) / 256 + ngroups + 1 + 3;
    }
    if (sched == Sched::GRID_REDUCE) own = 1;
    if (sched == Sched::SPLIT_REDUCE) own = (rows * cols + kThreads - 1) / kThreads;
    if (sched == Sched::SCAN1D && scan_gate) own = 1;
    return tail ? own + 1 : own;  // the tail's completion counter follows
}

string cuda_type(bh_type t) {
    switch (t) {
        case bh_type::BOOL: return "bool";
        case bh_type::INT8: return "signed char";
        case bh_type::INT16: return "short";
        case bh_type::INT32: return "int";
        case bh_type::INT64: return "long long";
        case bh_type::UINT8: return "unsigned char";
        case bh_type::UINT16: return "unsigned short";
        case bh_type::UINT32: return "unsigned int";
        case bh_type::UINT64: return "unsigned long long";
        case bh_type::FLOAT32: return "float";
        case bh_type::FLOAT64: return "double";
        case bh_type::COMPLEX64: return "bh_c64";
        case bh_type::COMPLEX128: return "bh_c128";
        case bh_type::R123: return "bh_r123";
    }
    throw runtime_error("cuda_type(): unknown type");
}

namespace {

// ------------------------------------------------------------------------------- kernel prelude
// Common device helpers: Philox2x32-10 (the counter-based generator behind BH_RANDOM, restated
// from Salmon et al., "Parallel Random Numbers: As Easy as 1, 2, 3", SC'11: ten rounds of
// (hi, lo) = M * x0; x0' = hi ^ k ^ x1; x1' = lo with the key bumped by W between rounds), warp
// shuffles for every element type and a small complex type.
const char *kPrelude = R"CUDA(
typedef long long bh_i64;
typedef unsigned long long bh_u64;
struct bh_r123 { bh_u64 start, key; };

// Programmatic dependent launch: a kernel launched with programmatic stream serialization may
// start while the kernel before it in the stream finishes; it waits here, before touching memory,
// until that kernel has completed and its writes are visible, and lets the next kernel start
// early in turn. For a launch without the attribute both are no-ops.
__device__ __forceinline__ void bh_grid_dependency() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__device__ __forceinline__ bh_u64 bh_random123(bh_u64 start, bh_u64 key, bh_u64 index) {
    const bh_u64 c = start + index;
    unsigned x0 = (unsigned)c, x1 = (unsigned)(c >> 32), k = (unsigned)key;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const unsigned hi = __umulhi(0xD256D193u, x0);
        const unsigned lo = 0xD256D193u * x0;
        x0 = hi ^ k ^ x1;
        x1 = lo;
        k += 0x9E3779B9u;
    }
    return ((bh_u64)x1 << 32) | (bh_u64)x0;
}

template <typename T> __device__ __forceinline__ T bh_shfl_xor(T v, int m) {
    if (sizeof(T) == 16) {
        long long x[2]; memcpy(x, &v, 16);
        x[0] = __shfl_xor_sync(0xffffffffu, x[0], m);
        x[1] = __shfl_xor_sync(0xffffffffu, x[1], m);
        T r; memcpy(&r, x, 16); return r;
    } else if (sizeof(T) == 8) {
        long long x; memcpy(&x, &v, 8);
        x = __shfl_xor_sync(0xffffffffu, x, m);
        T r; memcpy(&r, &x, 8); return r;
    } else {
        int x = 0; memcpy(&x, &v, sizeof(T));
        x = __shfl_xor_sync(0xffffffffu, x, m);
        T r; memcpy(&r, &x, sizeof(T)); return r;
    }
}

template <typename T> __device__ __forceinline__ T bh_shfl_idx(T v, int src) {
    long long x[2] = {0, 0};
    memcpy(x, &v, sizeof(T));
    x[0] = __shfl_sync(0xffffffffu, x[0], src);
    if (sizeof(T) > 8) x[1] = __shfl_sync(0xffffffffu, x[1], src);
    T r; memcpy(&r, x, sizeof(T)); return r;
}

template <typename T> __device__ __forceinline__ T bh_shfl_up(T v, int d) {
    long long x[2] = {0, 0};
    memcpy(x, &v, sizeof(T));
    x[0] = __shfl_up_sync(0xffffffffu, x[0], d);
    if (sizeof(T) > 8) x[1] = __shfl_up_sync(0xffffffffu, x[1], d);
    T r; memcpy(&r, x, sizeof(T)); return r;
}

// Completion counter of a reduction: an acquire-release increment at device scope, so the
// partials this thread stored before are visible to whichever CTA sees the final count.
__device__ __forceinline__ unsigned bh_arrive(unsigned *counter) {
    unsigned old;
    asm volatile("atom.add.acq_rel.gpu.u32 %0, [%1], 1;" : "=r"(old) : "l"(counter) : "memory");
    return old;
}
__device__ __forceinline__ unsigned bh_arrive_n(unsigned *counter, unsigned n) {
    unsigned old;
    asm volatile("atom.add.acq_rel.gpu.u32 %0, [%1], %2;" : "=r"(old) : "l"(counter), "r"(n) : "memory");
    return old;
}
__device__ __forceinline__ void bh_acquire() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// Load through L2 only (ld.global.cg): for values that other CTAs wrote during this launch.
template <typename T> __device__ __forceinline__ T bh_ldcg(const T *ptr) {
    T r;
    if (sizeof(T) == 16) {
        long long x[2];
        x[0] = __ldcg((const long long *)ptr);
        x[1] = __ldcg((const long long *)ptr + 1);
        memcpy(&r, x, 16);
    } else if (sizeof(T) == 8) {
        const long long x = __ldcg((const long long *)ptr); memcpy(&r, &x, 8);
    } else if (sizeof(T) == 4) {
        const int x = __ldcg((const int *)ptr); memcpy(&r, &x, 4);
    } else if (sizeof(T) == 2) {
        const short x = __ldcg((const short *)ptr); memcpy(&r, &x, 2);
    } else {
        const signed char x = __ldcg((const signed char *)ptr); memcpy(&r, &x, 1);
    }
    return r;
}

// Integer power by repeated squaring: exact wherever the result fits the type (CUDA's double pow
// can be an ulp below an exact integer, which truncation would turn into the wrong integer).
// Negative exponents give what pow() truncates to: 1 for a base of 1, +-1 for -1, else 0.
template <typename T> __device__ __forceinline__ T bh_ipow(T b, T e) {
    if (e < (T)0) {
        if (b == (T)1) return (T)1;
        if (b == (T)-1) return (e & (T)1) ? (T)-1 : (T)1;
        return (T)0;
    }
    T r = (T)1;
    while (e) {
        if (e & (T)1) r = (T)(r * b);
        e = (T)(e >> 1);
        b = (T)(b * b);
    }
    return r;
}
)CUDA";

// Complex element types (added to the sources of units that use them). bh_c64/bh_c128 have the
// memory layout of C99's float/double complex and of the bh_constant union (real, imaginary).
// Arithmetic is written from the definitions; division is Smith's algorithm (R. L. Smith,
// "Algorithm 116: Complex division", CACM 5(8), 1962), which scales by the larger component of
// the divisor. The elementary functions use the textbook identities:
//   exp(x+iy) = e^x (cos y + i sin y);  log z = ln|z| + i atan2(y, x), with ln|z| taken as
//   log1p((x-1)(x+1) + y^2)/2 near |z| = 1 (where log(hypot) loses the small result);
//   sqrt z: t = sqrt((|x| + |z|)/2), z^(1/2) = t + iy/(2t) for x >= 0, |y|/(2t) + i sign(y) t else;
//   sin, cos, sinh, cosh by the addition theorems; tan z = (sin x cos x + i sinh y cosh y) /
//   (cos^2 x + sinh^2 y) and tanh z = (sinh x cosh x + i sin y cos y) / (sinh^2 x + cos^2 y),
//   which stay accurate near the poles, with the limit +-i (tan) or +-1 (tanh) once the hyperbolic
//   terms would overflow; a^b = exp(b log a).
const char *kComplexPrelude = R"CUDA(
struct bh_c128;
struct alignas(8) bh_c64 {
    float re, im;
    bh_c64() = default;
    __device__ __forceinline__ constexpr bh_c64(float r, float i = 0.0f) : re(r), im(i) {}
    __device__ __forceinline__ bh_c64(const bh_c128 &z);
};
struct alignas(16) bh_c128 {
    double re, im;
    bh_c128() = default;
    __device__ __forceinline__ constexpr bh_c128(double r, double i = 0.0) : re(r), im(i) {}
    __device__ __forceinline__ bh_c128(const bh_c64 &z) : re(z.re), im(z.im) {}
};
__device__ __forceinline__ bh_c64::bh_c64(const bh_c128 &z) : re((float)z.re), im((float)z.im) {}

template <typename C> struct bh_cpart;
template <> struct bh_cpart<bh_c64> { typedef float R; static constexpr float hyp_max = 40.0f; };
template <> struct bh_cpart<bh_c128> { typedef double R; static constexpr double hyp_max = 300.0; };

__device__ __forceinline__ void bh_sincos(float x, float *s, float *c) { sincosf(x, s, c); }
__device__ __forceinline__ void bh_sincos(double x, double *s, double *c) { sincos(x, s, c); }

#define BH_COMPLEX_OPERATORS(C)                                                                    \
    __device__ __forceinline__ C operator+(C a, C b) { return C(a.re + b.re, a.im + b.im); }        \
    __device__ __forceinline__ C operator-(C a, C b) { return C(a.re - b.re, a.im - b.im); }        \
    __device__ __forceinline__ C operator*(C a, C b) {                                             \
        return C(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);                            \
    }                                                                                              \
    __device__ __forceinline__ C operator/(C a, C b) {                                             \
        if (fabs(b.re) >= fabs(b.im)) {                                                            \
            const auto r = b.im / b.re, d = b.re + b.im * r;                                       \
            return C((a.re + a.im * r) / d, (a.im - a.re * r) / d);                                \
        }                                                                                          \
        const auto r = b.re / b.im, d = b.re * r + b.im;                                           \
        return C((a.re * r + a.im) / d, (a.im * r - a.re) / d);                                    \
    }                                                                                              \
    __device__ __forceinline__ bool operator==(C a, C b) { return a.re == b.re && a.im == b.im; }  \
    __device__ __forceinline__ bool operator!=(C a, C b) { return a.re != b.re || a.im != b.im; }
BH_COMPLEX_OPERATORS(bh_c64)
BH_COMPLEX_OPERATORS(bh_c128)

template <typename C> __device__ __forceinline__ typename bh_cpart<C>::R bh_cabs(C z) { return hypot(z.re, z.im); }
template <typename C> __device__ __forceinline__ C bh_conj(C z) { return C(z.re, -z.im); }
template <typename C> __device__ __forceinline__ C bh_csign(C z) {
    typedef typename bh_cpart<C>::R R;
    const R v = z.re == (R)0 ? (R)((z.im > (R)0) - ((R)0 > z.im)) : (R)((z.re > (R)0) - ((R)0 > z.re));
    return C(v, (R)0);
}
template <typename C> __device__ __forceinline__ C bh_cexp(C z) {
    typedef typename bh_cpart<C>::R R;
    const R e = exp(z.re);
    R s, c;
    bh_sincos(z.im, &s, &c);
    return C(e * c, e * s);
}
template <typename C> __device__ __forceinline__ C bh_clog(C z) {
    typedef typename bh_cpart<C>::R R;
    const R h = hypot(z.re, z.im);
    const R lr = (h > (R)0.75 && h < (R)1.25)
                     ? (R)0.5 * log1p((z.re - (R)1) * (z.re + (R)1) + z.im * z.im)
                     : log(h);
    return C(lr, atan2(z.im, z.re));
}
template <typename C> __device__ __forceinline__ C bh_clog10(C z) {
    // the complex log divided by log(10.0f): ln 10 rounded to float, as the reference's engines do
    typedef typename bh_cpart<C>::R R;
    const C l = bh_clog(z);
    const R ln10 = (R)logf(10.0f);
    return C(l.re / ln10, l.im / ln10);
}
template <typename C> __device__ __forceinline__ C bh_csqrt(C z) {
    typedef typename bh_cpart<C>::R R;
    if (z.re == (R)0 && z.im == (R)0) return C((R)0, z.im);
    const R t = sqrt((fabs(z.re) + hypot(z.re, z.im)) * (R)0.5);
    if (z.re >= (R)0) return C(t, z.im / (t + t));
    return C(fabs(z.im) / (t + t), copysign(t, z.im));
}
template <typename C> __device__ __forceinline__ C bh_csin(C z) {
    typedef typename bh_cpart<C>::R R;
    R s, c;
    bh_sincos(z.re, &s, &c);
    return C(s * cosh(z.im), c * sinh(z.im));
}
template <typename C> __device__ __forceinline__ C bh_ccos(C z) {
    typedef typename bh_cpart<C>::R R;
    R s, c;
    bh_sincos(z.re, &s, &c);
    return C(c * cosh(z.im), -(s * sinh(z.im)));
}
template <typename C> __device__ __forceinline__ C bh_csinh(C z) {
    typedef typename bh_cpart<C>::R R;
    R s, c;
    bh_sincos(z.im, &s, &c);
    return C(sinh(z.re) * c, cosh(z.re) * s);
}
template <typename C> __device__ __forceinline__ C bh_ccosh(C z) {
    typedef typename bh_cpart<C>::R R;
    R s, c;
    bh_sincos(z.im, &s, &c);
    return C(cosh(z.re) * c, sinh(z.re) * s);
}
template <typename C> __device__ __forceinline__ C bh_ctan(C z) {
    typedef typename bh_cpart<C>::R R;
    R s, c;
    bh_sincos(z.re, &s, &c);
    if (fabs(z.im) > bh_cpart<C>::hyp_max) return C(copysign((R)0, s * c), copysign((R)1, z.im));
    const R sh = sinh(z.im), ch = cosh(z.im);
    const R d = c * c + sh * sh;
    return C(s * c / d, sh * ch / d);
}
template <typename C> __device__ __forceinline__ C bh_ctanh(C z) {
    typedef typename bh_cpart<C>::R R;
    R s, c;
    bh_sincos(z.im, &s, &c);
    if (fabs(z.re) > bh_cpart<C>::hyp_max) return C(copysign((R)1, z.re), copysign((R)0, s * c));
    const R sh = sinh(z.re), ch = cosh(z.re);
    const R d = sh * sh + c * c;
    return C(sh * ch / d, s * c / d);
}
template <typename C> __device__ __forceinline__ C bh_cpow(C a, C b) {
    typedef typename bh_cpart<C>::R R;
    if (a.re == (R)0 && a.im == (R)0) {
        if (b.re == (R)0 && b.im == (R)0) return C((R)1, (R)0);
        if (b.im == (R)0 && b.re > (R)0) return C((R)0, (R)0);
    }
    return bh_cexp(b * bh_clog(a));
}
)CUDA";

// ---------------------------------------------------------------------------- operation emitting
// TMA and mbarrier helpers of TILE2D units (inline PTX for sm_100a). A tensor map is a kernel
// parameter (the plain kernel's __grid_constant__ struct), so the bulk-tensor copy reads it from
// parameter space. Waits on an mbarrier poll a bounded number of times and report failure instead
// of spinning forever.
const char *kTmaPrelude = R"CUDA(
struct alignas(64) bh_tmap { unsigned long long w[16]; };
__device__ __forceinline__ unsigned bh_saddr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void bh_mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(bh_saddr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void bh_mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void bh_mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bh_saddr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool bh_mbar_try_wait(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok) : "r"(bh_saddr(bar)), "r"(parity) : "memory");
    return ok != 0u;
}
__device__ __forceinline__ bool bh_mbar_wait(unsigned long long *bar, unsigned parity) {
    for (int i = 0; i < (1 << 20); ++i)
        if (bh_mbar_try_wait(bar, parity)) return true;
    return false;
}
// One contiguous global -> shared copy by the TMA engine (16-byte aligned addresses, a multiple
// of 16 bytes), counted on `bar`; the copy lands in this CTA's shared memory only.
__device__ __forceinline__ void bh_bulk_row(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(bh_saddr(dst)), "l"(src), "r"(bytes), "r"(bh_saddr(bar)) : "memory");
}
__device__ __forceinline__ void bh_tma_2d(void *dst, const bh_tmap *map, int x, int y, unsigned long long *bar) {
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                 :: "r"(bh_saddr(dst)), "l"(map), "r"(x), "r"(y), "r"(bh_saddr(bar)) : "memory");
}
)CUDA";

bool is_float(bh_type t) { return t == bh_type::FLOAT32 || t == bh_type::FLOAT64; }

// Name of a math function for element type `t` (float uses the f-suffixed variant, as C's
// <tgmath.h> does for the reference's generated C code).
string fn(const char *name, bh_type t) { return t == bh_type::FLOAT32 ? string(name) + "f" : string(name); }

string sign_expr(const string &x) { return "((" + x + " > 0) - (0 > " + x + "))"; }

// Bytes of one reduction partial in scratch: 8, or 16 when a reduction is complex128.
int red_slot_bytes(const vector<InstrPtr> &reds) {
    for (const InstrPtr &r : reds)
        if (r->operand[0].base->dtype() == bh_type::COMPLEX128) return 16;
    return 8;
}

// The combine expression of a reduction: `acc op x`.
string reduce_expr(bh_opcode op, const string &acc, const string &x) {
    switch (op) {
        case BH_ADD_REDUCE: return acc + " + " + x;
        case BH_MULTIPLY_REDUCE: return acc + " * " + x;
        case BH_MINIMUM_REDUCE: return acc + " < " + x + " ? " + acc + " : " + x;
        case BH_MAXIMUM_REDUCE: return acc + " > " + x + " ? " + acc + " : " + x;
        case BH_LOGICAL_AND_REDUCE: return acc + " && " + x;
        case BH_LOGICAL_OR_REDUCE: return acc + " || " + x;
        case BH_LOGICAL_XOR_REDUCE: return "!" + acc + " != !" + x;
        case BH_BITWISE_AND_REDUCE: return acc + " & " + x;
        case BH_BITWISE_OR_REDUCE: return acc + " | " + x;
        case BH_BITWISE_XOR_REDUCE: return acc + " ^ " + x;
        default: throw runtime_error(string("reduce_expr(): not a reduction: ") + bh_opcode_text(op));
    }
}

// One statement for an instruction with a complex operand (the complex type signatures of
// core/codegen/opcodes.json; semantics of core/jitk/instruction.cpp:58-544 for C99 complex:
// ISNAN/ISINF/ISFINITE test the real part, SIGN is csgn with a zero imaginary part). Arithmetic,
// comparisons, reductions, accumulates and conversions use the operators and converting
// constructors of bh_c64/bh_c128.
string complex_statement(const bh_instruction &instr, const vector<string> &ops) {
    const bh_opcode op = instr.opcode;
    const string &o = ops[0];
    auto call = [&](const char *f) { return o + " = " + f + "(" + ops[1] + ");"; };
    switch (op) {
        case BH_ADD: return o + " = " + ops[1] + " + " + ops[2] + ";";
        case BH_SUBTRACT: return o + " = " + ops[1] + " - " + ops[2] + ";";
        case BH_MULTIPLY: return o + " = " + ops[1] + " * " + ops[2] + ";";
        case BH_DIVIDE: return o + " = " + ops[1] + " / " + ops[2] + ";";
        case BH_POWER: return o + " = bh_cpow(" + ops[1] + ", " + ops[2] + ");";
        case BH_EQUAL: return o + " = " + ops[1] + " == " + ops[2] + ";";
        case BH_NOT_EQUAL: return o + " = " + ops[1] + " != " + ops[2] + ";";
        case BH_ABSOLUTE: return call("bh_cabs");
        case BH_COS: return call("bh_ccos");
        case BH_SIN: return call("bh_csin");
        case BH_TAN: return call("bh_ctan");
        case BH_COSH: return call("bh_ccosh");
        case BH_SINH: return call("bh_csinh");
        case BH_TANH: return call("bh_ctanh");
        case BH_EXP: return call("bh_cexp");
        case BH_LOG: return call("bh_clog");
        case BH_LOG10: return call("bh_clog10");
        case BH_SQRT: return call("bh_csqrt");
        case BH_SIGN: return call("bh_csign");
        case BH_CONJ: return call("bh_conj");
        case BH_REAL: return o + " = " + ops[1] + ".re;";
        case BH_IMAG: return o + " = " + ops[1] + ".im;";
        case BH_ISNAN: return o + " = isnan(" + ops[1] + ".re);";
        case BH_ISINF: return o + " = isinf(" + ops[1] + ".re);";
        case BH_ISFINITE: return o + " = isfinite(" + ops[1] + ".re);";
        case BH_IDENTITY:
        case BH_GATHER:
        case BH_SCATTER: return o + " = " + ops[1] + ";";
        case BH_COND_SCATTER: return "if (" + ops[2] + ") { " + o + " = " + ops[1] + "; }";
        case BH_ADD_ACCUMULATE: return o + " = " + ops[1] + " + " + ops[2] + ";";
        case BH_MULTIPLY_ACCUMULATE: return o + " = " + ops[1] + " * " + ops[2] + ";";
        case BH_ADD_REDUCE:
        case BH_MULTIPLY_REDUCE: return o + " = " + reduce_expr(op, o, ops[1]) + ";";
        default: break;
    }
    throw runtime_error(string("Instruction not supported for complex element types by the CUDA engine: ") +
                        bh_opcode_text(op));
}

// One statement computing `instr` given its operand expressions (ops[0] is the output lvalue).
string op_statement(const bh_instruction &instr, const vector<string> &ops) {
    const bh_opcode op = instr.opcode;
    const bh_type t0 = instr.operand_type(0);
    const bh_type t1 = instr.operand.size() > 1 ? instr.operand_type(1) : t0;
    for (size_t i = 0; i < instr.operand.size(); ++i)
        if (bh_type_is_complex(instr.operand_type(static_cast<int>(i)))) return complex_statement(instr, ops);
    const string &o = ops[0];
    auto un = [&](const char *f) { return o + " = " + fn(f, t1) + "(" + ops[1] + ");"; };
    auto bin = [&](const char *sym) { return o + " = " + ops[1] + " " + sym + " " + ops[2] + ";"; };
    if (bh_opcode_is_reduction(op)) return o + " = " + reduce_expr(op, o, ops[1]) + ";";
    switch (op) {
        case BH_ADD: return bin("+");
        case BH_SUBTRACT: return bin("-");
        case BH_MULTIPLY: return bin("*");
        case BH_DIVIDE:
            if (bh_type_is_signed_integer(t0)) {
                const string &a = ops[1], &b = ops[2];
                return o + " = ((" + a + " > 0) != (" + b + " > 0) && (" + a + " % " + b + ") != 0) ? (" + a +
                       " / " + b + " - 1) : (" + a + " / " + b + ");";
            }
            return bin("/");
        case BH_POWER:
            if (t0 == bh_type::BOOL) return o + " = !" + ops[2] + " || " + ops[1] + ";";
            if (bh_type_is_integer(t0))
                return o + " = bh_ipow<" + cuda_type(t0) + ">(" + ops[1] + ", " + ops[2] + ");";
            return o + " = " + fn("pow", t0) + "(" + ops[1] + ", " + ops[2] + ");";
        case BH_ABSOLUTE:
            if (t1 == bh_type::BOOL || bh_type_is_unsigned_integer(t1)) return o + " = " + ops[1] + ";";
            if (is_float(t1)) return un("fabs");
            if (t1 == bh_type::INT64) return o + " = llabs(" + ops[1] + ");";
            return o + " = abs((int)" + ops[1] + ");";
        case BH_GREATER: return bin(">");
        case BH_GREATER_EQUAL: return bin(">=");
        case BH_LESS: return bin("<");
        case BH_LESS_EQUAL: return bin("<=");
        case BH_EQUAL: return bin("==");
        case BH_NOT_EQUAL: return bin("!=");
        case BH_LOGICAL_AND: return bin("&&");
        case BH_LOGICAL_OR: return bin("||");
        case BH_LOGICAL_XOR: return o + " = !" + ops[1] + " != !" + ops[2] + ";";
        case BH_LOGICAL_NOT: return o + " = !" + ops[1] + ";";
        case BH_MAXIMUM: return o + " = " + ops[1] + " > " + ops[2] + " ? " + ops[1] + " : " + ops[2] + ";";
        case BH_MINIMUM: return o + " = " + ops[1] + " < " + ops[2] + " ? " + ops[1] + " : " + ops[2] + ";";
        case BH_BITWISE_AND: return bin("&");
        case BH_BITWISE_OR: return bin("|");
        case BH_BITWISE_XOR: return bin("^");
        case BH_INVERT:
            if (t0 == bh_type::BOOL) return o + " = !" + ops[1] + ";";
            return o + " = ~" + ops[1] + ";";
        case BH_LEFT_SHIFT: return bin("<<");
        case BH_RIGHT_SHIFT: return bin(">>");
        case BH_COS: return un("cos");
        case BH_SIN: return un("sin");
        case BH_TAN: return un("tan");
        case BH_COSH: return un("cosh");
        case BH_SINH: return un("sinh");
        case BH_TANH: return un("tanh");
        case BH_ARCSIN: return un("asin");
        case BH_ARCCOS: return un("acos");
        case BH_ARCTAN: return un("atan");
        case BH_ARCSINH: return un("asinh");
        case BH_ARCCOSH: return un("acosh");
        case BH_ARCTANH: return un("atanh");
        case BH_ARCTAN2: return o + " = " + fn("atan2", t1) + "(" + ops[1] + ", " + ops[2] + ");";
        case BH_EXP: return un("exp");
        case BH_EXP2: return un("exp2");
        case BH_EXPM1: return un("expm1");
        case BH_LOG: return un("log");
        case BH_LOG2: return un("log2");
        case BH_LOG10: return un("log10");
        case BH_LOG1P: return un("log1p");
        case BH_SQRT: return un("sqrt");
        case BH_CEIL: return un("ceil");
        case BH_TRUNC: return un("trunc");
        case BH_FLOOR: return un("floor");
        case BH_RINT: return un("rint");
        case BH_MOD:
            if (is_float(t0)) return o + " = " + fn("fmod", t0) + "(" + ops[1] + ", " + ops[2] + ");";
            return bin("%");
        case BH_REMAINDER: {
            const string &a = ops[1], &b = ops[2];
            if (is_float(t0)) return o + " = " + a + " - " + fn("floor", t0) + "(" + a + " / " + b + ") * " + b + ";";
            if (bh_type_is_unsigned_integer(t0)) return bin("%");
            return o + " = ((" + a + " > 0) == (" + b + " > 0) || (" + a + " % " + b + ") == 0) ? (" + a + " % " +
                   b + ") : (" + a + " % " + b + ") + " + b + ";";
        }
        case BH_ISNAN:
            return is_float(t1) ? o + " = isnan(" + ops[1] + ");" : o + " = false;";
        case BH_ISINF:
            return is_float(t1) ? o + " = isinf(" + ops[1] + ");" : o + " = false;";
        case BH_ISFINITE:
            return is_float(t1) ? o + " = isfinite(" + ops[1] + ");" : o + " = true;";
        case BH_IDENTITY: return o + " = " + ops[1] + ";";
        case BH_SIGN: return o + " = " + sign_expr(ops[1]) + ";";
        case BH_RANGE: return o + " = " + ops[1] + ";";
        case BH_RANDOM: return o + " = " + ops[1] + ";";
        case BH_GATHER: return o + " = " + ops[1] + ";";
        case BH_SCATTER: return o + " = " + ops[1] + ";";
        case BH_COND_SCATTER: return "if (" + ops[2] + ") { " + o + " = " + ops[1] + "; }";
        case BH_ADD_ACCUMULATE: return o + " = " + ops[1] + " + " + ops[2] + ";";
        case BH_MULTIPLY_ACCUMULATE: return o + " = " + ops[1] + " * " + ops[2] + ";";
        default: break;
    }
    throw runtime_error(string("Instruction not supported by the CUDA engine: ") + bh_opcode_text(op));
}

// Literal CUDA expression of a constant (used for identities folded into accumulator init).
string constant_literal(const bh_constant &c) {
    stringstream ss;
    ss.precision(17);
    switch (c.type) {
        case bh_type::BOOL: ss << (c.value.bool8 ? "true" : "false"); break;
        case bh_type::INT8: ss << "((signed char)" << static_cast<int>(c.value.int8) << ")"; break;
        case bh_type::INT16: ss << "((short)" << c.value.int16 << ")"; break;
        case bh_type::INT32: ss << "((int)" << c.value.int32 << ")"; break;
        case bh_type::INT64:
            // INT64_MIN+1 and friends: write through the unsigned bit pattern to avoid overflowing literals.
            ss << "((long long)" << static_cast<uint64_t>(c.value.int64) << "ULL)";
            break;
        case bh_type::UINT8: ss << "((unsigned char)" << static_cast<unsigned>(c.value.uint8) << "u)"; break;
        case bh_type::UINT16: ss << "((unsigned short)" << c.value.uint16 << "u)"; break;
        case bh_type::UINT32: ss << c.value.uint32 << "u"; break;
        case bh_type::UINT64: ss << c.value.uint64 << "ULL"; break;
        case bh_type::FLOAT32: {
            uint32_t bits;
            memcpy(&bits, &c.value.float32, 4);
            ss << "__int_as_float(" << static_cast<int32_t>(bits) << ")";
            break;
        }
        case bh_type::FLOAT64: {
            int64_t bits;
            memcpy(&bits, &c.value.float64, 8);
            ss << "__longlong_as_double(" << static_cast<uint64_t>(bits) << "LL)";
            break;
        }
        case bh_type::COMPLEX64: {
            uint32_t re, im;
            memcpy(&re, &c.value.complex64.real, 4);
            memcpy(&im, &c.value.complex64.imag, 4);
            ss << "bh_c64(__int_as_float(" << static_cast<int32_t>(re) << "), __int_as_float(" << static_cast<int32_t>(im)
               << "))";
            break;
        }
        case bh_type::COMPLEX128: {
            uint64_t re, im;
            memcpy(&re, &c.value.complex128.real, 8);
            memcpy(&im, &c.value.complex128.imag, 8);
            ss << "bh_c128(__longlong_as_double(" << re << "LL), __longlong_as_double(" << im << "LL))";
            break;
        }
        default: throw runtime_error("constant_literal(): unsupported constant type");
    }
    return ss.str();
}

// ------------------------------------------------------------------------------- view identity
// Views compared like the reference's IgnoreOneDim_less (base, start and the (shape, stride) of
// dimensions larger than one); used to find scalar-replaced reduction outputs.
struct ViewKey {
    const bh_base *base;
    int64_t start;
    vector<pair<int64_t, int64_t>> dims;
    explicit ViewKey(const bh_view &v) : base(v.base), start(v.start) {
        for (int64_t i = 0; i < v.ndim; ++i)
            if (v.shape[i] > 1) dims.emplace_back(v.shape[i], v.stride[i]);
    }
    bool operator<(const ViewKey &o) const { return tie(base, start, dims) < tie(o.base, o.start, o.dims); }
};

// ------------------------------------------------------------------------------- unit symbols
struct Symbols {
    vector<bh_base *> params;
    map<const bh_base *, int> param_id;
    map<const bh_base *, int> base_id; // every base (params and temporaries)
    set<const bh_base *> temps;
    set<const bh_base *> always_array;
    map<bh_view, int> view_id; // exact view -> offset slot
    vector<bh_view> views;
    // Views with equal strides share one set of stride parameters (a stride group), and their
    // index expressions share the strided part, so the compiler computes it once.
    map<vector<int64_t>, int> stride_group_id;
    vector<vector<int64_t>> stride_groups;
    vector<int> view_group; // per view
    map<const LoopB *, int> loop_id;
    vector<const LoopB *> loops;
    map<const bh_instruction *, int> const_id;
    vector<const bh_instruction *> consts;

    int base_index(const bh_base *b) {
        auto it = base_id.find(b);
        if (it != base_id.end()) return it->second;
        const int id = static_cast<int>(base_id.size());
        base_id[b] = id;
        return id;
    }
};

void collect_loops(const LoopB &l, Symbols &s) {
    if (l.rank >= 0 && !s.loop_id.count(&l)) {
        s.loop_id[&l] = static_cast<int>(s.loops.size());
        s.loops.push_back(&l);
    }
    for (const Block &b : l._block_list)
        if (!b.isInstr()) collect_loops(b.getLoop(), s);
}

// Build the symbols of a unit made of `items` (instruction and loop blocks, in order).
// `folded` instructions are identities turned into accumulator initialisation (no constant slot).
Symbols build_symbols(const vector<const Block *> &items, const set<const bh_instruction *> &folded) {
    Symbols s;
    vector<InstrPtr> instrs;
    set<bh_base *> temps, frees;
    for (const Block *b : items) {
        if (b->isInstr()) {
            instrs.push_back(b->getInstr());
        } else {
            jitk::all_instr(b->getLoop(), instrs);
            const auto t = b->getLoop().getAllTemps();
            temps.insert(t.begin(), t.end());
            const auto f = b->getLoop().getAllFrees();
            frees.insert(f.begin(), f.end());
            collect_loops(b->getLoop(), s);
        }
    }
    for (const InstrPtr &instr : instrs) {
        if (bh_opcode_is_accumulate(instr->opcode)) {
            s.always_array.insert(instr->operand[0].base);
        } else if (instr->opcode == BH_GATHER) {
            s.always_array.insert(instr->operand[1].base);
        } else if (instr->opcode == BH_SCATTER || instr->opcode == BH_COND_SCATTER) {
            s.always_array.insert(instr->operand[0].base);
        }
    }
    for (const bh_base *t : temps)
        if (!s.always_array.count(t)) s.temps.insert(t);
    for (const InstrPtr &instr : instrs) {
        for (const bh_view &v : instr->getViews()) {
            s.base_index(v.base);
            if (!s.temps.count(v.base) && !s.param_id.count(v.base)) {
                s.param_id[v.base] = static_cast<int>(s.params.size());
                s.params.push_back(v.base);
            }
            // Views of temporaries are registered too: BH_RANGE/BH_RANDOM use their index.
            if (!s.view_id.count(v)) {
                s.view_id[v] = static_cast<int>(s.views.size());
                s.views.push_back(v);
                vector<int64_t> key(v.stride.begin(), v.stride.begin() + v.ndim);
                auto g = s.stride_group_id.find(key);
                if (g == s.stride_group_id.end()) {
                    g = s.stride_group_id.emplace(key, static_cast<int>(s.stride_groups.size())).first;
                    s.stride_groups.push_back(key);
                }
                s.view_group.push_back(g->second);
            }
        }
        if (instr->has_constant() && !bh_opcode_is_sweep(instr->opcode) && !folded.count(instr.get())) {
            s.const_id[instr.get()] = static_cast<int>(s.consts.size());
            s.consts.push_back(instr.get());
        }
    }
    return s;
}

// ------------------------------------------------------------------------------------ emitter
struct Scope {
    const Scope *parent = nullptr;
    set<const bh_base *> tmps;
    map<ViewKey, string> repl; // scalar-replaced views
    bool is_tmp(const bh_base *b) const { return tmps.count(b) || (parent && parent->is_tmp(b)); }
    const string *replaced(const bh_view &v) const {
        auto it = repl.find(ViewKey(v));
        if (it != repl.end()) return &it->second;
        return parent ? parent->replaced(v) : nullptr;
    }
};

class Emitter {
public:
    Symbols &sym;
    ostream &out;
    const CodegenOptions &opt;
    // Views replaced by accumulators owned by the schedule (no write-back by the emitter).
    map<ViewKey, string> external_acc;

    Emitter(Symbols &s, ostream &o, const CodegenOptions &op) : sym(s), out(o), opt(op) {}

    void indent(int n) { out << string(static_cast<size_t>(n), ' '); }

    // Local temporaries of `loop` in symbol order (deterministic source text).
    vector<const bh_base *> sorted_temps(const LoopB &loop) {
        vector<const bh_base *> ret;
        for (const bh_base *b : loop.getLocalTemps())
            if (sym.base_id.count(b)) ret.push_back(b);
        sort(ret.begin(), ret.end(), [&](const bh_base *a, const bh_base *b) { return sym.base_id.at(a) < sym.base_id.at(b); });
        return ret;
    }

    // Element index of view `v`: (sum of loop index x group stride) + view offset. The strided
    // part is written identically for all views of a stride group.
    // Views whose address is split into a pointer computed once outside the innermost loop (the
    // schedule declares it) and that loop's term: view id -> pointer name. `hoist_axis` is the
    // index of that loop.
    map<int, string> hoisted;
    int hoist_axis = -1;

    // The term of loop index `axis` in the index of `v` ("0" for a broadcast axis).
    string axis_term(const bh_view &v, int axis) {
        const int vid = sym.view_id.at(v);
        const int gid = sym.view_group.at(static_cast<size_t>(vid));
        const vector<int64_t> &st = sym.stride_groups.at(static_cast<size_t>(gid));
        if (axis >= v.ndim) return "0";
        const int64_t stride = st.at(static_cast<size_t>(axis));
        if (stride == 0) return "0";
        if (stride == 1) return "i" + to_string(axis);
        return "i" + to_string(axis) + " * p.g" + to_string(gid) + "_s" + to_string(axis);
    }

    string index_expr(const bh_view &v, int hidden_axis = BH_MAXDIM, pair<int, int> axis_offset = {-1, 0},
                      int skip_axis = -1) {
        const int vid = sym.view_id.at(v);
        const int gid = sym.view_group.at(static_cast<size_t>(vid));
        if (v.is_scalar() || v.ndim == 0) return "(p.v" + to_string(vid) + "_o)";
        // Unit and zero strides are structural (part of the plan key), so they are written as
        // literals: no multiply for a contiguous axis, no term for a broadcast one.
        const vector<int64_t> &st = sym.stride_groups.at(static_cast<size_t>(gid));
        stringstream ss;
        ss << "((";
        bool any = false;
        for (int64_t i = 0; i < v.ndim; ++i) {
            int t = static_cast<int>(i);
            if (t >= hidden_axis) ++t;
            const int64_t stride = st.at(static_cast<size_t>(i));
            if (stride == 0 || t == skip_axis) continue;
            if (any) ss << " + ";
            any = true;
            if (axis_offset.first == t) {
                ss << "(i" << t << " == 0 ? 0 : i" << t << " + (" << axis_offset.second << "))";
            } else {
                ss << "i" << t;
            }
            if (stride != 1) ss << " * p.g" << gid << "_s" << i;
        }
        if (!any) ss << "0";
        ss << ") + p.v" << vid << "_o)";
        return ss.str();
    }

    string array_ref(const bh_view &v, int hidden_axis = BH_MAXDIM, pair<int, int> axis_offset = {-1, 0}) {
        if (!opt.bounds_check && hidden_axis == BH_MAXDIM && axis_offset.first < 0 && !hoisted.empty()) {
            auto it = hoisted.find(sym.view_id.at(v));
            if (it != hoisted.end()) return it->second + "[" + axis_term(v, hoist_axis) + "]";
        }
        const string idx = index_expr(v, hidden_axis, axis_offset);
        const int pid = sym.param_id.at(v.base);
        if (opt.bounds_check) {
            return "a" + to_string(pid) + "[bh_check(" + idx + ", p.nelem" + to_string(pid) + ", p.err)]";
        }
        return "a" + to_string(pid) + "[" + idx + "]";
    }

    string name(const bh_view &v, const Scope &s, int hidden_axis = BH_MAXDIM) {
        if (s.is_tmp(v.base)) return "t" + to_string(sym.base_index(v.base));
        auto ext = external_acc.find(ViewKey(v));
        if (ext != external_acc.end()) return ext->second;
        if (const string *r = s.replaced(v)) return *r;
        return array_ref(v, hidden_axis);
    }

    bool is_array(const bh_view &v, const Scope &s) {
        return !(s.is_tmp(v.base) || s.replaced(v) || external_acc.count(ViewKey(v)));
    }

    string const_ref(const bh_instruction &instr) {
        const string c = "p.c" + to_string(sym.const_id.at(&instr));
        if (instr.constant.type == bh_type::COMPLEX128) return "bh_c128(" + c + "_re, " + c + "_im)";
        return c;
    }

    // Operand o (1..3) of a fused multiply-add: a view, or the constant -- with two constants,
    // the multiplier (o = 2) is the real and the addend (o = 3) the imaginary part of the slot.
    string fma_operand(const bh_instruction &instr, size_t o, const Scope &s) {
        const bh_view &v = instr.operand[o];
        if (!v.isConstant()) return name(v, s);
        const string c = "p.c" + to_string(sym.const_id.at(&instr));
        if (instr.constant.type == bh_type::COMPLEX64) return c + (o == 2 ? ".re" : ".im");
        if (instr.constant.type == bh_type::COMPLEX128) return c + (o == 2 ? "_re" : "_im");
        return c;
    }

    void write_instr(const bh_instruction &instr, const Scope &s, int ind) {
        if (is_fma_opcode(instr.opcode)) {
            const string f = instr.operand[0].base->dtype() == bh_type::FLOAT32 ? "fmaf" : "fma";
            const string o = name(instr.operand[0], s), a = fma_operand(instr, 1, s), b = fma_operand(instr, 2, s),
                         c = fma_operand(instr, 3, s);
            indent(ind);
            if (instr.opcode == BH_X_FMA) out << o << " = " << f << "(" << a << ", " << b << ", " << c << ");\n";
            if (instr.opcode == BH_X_FMS) out << o << " = " << f << "(" << a << ", " << b << ", -(" << c << "));\n";
            if (instr.opcode == BH_X_FNMA) out << o << " = " << f << "(-(" << a << "), " << b << ", " << c << ");\n";
            return;
        }
        if (bh_opcode_is_system(instr.opcode) || instr.operand.empty()) return;
        vector<string> ops;
        if (instr.opcode == BH_RANGE) {
            ops.push_back(name(instr.operand[0], s));
            ops.push_back("(bh_u64)" + index_expr(instr.operand[0]));
        } else if (instr.opcode == BH_RANDOM) {
            ops.push_back(name(instr.operand[0], s));
            const int cid = sym.const_id.at(&instr);
            ops.push_back("bh_random123(p.c" + to_string(cid) + "_start, p.c" + to_string(cid) + "_key, (bh_u64)" +
                          index_expr(instr.operand[0]) + ")");
        } else if (instr.opcode == BH_GATHER) {
            ops.push_back(name(instr.operand[0], s));
            const bh_view &in = instr.operand[1];
            ops.push_back("a" + to_string(sym.param_id.at(in.base)) + "[p.v" + to_string(sym.view_id.at(in)) +
                          "_o + (bh_i64)" + name(instr.operand[2], s) + "]");
        } else if (instr.opcode == BH_SCATTER || instr.opcode == BH_COND_SCATTER) {
            const bh_view &outv = instr.operand[0];
            ops.push_back("a" + to_string(sym.param_id.at(outv.base)) + "[p.v" + to_string(sym.view_id.at(outv)) +
                          "_o + (bh_i64)" + name(instr.operand[2], s) + "]");
            ops.push_back(name(instr.operand[1], s));
            if (instr.opcode == BH_COND_SCATTER) ops.push_back(name(instr.operand[3], s));
        } else if (bh_opcode_is_accumulate(instr.opcode)) {
            ops.push_back(name(instr.operand[0], s));
            ops.push_back(array_ref(instr.operand[0], BH_MAXDIM, {instr.sweep_axis(), -1}));
            ops.push_back(name(instr.operand[1], s));
        } else if (bh_opcode_is_reduction(instr.opcode)) {
            // The constant operand of a reduction is its axis, not a value.
            const bh_view &v = instr.operand[0];
            if (instr.operand[1].ndim > 1 && is_array(v, s)) {
                ops.push_back(array_ref(v, instr.sweep_axis()));
            } else {
                ops.push_back(name(v, s));
            }
            ops.push_back(name(instr.operand[1], s));
        } else {
            for (size_t o = 0; o < instr.operand.size(); ++o) {
                const bh_view &v = instr.operand[o];
                if (v.isConstant()) {
                    ops.push_back(const_ref(instr));
                } else if (o == 0 && bh_opcode_is_reduction(instr.opcode) && instr.operand[1].ndim > 1 &&
                           is_array(v, s)) {
                    ops.push_back(array_ref(v, instr.sweep_axis()));
                } else {
                    ops.push_back(name(v, s));
                }
            }
        }
        indent(ind);
        out << op_statement(instr, ops) << "\n";
    }

    // Emit the body of `loop` (its temporaries, accumulators of swept children, instructions and
    // serial sub-loops). Loop heads of `loop` itself are written by the caller.
    void write_body(const LoopB &loop, Scope &scope, int ind) {
        // Temporaries local to this loop become registers.
        for (const bh_base *b : sorted_temps(loop)) {
            if (sym.temps.count(b) && !scope.is_tmp(b)) {
                scope.tmps.insert(b);
                indent(ind);
                out << cuda_type(b->dtype()) << " t" << sym.base_index(b) << ";\n";
            }
        }
        // Outputs of reductions over the innermost axis of a child loop live in registers here.
        vector<pair<const bh_view *, const bh_instruction *>> replaced_here;
        for (const Block &b1 : loop._block_list) {
            if (b1.isInstr()) continue;
            for (const InstrPtr &instr : jitk::all_local_instr(b1.getLoop())) {
                if (bh_opcode_is_reduction(instr->opcode) && jitk::sweeping_innermost_axis(instr)) {
                    const bh_view &v = instr->operand[0];
                    if (scope.is_tmp(v.base) || scope.replaced(v) || external_acc.count(ViewKey(v)) ||
                        sym.always_array.count(v.base))
                        continue;
                    const string nm = "s" + to_string(sym.base_index(v.base)) + "_" + to_string(replaced_here.size()) +
                                      "_r" + to_string(loop.rank + 1);
                    scope.repl[ViewKey(v)] = nm;
                    replaced_here.emplace_back(&v, instr.get());
                    indent(ind);
                    out << cuda_type(v.base->dtype()) << " " << nm << ";\n";
                }
            }
        }
        for (const Block &b : loop._block_list) {
            if (b.isInstr()) {
                write_instr(*b.getInstr(), scope, ind);
            } else {
                const LoopB &sub = b.getLoop();
                if (sub.isSystemOnly()) continue;
                indent(ind);
                out << "for (bh_i64 i" << sub.rank << " = 0; i" << sub.rank << " < p.n"
                    << sym.loop_id.at(&sub) << "; ++i" << sub.rank << ") {\n";
                Scope inner;
                inner.parent = &scope;
                write_body(sub, inner, ind + 4);
                indent(ind);
                out << "}\n";
            }
        }
        // Write the scalar-replaced reduction outputs back (temporaries stay registers).
        for (const auto &rp : replaced_here) {
            const bh_view &v = *rp.first;
            if (scope.is_tmp(v.base)) continue;
            indent(ind);
            out << array_ref(v, rp.second->sweep_axis()) << " = " << scope.repl.at(ViewKey(v)) << ";\n";
            scope.repl.erase(ViewKey(v));
        }
    }
};

// ------------------------------------------------------------------------------ param struct
struct ParamLayout {
    vector<ParamField> fields;
    stringstream decl; // members of `struct P`
    void add(const ParamField &f, const string &ctype, const string &name) {
        fields.push_back(f);
        decl << "    alignas(8) " << ctype << " " << name << ";\n";
    }
    // A 128-byte, 64-byte aligned tensor map: 16 slots. Tensor maps come first in P, so no
    // padding precedes them.
    void add_tmap(ParamField f, const string &name) {
        for (int k = 0; k < 16; ++k) {
            f.part = k;
            fields.push_back(f);
        }
        decl << "    bh_tmap " << name << ";\n";
    }
    // Round the struct up to a multiple of 64 bytes (its alignment with tensor maps), so that its
    // size is exactly 8 bytes per field.
    void pad64() {
        int k = 0;
        while (fields.size() % 8 != 0) add(work_pad(), "bh_i64", "pad" + to_string(k++));
    }
    static ParamField work_pad() {
        ParamField f{ParamField::I64};
        return f;
    }
};

void add_common_fields(Symbols &sym, ParamLayout &pl, const CodegenOptions &opt) {
    for (size_t i = 0; i < sym.params.size(); ++i) {
        ParamField f{ParamField::PTR};
        f.base = sym.params[i];
        pl.add(f, cuda_type(sym.params[i]->dtype()) + "* __restrict__", "a" + to_string(i));
    }
    for (size_t i = 0; i < sym.views.size(); ++i) {
        ParamField f{ParamField::I64};
        f.i64 = sym.views[i].start;
        pl.add(f, "bh_i64", "v" + to_string(i) + "_o");
    }
    for (size_t g = 0; g < sym.stride_groups.size(); ++g) {
        for (size_t d = 0; d < sym.stride_groups[g].size(); ++d) {
            ParamField f{ParamField::I64};
            f.i64 = sym.stride_groups[g][d];
            pl.add(f, "bh_i64", "g" + to_string(g) + "_s" + to_string(d));
        }
    }
    for (size_t i = 0; i < sym.loops.size(); ++i) {
        ParamField f{ParamField::I64};
        f.i64 = sym.loops[i]->size;
        pl.add(f, "bh_i64", "n" + to_string(i));
    }
    for (size_t i = 0; i < sym.consts.size(); ++i) {
        const bh_instruction *instr = sym.consts[i];
        if (instr->constant.type == bh_type::R123) {
            ParamField f{ParamField::R123_START};
            f.c = instr->constant;
            f.origin = instr->origin_id;
            pl.add(f, "bh_u64", "c" + to_string(i) + "_start");
            f.kind = ParamField::R123_KEY;
            pl.add(f, "bh_u64", "c" + to_string(i) + "_key");
        } else if (instr->constant.type == bh_type::COMPLEX128) {
            // 16 bytes: two 8-byte parameter slots, the real and the imaginary part
            ParamField f{ParamField::CONST};
            f.c = instr->constant;
            f.origin = instr->origin_id;
            pl.add(f, "double", "c" + to_string(i) + "_re");
            f.part = 1;
            pl.add(f, "double", "c" + to_string(i) + "_im");
        } else {
            ParamField f{ParamField::CONST};
            f.c = instr->constant;
            f.origin = instr->origin_id;
            pl.add(f, cuda_type(instr->constant.type), "c" + to_string(i));
        }
    }
    if (opt.bounds_check) {
        for (size_t i = 0; i < sym.params.size(); ++i) {
            ParamField f{ParamField::I64};
            f.i64 = sym.params[i]->nelem();
            pl.add(f, "bh_i64", "nelem" + to_string(i));
        }
        ParamField f{ParamField::SCRATCH};
        f.i64 = -1; // the engine's error record
        pl.add(f, "unsigned long long*", "err");
    }
}

string bounds_check_helper() {
    return R"CUDA(
__device__ __forceinline__ bh_i64 bh_check(bh_i64 idx, bh_i64 n, unsigned long long *err) {
    if (idx < 0 || idx >= n) { atomicCAS(err, 0ULL, (unsigned long long)idx | 0x8000000000000000ULL); return 0; }
    return idx;
}
)CUDA";
}

uint64_t fnv1a(const string &s) {
    uint64_t h = 1469598103934665603ULL;
    for (unsigned char c : s) {
        h ^= c;
        h *= 1099511628211ULL;
    }
    return h;
}

// The wrappers of every unit: bh_main (what one CTA of a plain launch does; the stencil staging
// replaces its loop) and the two kernels. The kernels' text (kKernels) is the same for every unit.
const char *kKernels = R"CUDA(
extern "C" __global__ void __launch_bounds__(256) __KERNEL_NAME__(const __grid_constant__ P p) {
    bh_grid_dependency();
    bh_main(p);
}
extern "C" __global__ void __launch_bounds__(256) __KERNEL_NAME___batch(const P* __restrict__ items,
        const bh_i64* __restrict__ prefix, int nitems, bh_i64 total) {
    // Each CTA takes a contiguous range of the work items of all items, so consecutive work items
    // of a CTA belong to the same item except at item boundaries. The parameters of the current
    // item live in shared memory and are looked up and reloaded only at those boundaries.
    bh_grid_dependency();
    __shared__ P sp;
    int have = -1;
    bh_i64 have_lo = 0, have_hi = 0;
    const bh_i64 g_lo = (bh_i64)blockIdx.x * total / gridDim.x;
    const bh_i64 g_hi = ((bh_i64)blockIdx.x + 1) * total / gridDim.x;
    for (bh_i64 g = g_lo; g < g_hi; ++g) {
        if (g < have_lo || g >= have_hi) {
            int lo = 0, hi = nitems - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (prefix[mid] <= g) lo = mid; else hi = mid - 1;
            }
            __syncthreads();
            for (int k = threadIdx.x; k < (int)(sizeof(P) / 8); k += blockDim.x)
                ((unsigned long long*)&sp)[k] = ((const unsigned long long*)(items + lo))[k];
            __syncthreads();
            have = lo;
            have_lo = prefix[lo];
            have_hi = prefix[lo + 1];
        }
        bh_batch_work(sp, g - have_lo);
    }
    (void)have;
}
)CUDA";
// What one CTA of a plain launch does, and the device code of one work item of a grouped launch
// (the same as a plain launch's unless a unit defines its own).
const char *kMainWrapper = R"CUDA(
__device__ __forceinline__ void bh_main(const P &p) {
    for (bh_i64 w = blockIdx.x; w < p.work; w += gridDim.x) bh_work(p, w);
}
)CUDA";
const char *kBatchWork = R"CUDA(
__device__ __forceinline__ void bh_batch_work(const P &p, bh_i64 w) { bh_work(p, w); }
)CUDA";
const string kWrappers = string(kMainWrapper) + kBatchWork + kKernels;

void finish_source(LaunchUnit &u, const string &params_decl, const string &body, const CodegenOptions &opt) {
    u.params_decl = params_decl;
    u.body_core = body;
    const string kk = kKernels;
    if (u.body_core.size() >= kk.size() && u.body_core.compare(u.body_core.size() - kk.size(), kk.size(), kk) == 0)
        u.body_core.resize(u.body_core.size() - kk.size());
    else
        u.body_core.clear();  // wrappers of its own: not combinable with another unit
    stringstream src;
    src << kPrelude;
    auto uses = [&](const char *name) { return params_decl.find(name) != string::npos || body.find(name) != string::npos; };
    if (uses("bh_c64") || uses("bh_c128")) src << kComplexPrelude;
    if (uses("bh_tmap") || uses("bh_mbar")) src << kTmaPrelude;
    if (opt.bounds_check) src << bounds_check_helper();
    src << "struct P {\n" << params_decl << "};\n";
    src << body;
    const string without_name = src.str();
    stringstream nm;
    nm << "bh_" << sched_name(u.sched) << "_" << hex << fnv1a(without_name);
    u.name = nm.str();
    string s = without_name;
    const string placeholder = "__KERNEL_NAME__";
    for (size_t pos = s.find(placeholder); pos != string::npos; pos = s.find(placeholder))
        s.replace(pos, placeholder.size(), u.name);
    u.source = s;
}

// Unpack the pointer fields into local restrict pointers.
string pointer_locals(const Symbols &sym) {
    stringstream ss;
    for (size_t i = 0; i < sym.params.size(); ++i)
        ss << "    " << cuda_type(sym.params[i]->dtype()) << "* __restrict__ a" << i << " = p.a" << i << ";\n";
    return ss.str();
}

// Algorithmic bytes of a unit: for every non-temporary base, the bytes of its distinct views that
// are read plus those that are written, each capped at the base's size (overlapping views such as
// the shifted views of a stencil count once).
int64_t unit_bytes(const Symbols &sym, const vector<InstrPtr> &instrs) {
    map<const bh_base *, set<bh_view>> reads, writes;
    for (const InstrPtr &instr : instrs) {
        if (bh_opcode_is_system(instr->opcode)) continue;
        for (size_t o = 0; o < instr->operand.size(); ++o) {
            const bh_view &v = instr->operand[o];
            if (v.isConstant() || sym.temps.count(v.base)) continue;
            const bool write = o == 0 && instr->opcode != BH_GATHER;
            (write ? writes : reads)[v.base].insert(v);
            if (instr->opcode == BH_SCATTER || instr->opcode == BH_COND_SCATTER || bh_opcode_is_accumulate(instr->opcode))
                if (o == 0) reads[v.base].insert(v);
        }
    }
    int64_t total = 0;
    for (auto *m : {&reads, &writes}) {
        for (const auto &kv : *m) {
            int64_t b = 0;
            for (const bh_view &v : kv.second) b += v.shape.prod() * bh_type_size(v.base->dtype());
            total += min<int64_t>(b, kv.first->nbytes());
        }
    }
    return total;
}

int64_t unit_bytes(const Symbols &sym, const vector<const Block *> &items) {
    vector<InstrPtr> instrs;
    for (const Block *b : items) {
        if (b->isInstr()) {
            instrs.push_back(b->getInstr());
        } else {
            jitk::all_instr(b->getLoop(), instrs);
        }
    }
    return unit_bytes(sym, instrs);
}

// ------------------------------------------------------------------------------------ schedules
// Every schedule is written as `bh_work(p, w)` for work items w in [0, p.work), plus two kernels:
// the plain launch (grid-stride over the unit's own work items) and the batched launch, which runs
// the work items of many units of the same kernel in one persistent grid (item lookup by binary
// search over the prefix sums of their work counts). Both call the same device code on the same
// work items, so batched results equal plain results bit for bit.


ParamField work_field(int64_t work) {
    ParamField f{ParamField::I64};
    f.i64 = work;
    return f;
}

LaunchUnit lower_serial(const vector<const Block *> &items, const CodegenOptions &opt) {
    LaunchUnit u;
    u.sched = Sched::SERIAL;
    // The kernel is a loop of rank -1: wrap the items in a pseudo loop so temporaries and
    // scalar replacement are handled uniformly.
    LoopB pseudo{-1, 1};
    for (const Block *b : items) pseudo._block_list.push_back(*b);
    pseudo.metadataUpdate();
    vector<const Block *> pitems;
    for (const Block &b : pseudo._block_list) pitems.push_back(&b);
    Symbols sym = build_symbols(pitems, {});
    ParamLayout pl;
    add_common_fields(sym, pl, opt);
    pl.add(work_field(1), "bh_i64", "work");
    stringstream body;
    Emitter em(sym, body, opt);
    body << "__device__ __forceinline__ void bh_work(const P &p, bh_i64 w) {\n";
    body << "    if (threadIdx.x != 0) return;\n";
    body << pointer_locals(sym);
    Scope scope;
    em.write_body(pseudo, scope, 4);
    body << "}\n" << kWrappers;
    u.fields = pl.fields;
    u.algorithmic_bytes = unit_bytes(sym, pitems);
    finish_source(u, pl.decl.str(), body.str(), opt);
    return u;
}

// Temporaries declared on the threaded chain above the innermost threaded loop.
void declare_chain_temps(Emitter &em, Symbols &sym, Scope &scope, const vector<const LoopB *> &chain, unsigned upto,
                         ostream &body, int ind) {
    for (unsigned r = 0; r < upto; ++r) {
        for (const bh_base *b : em.sorted_temps(*chain[r])) {
            if (sym.temps.count(b) && !scope.is_tmp(b)) {
                scope.tmps.insert(b);
                body << string(static_cast<size_t>(ind), ' ') << cuda_type(b->dtype()) << " t" << sym.base_index(b)
                     << ";\n";
            }
        }
    }
}

// A heavy element body -- many instructions, or float64 divisions and transcendentals -- is
// bound by the arithmetic pipes rather than by memory latency.
bool heavy_body(const LoopB &L) {
    int n = 0, heavy = 0;
    for (const InstrPtr &i : jitk::all_instr(L)) {
        ++n;
        const bh_opcode op = i->opcode;
        const bool f64 = !i->operand.empty() && !i->operand[0].isConstant() &&
                         i->operand[0].base->dtype() == bh_type::FLOAT64;
        if (f64 && (op == BH_DIVIDE || op == BH_EXP || op == BH_LOG || op == BH_SQRT || op == BH_POWER ||
                    op == BH_SIN || op == BH_COS || op == BH_TANH))
            ++heavy;
    }
    return n > 24 || heavy > 0;
}

// FLAT: `loop` has P >= 1 leading parallel ranks.
// Views that an innermost element loop only reads: the view's base is an array (not a
// temporary) that no instruction of the kernel writes, and the view is read by a plain
// elementwise or reduction instruction. Their V elements per thread can be loaded into registers
// before the computation, so that all V loads are in flight together (branches in the element
// code, e.g. IEEE sqrt's special-case path, would otherwise keep the compiler from hoisting them).
vector<bh_view> preloadable_views(const LoopB &inner, const LoopB &kernel, const Symbols &sym) {
    set<const bh_base *> written;
    for (const InstrPtr &i : jitk::all_instr(kernel))
        if (!i->operand.empty() && !i->operand[0].isConstant()) written.insert(i->operand[0].base);
    vector<bh_view> ret;
    set<ViewKey> seen;
    for (const Block &b : inner._block_list) {
        if (!b.isInstr()) return {};  // not an innermost loop
        const bh_instruction &in = *b.getInstr();
        const bh_opcode op = in.opcode;
        if (bh_opcode_is_system(op) || op == BH_GATHER || op == BH_SCATTER || op == BH_COND_SCATTER ||
            op == BH_RANGE || op == BH_RANDOM || bh_opcode_is_accumulate(op))
            continue;
        for (size_t o = 1; o < in.operand.size(); ++o) {
            const bh_view &v = in.operand[o];
            if (v.isConstant() || sym.temps.count(v.base) || written.count(v.base)) continue;
            if (bh_opcode_is_sweep(op) && o > 1) continue;
            if (seen.insert(ViewKey(v)).second) ret.push_back(v);
        }
    }
    return ret;
}

// Declare, for every array view read or written in the innermost loop `inner` (index i<axis>,
// all higher loop indices defined), a pointer to the view's element at i<axis> = 0, and register
// them with the emitter so that references inside the loop index the pointer by the loop term
// only. Nothing is hoisted under bounds checking.
void hoist_views(Emitter &em, const LoopB &inner, int axis, ostream &out, int ind) {
    if (em.opt.bounds_check) return;
    const string sp(static_cast<size_t>(ind), ' ');
    for (const Block &b : inner._block_list) {
        if (!b.isInstr()) return;
    }
    for (const InstrPtr &ip : jitk::all_instr(inner)) {
        const bh_opcode op = ip->opcode;
        if (bh_opcode_is_system(op) || op == BH_GATHER || op == BH_SCATTER || op == BH_COND_SCATTER) continue;
        for (size_t o = 0; o < ip->operand.size(); ++o) {
            const bh_view &v = ip->operand[o];
            if (v.isConstant() || em.sym.temps.count(v.base) || v.ndim != axis + 1) continue;
            if (o == 0 && bh_opcode_is_sweep(op)) continue;  // an accumulator, not an array
            const int vid = em.sym.view_id.at(v);
            if (em.hoisted.count(vid)) continue;
            const string nm = "hp" + to_string(em.hoisted.size());
            out << sp << cuda_type(v.base->dtype()) << "* __restrict__ " << nm << " = a" << em.sym.param_id.at(v.base)
                << " + " << em.index_expr(v, BH_MAXDIM, {-1, 0}, axis) << ";\n";
            em.hoisted[vid] = nm;
        }
    }
    em.hoist_axis = axis;
}

// Emit the register arrays and the load loop of `views` for V elements per thread; element j has
// index `idx_init(j)` (a statement defining the innermost loop index). With `guard` the loads
// stop at the loop bound. Registers the replacements in `scope`.
void emit_preload(Emitter &em, const vector<bh_view> &views, int V, const string &index_decl, const string &guard,
                  Scope &scope, ostream &out, int ind) {
    if (views.empty()) return;
    const string sp(static_cast<size_t>(ind), ' ');
    for (size_t k = 0; k < views.size(); ++k)
        out << sp << cuda_type(views[k].base->dtype()) << " pl" << k << "[" << V << "];\n";
    out << sp << "#pragma unroll\n";
    out << sp << "for (int j = 0; j < " << V << "; ++j) {\n";
    out << sp << "    " << index_decl << "\n";
    if (!guard.empty()) out << sp << "    if (" << guard << ") break;\n";
    for (size_t k = 0; k < views.size(); ++k)
        out << sp << "    pl" << k << "[j] = " << em.array_ref(views[k]) << ";\n";
    out << sp << "}\n";
    for (size_t k = 0; k < views.size(); ++k) scope.repl[ViewKey(views[k])] = "pl" + to_string(k) + "[j]";
}

// 128-bit access for FLAT: thread t of a work item handles the 4 consecutive elements
// cbase .. cbase + 3 (cbase = chunk * 1024 + 4t) of the innermost parallel rank, so a view with
// unit stride along it is one 16-byte (or 4 x element size) word per thread. Read-only such views
// are loaded, and arrays written by the element code stored, as whole words when every such view's
// first element is aligned to the word (checked per work item); otherwise, and for views with other
// strides, element by element. The written values stay in registers until the words are stored,
// and later reads of them in the element code use the registers. Every element is computed by the
// same statements either way, so the results do not depend on the path.
// Views that can be moved as words: unit stride along the innermost rank `axis`, an array (not a
// temporary) of any element type.
bool unit_stride_view(const bh_view &v, int axis, const Symbols &sym) {
    if (v.isConstant() || sym.temps.count(v.base) || v.ndim != axis + 1) return false;
    return v.stride[axis] == 1;
}

// Loads or stores of `bytes` bytes at `addr` (a register array `reg`) as the widest aligned words.
string word_copy(const string &dst, const string &src, int bytes) {
    stringstream ss;
    if (bytes >= 16) {
        for (int k = 0; k < bytes / 16; ++k)
            ss << "((uint4 *)(" << dst << "))[" << k << "] = ((const uint4 *)(" << src << "))[" << k << "]; ";
    } else if (bytes == 8) {
        ss << "*(uint2 *)(" << dst << ") = *(const uint2 *)(" << src << "); ";
    } else {
        ss << "*(unsigned *)(" << dst << ") = *(const unsigned *)(" << src << "); ";
    }
    return ss.str();
}

void emit_flat_vector(Symbols &sym, ostream &body, const CodegenOptions &opt, const LoopB &inner,
                      const vector<const LoopB *> &chain, unsigned P, const vector<bh_view> &pre, int64_t per,
                      const string &n_inner, const string &iv) {
    const int axis = static_cast<int>(P) - 1;
    // Written views that can be stored as words: outputs of elementwise instructions of `inner`,
    // unit stride, their base written and read in the kernel through this one view only.
    map<const bh_base *, set<ViewKey>> touched;
    for (const InstrPtr &i : jitk::all_instr(inner))
        for (const bh_view &v : i->operand)
            if (!v.isConstant()) touched[v.base].insert(ViewKey(v));
    vector<bh_view> outs;
    set<ViewKey> seen_out;
    for (const InstrPtr &i : jitk::all_instr(inner)) {
        const bh_opcode op = i->opcode;
        if (bh_opcode_is_system(op) || bh_opcode_is_sweep(op) || op == BH_GATHER || op == BH_SCATTER ||
            op == BH_COND_SCATTER || i->operand.empty())
            continue;
        const bh_view &v = i->operand[0];
        if (!unit_stride_view(v, axis, sym) || sym.always_array.count(v.base) || touched[v.base].size() != 1) continue;
        if (seen_out.insert(ViewKey(v)).second) outs.push_back(v);
    }
    vector<bool> vec_pre(pre.size());
    for (size_t k = 0; k < pre.size(); ++k) vec_pre[k] = unit_stride_view(pre[k], axis, sym);
    Emitter em(sym, body, opt);
    body << "    const bh_i64 cbase = chunk * " << per << " + threadIdx.x * 4;\n";
    body << "    if ((chunk + 1) * " << per << " <= " << n_inner << ") {\n";
    // Word alignment of every word-moved view at element cbase.
    body << "        bool vec = true;\n";
    body << "        {\n";
    body << "            const bh_i64 " << iv << " = cbase;\n";
    auto align_check = [&](const bh_view &v) {
        const int bytes = min(16, 4 * static_cast<int>(bh_type_size(v.base->dtype())));
        body << "            vec = vec && (((unsigned long long)&" << em.array_ref(v) << ") & " << bytes - 1 << "ull) == 0;\n";
    };
    for (size_t k = 0; k < pre.size(); ++k)
        if (vec_pre[k]) align_check(pre[k]);
    for (const bh_view &v : outs) align_check(v);
    body << "        }\n";
    Scope scope;
    for (size_t k = 0; k < pre.size(); ++k) {
        const string T = cuda_type(pre[k].base->dtype());
        body << "        " << T << " pl" << k << "[4];\n";
        const int bytes = 4 * static_cast<int>(bh_type_size(pre[k].base->dtype()));
        if (vec_pre[k]) {
            body << "        if (vec) {\n";
            body << "            const bh_i64 " << iv << " = cbase;\n";
            body << "            " << word_copy("pl" + to_string(k), "&" + em.array_ref(pre[k]), bytes) << "\n";
            body << "        } else {\n";
        } else {
            body << "        {\n";
        }
        body << "#pragma unroll\n";
        body << "            for (int j = 0; j < 4; ++j) {\n";
        body << "                const bh_i64 " << iv << " = cbase + j;\n";
        body << "                pl" << k << "[j] = " << em.array_ref(pre[k]) << ";\n";
        body << "            }\n";
        body << "        }\n";
        scope.repl[ViewKey(pre[k])] = "pl" + to_string(k) + "[j]";
    }
    for (size_t k = 0; k < outs.size(); ++k) {
        body << "        " << cuda_type(outs[k].base->dtype()) << " so" << k << "[4];\n";
        scope.repl[ViewKey(outs[k])] = "so" + to_string(k) + "[j]";
    }
    body << "#pragma unroll\n";
    body << "        for (int j = 0; j < 4; ++j) {\n";
    body << "            const bh_i64 " << iv << " = cbase + j;\n";
    {
        Emitter eb(sym, body, opt);
        declare_chain_temps(eb, sym, scope, chain, P - 1, body, 12);
        eb.write_body(inner, scope, 12);
    }
    body << "        }\n";
    for (size_t k = 0; k < outs.size(); ++k) {
        const int bytes = 4 * static_cast<int>(bh_type_size(outs[k].base->dtype()));
        body << "        if (vec) {\n";
        body << "            const bh_i64 " << iv << " = cbase;\n";
        body << "            " << word_copy("&" + em.array_ref(outs[k]), "so" + to_string(k), bytes) << "\n";
        body << "        } else {\n";
        body << "#pragma unroll\n";
        body << "            for (int j = 0; j < 4; ++j) {\n";
        body << "                const bh_i64 " << iv << " = cbase + j;\n";
        body << "                " << em.array_ref(outs[k]) << " = so" << k << "[j];\n";
        body << "            }\n";
        body << "        }\n";
    }
    body << "    } else {\n";
    {
        Scope s1;
        Emitter eb(sym, body, opt);
        body << "        for (int j = 0; j < 4; ++j) {\n";
        body << "            const bh_i64 " << iv << " = cbase + j;\n";
        body << "            if (" << iv << " >= " << n_inner << ") break;\n";
        declare_chain_temps(eb, sym, s1, chain, P - 1, body, 12);
        eb.write_body(inner, s1, 12);
        body << "        }\n";
    }
    body << "    }\n";
}

// Elements of a map small enough to run in another kernel's tail: a few values computed from a
// reduction's result, such as a mean. (Maps of up to 4096 elements there made small flushes of the
// learned-fuser workload slower: one CTA after the producer's last one is a serial step.)
constexpr int64_t kFlatTailElements = 32;

LaunchUnit lower_flat(const LoopB &loop, unsigned P, const CodegenOptions &opt) {
    LaunchUnit u;
    u.sched = Sched::FLAT;
    const Block holder(loop);
    Symbols sym = build_symbols({&holder}, {});
    const LoopB &L = holder.getLoop();
    const vector<const LoopB *> chain = jitk::get_first_loop_blocks(L);
    const LoopB &inner = *chain[P - 1];
    u.V = inner.isInnermost() ? opt.flat_v : 1;
    int64_t rows = 1;
    for (unsigned r = 0; r + 1 < P; ++r) rows *= chain[r]->size;
    u.rows = rows;
    u.cols = inner.size;
    const int64_t per = static_cast<int64_t>(kThreads) * u.V;
    const int64_t chunks = (u.cols + per - 1) / per;
    ParamLayout pl;
    add_common_fields(sym, pl, opt);
    pl.add(work_field(chunks), "bh_i64", "chunks");
    pl.add(work_field(rows * chunks), "bh_i64", "work");

    stringstream body;
    Emitter em(sym, body, opt);
    body << "__device__ __forceinline__ void bh_work(const P &p, bh_i64 w) {\n";
    body << pointer_locals(sym);
    body << "    const bh_i64 row = w / p.chunks;\n";
    body << "    const bh_i64 chunk = w - row * p.chunks;\n";
    body << "    bh_i64 rem = row;\n";
    for (int r = static_cast<int>(P) - 2; r >= 0; --r) {
        const int lid = sym.loop_id.at(chain[r]);
        if (r == 0) {
            body << "    const bh_i64 i0 = rem;\n";
        } else {
            body << "    const bh_i64 i" << r << " = rem % p.n" << lid << "; rem /= p.n" << lid << ";\n";
        }
    }
    body << "    (void)rem;\n";
    const vector<bh_view> pre =
        u.V > 1 && !(heavy_body(inner) && !opt.preload_heavy) ? preloadable_views(inner, L, sym) : vector<bh_view>{};
    const string n_inner = "p.n" + to_string(sym.loop_id.at(&inner));
    const string iv = "i" + to_string(P - 1);
    // A tiny map (at most kFlatTailElements elements) can also run in the tail of the kernel
    // before it, by the CTA that finishes that kernel last (fuse_tails): one CTA runs every work
    // item in turn. Elementwise results do not depend on which thread computes them. (bh_tail is
    // in every map's source, so that maps of every size share one compiled kernel.)
    const string tail_fn = opt.bounds_check ? ""
                                            : "__device__ void bh_tail(const P &p) {\n"
                                              "    for (bh_i64 w = 0; w < p.work; ++w) bh_work(p, w);\n"
                                              "}\n";
    u.tail_capable = !opt.bounds_check && rows * u.cols <= kFlatTailElements;
    if (u.V == 4 && opt.vector_access && !opt.bounds_check) {
        emit_flat_vector(sym, body, opt, inner, chain, P, pre, per, n_inner, iv);
        body << "}\n" << tail_fn << kWrappers;
        u.fields = pl.fields;
        u.algorithmic_bytes = unit_bytes(sym, vector<const Block *>{&holder});
        u.elements = rows * u.cols;
        finish_source(u, pl.decl.str(), body.str(), opt);
        return u;
    }
    body << "    const bh_i64 cbase = chunk * " << per << " + threadIdx.x;\n";
    // The element body is written once and used twice: full chunks run without bounds checks (so
    // the compiler can issue every load of the unrolled loop early), the last chunk with them.
    const string idx_decl = "const bh_i64 i" + to_string(P - 1) + " = cbase + j * " + to_string(kThreads) + ";";
    for (int path = 0; path < 2; ++path) {
        // path 0: full chunks without bounds checks; path 1: the last chunk, with them.
        const string guard = path == 0 ? "" : "i" + to_string(P - 1) + " >= " + n_inner;
        body << (path == 0 ? "    if ((chunk + 1) * " + to_string(per) + " <= " + n_inner + ") {\n" : "    } else {\n");
        Scope scope;
        Emitter eb(sym, body, opt);
        emit_preload(eb, pre, u.V, idx_decl, guard, scope, body, 8);
        if (path == 0) body << "#pragma unroll\n";
        body << "        for (int j = 0; j < " << u.V << "; ++j) {\n";
        body << "            " << idx_decl << "\n";
        if (path == 1) body << "            if (" << guard << ") break;\n";
        declare_chain_temps(eb, sym, scope, chain, P - 1, body, 12);
        eb.write_body(inner, scope, 12);
        body << "        }\n";
    }
    body << "    }\n}\n" << tail_fn << kWrappers;
    u.fields = pl.fields;
    u.algorithmic_bytes = unit_bytes(sym, vector<const Block *>{&holder});
    u.elements = rows * u.cols;
    finish_source(u, pl.decl.str(), body.str(), opt);
    return u;
}

// ------------------------------------------------------------------------------------- TILE2D
// A 2-D map (loop ranks 0 and 1 parallel, rank 1 innermost) that reads arrays through transposed
// views: stride 1 along rank 0 and a positive stride (the array's row length) along rank 1. The
// plain FLAT schedule walks rank 1 across a warp, so each warp load of such a view touches 32
// rows. Here a work item is a tile of TR rows x 64 columns of the index space, TR = 128 bytes /
// element size; thread t handles column t % 64 and rows (t / 64) * TR/4 ... + TR/4 - 1, so each
// output row of the tile is written by consecutive threads. A transposed view's part of a tile is
// a TR x 64 box of its base array (64 rows of 128 contiguous bytes), brought into a 4-stage
// shared-memory ring by one TMA copy per tile, up to 4 tiles ahead, with the 128-byte swizzle; a
// thread reads its TR/4 values as two 16-byte words (distinct banks across every 8 threads).
constexpr int kTileCols = 64;
constexpr int kTileStages = 4;
constexpr int kTileBoxBytes = kTileCols * 128;

// The views of `inner` that TILE2D stages: first the transposed ones -- read-only (their base is
// not written by the kernel), 2-D, stride 1 along rank 0 and > 1 along rank 1 -- at most two; then
// read-only row-wise ones (stride 1 along rank 1, > 1 along rank 0), up to three views in all. All
// of 4- or 8-byte elements of one size. `transposed[k]` tells the kinds apart. Empty when the loop
// has no transposed view or does not qualify.
vector<bh_view> tile2d_views(const LoopB &L, const LoopB &inner, const Symbols &sym, const CodegenOptions &opt,
                             vector<bool> &transposed) {
    transposed.clear();
    if (!opt.tile2d || opt.bounds_check || !inner.isInnermost() || !L._sweeps.empty() || !inner._sweeps.empty()) return {};
    if (L.size < 32 || inner.size < kTileCols) return {};
    set<const bh_base *> written;
    for (const InstrPtr &i : jitk::all_instr(L)) {
        if (bh_opcode_is_sweep(i->opcode)) return {};
        if (!i->operand.empty() && !i->operand[0].isConstant()) written.insert(i->operand[0].base);
    }
    auto usable = [&](const bh_view &v) {
        const int es = bh_type_size(v.base->dtype());
        return v.ndim == 2 && !written.count(v.base) && !bh_type_is_complex(v.base->dtype()) && (es == 4 || es == 8) &&
               v.base->dtype() != bh_type::R123;
    };
    const vector<bh_view> cand = preloadable_views(inner, L, sym);
    vector<bh_view> ret;
    set<ViewKey> seen;
    int esize = 0;
    for (const bh_view &v : cand) {
        if (!usable(v) || v.stride[0] != 1 || v.stride[1] <= 1) continue;
        const int es = bh_type_size(v.base->dtype());
        if (esize != 0 && es != esize) return {};
        esize = es;
        if (seen.insert(ViewKey(v)).second) {
            ret.push_back(v);
            transposed.push_back(true);
        }
    }
    if (ret.empty() || ret.size() > 2) {
        transposed.clear();
        return {};
    }
    for (const bh_view &v : cand) {
        if (ret.size() >= 3) break;
        if (!usable(v) || v.stride[1] != 1 || v.stride[0] <= 1 || bh_type_size(v.base->dtype()) != esize) continue;
        if (seen.insert(ViewKey(v)).second) {
            ret.push_back(v);
            transposed.push_back(false);
        }
    }
    return ret;
}

bool lower_tile2d(const LoopB &loop, const CodegenOptions &opt, LaunchUnit &u) {
    const Block holder(loop);
    Symbols sym = build_symbols({&holder}, {});
    const LoopB &L = holder.getLoop();
    const vector<const LoopB *> chain = jitk::get_first_loop_blocks(L);
    if (chain.size() < 2) return false;
    const LoopB &inner = *chain[1];
    vector<bool> tpose;
    const vector<bh_view> tv = tile2d_views(L, inner, sym, opt, tpose);
    if (tv.empty()) return false;
    const int stages = tv.size() <= 2 ? kTileStages : kTileStages - 1;
    const int esize = bh_type_size(tv[0].base->dtype());
    const int TR = 128 / esize, RPT = TR / 4;  // rows per tile, rows per thread
    u = LaunchUnit();
    u.sched = Sched::TILE2D;
    u.V = TR;
    u.rows = L.size;
    u.cols = inner.size;
    const int64_t tiles_c = (u.cols + kTileCols - 1) / kTileCols;
    ParamLayout pl;
    for (size_t k = 0; k < tv.size(); ++k) {
        // A transposed view's tile is TR elements along its base rows x 64 rows (128-byte swizzle);
        // a row-wise view's tile is 64 elements along its base rows x TR rows (no swizzle).
        ParamField f{ParamField::TMAP};
        f.base = tv[k].base;
        f.i64 = tv[k].start;
        f.tm_ld = tpose[k] ? tv[k].stride[1] : tv[k].stride[0];
        f.tm_box_x = tpose[k] ? TR : kTileCols;
        f.tm_box_y = tpose[k] ? kTileCols : TR;
        f.tm_xspan = tpose[k] ? u.rows : u.cols;
        f.tm_yspan = tpose[k] ? u.cols : u.rows;
        f.tm_swizzle = tpose[k];
        pl.add_tmap(f, "tm" + to_string(k));
    }
    add_common_fields(sym, pl, opt);
    pl.add(work_field(tiles_c), "bh_i64", "tiles_c");
    pl.add(work_field(u.work_items()), "bh_i64", "work");
    for (size_t k = 0; k < tv.size(); ++k) {
        // Tensor coordinates of the view's element (0, 0): column and row of its base array.
        const int64_t ld = tpose[k] ? tv[k].stride[1] : tv[k].stride[0];
        pl.add(work_field(tv[k].start >= 0 ? tv[k].start % ld : 0), "bh_i64", "tx" + to_string(k));
        pl.add(work_field(tv[k].start >= 0 ? tv[k].start / ld : 0), "bh_i64", "ty" + to_string(k));
    }
    ParamField ok{ParamField::TMA_OK};
    pl.add(ok, "bh_i64", "tma_ok");
    ParamField err{ParamField::SCRATCH};
    err.i64 = -1;  // the engine's error record
    pl.add(err, "unsigned long long*", "err");
    pl.pad64();

    const string T = cuda_type(tv[0].base->dtype());
    const string rows = "p.n" + to_string(sym.loop_id.at(&L)), cols = "p.n" + to_string(sym.loop_id.at(&inner));
    stringstream body;
    body << "// bh_dynamic_shared_bytes: " << stages * static_cast<int>(tv.size()) * kTileBoxBytes + 1024 << "\n";
    body << "template <bool STAGED> __device__ __forceinline__ void bh_tile(const P &p, bh_i64 w, const unsigned char *stage) {\n";
    body << pointer_locals(sym);
    body << "    const bh_i64 tr = w / p.tiles_c;\n";
    body << "    const bh_i64 tc = w - tr * p.tiles_c;\n";
    body << "    const int c = threadIdx.x & 63, rq = threadIdx.x >> 6;\n";
    body << "    const bh_i64 i1 = tc * 64 + c;\n";
    body << "    const bh_i64 rbase = tr * " << TR << " + rq * " << RPT << ";\n";
    for (size_t k = 0; k < tv.size(); ++k) {
        body << "    " << T << " tv" << k << "[" << RPT << "];\n";
        if (!tpose[k]) {
            // row-wise: row r of the tile at r * 64 elements, read in the element loop
            body << "    const " << T << " *tr" << k << " = (const " << T << " *)(stage + " << k * kTileBoxBytes
                 << ") + (rq * " << RPT << ") * 64 + c;\n";
            continue;
        }
        body << "    if (STAGED) {\n";
        body << "        const unsigned char *row = stage + " << k * kTileBoxBytes << " + c * 128;\n";
        body << "        const uint4 q0 = *(const uint4 *)(row + (((2 * rq) ^ (c & 7)) << 4));\n";
        body << "        const uint4 q1 = *(const uint4 *)(row + (((2 * rq + 1) ^ (c & 7)) << 4));\n";
        body << "        memcpy(&tv" << k << "[0], &q0, 16);\n";
        body << "        memcpy((char *)&tv" << k << "[0] + 16, &q1, 16);\n";
        body << "    }\n";
    }
    for (int path = 0; path < 2; ++path) {
        body << (path == 0 ? "    if (rbase + " + to_string(RPT) + " <= " + rows + " && i1 < " + cols + ") {\n"
                           : "    } else {\n");
        Scope scope;
        Emitter eb(sym, body, opt);
        for (size_t k = 0; k < tv.size(); ++k) scope.repl[ViewKey(tv[k])] = "tv" + to_string(k) + "[e]";
        if (path == 0) body << "#pragma unroll\n";
        body << "        for (int e = 0; e < " << RPT << "; ++e) {\n";
        body << "            const bh_i64 i0 = rbase + e;\n";
        if (path == 1) body << "            if (i0 >= " << rows << " || i1 >= " << cols << ") break;\n";
        for (size_t k = 0; k < tv.size(); ++k) {
            if (tpose[k]) {
                body << "            if (!STAGED) tv" << k << "[e] = " << eb.array_ref(tv[k]) << ";\n";
            } else {
                body << "            tv" << k << "[e] = STAGED ? tr" << k << "[e * 64] : " << eb.array_ref(tv[k]) << ";\n";
            }
        }
        declare_chain_temps(eb, sym, scope, chain, 1, body, 12);
        eb.write_body(inner, scope, 12);
        body << "        }\n";
    }
    body << "    }\n}\n";
    body << "__device__ __forceinline__ void bh_work(const P &p, bh_i64 w) { bh_tile<false>(p, w, nullptr); }\n";
    // One thread issues a tile's boxes: expect their bytes on the stage's barrier, then copy.
    body << "__device__ __forceinline__ void bh_tile_issue(const P &p, bh_i64 w, unsigned char *stage, unsigned long long *bar) {\n";
    body << "    const bh_i64 tr = w / p.tiles_c;\n";
    body << "    const bh_i64 tc = w - tr * p.tiles_c;\n";
    body << "    bh_mbar_expect_tx(bar, " << tv.size() * kTileBoxBytes << "u);\n";
    for (size_t k = 0; k < tv.size(); ++k) {
        if (tpose[k]) {
            body << "    bh_tma_2d(stage + " << k * kTileBoxBytes << ", &p.tm" << k << ", (int)(p.tx" << k << " + tr * " << TR
                 << "), (int)(p.ty" << k << " + tc * 64), bar);\n";
        } else {
            body << "    bh_tma_2d(stage + " << k * kTileBoxBytes << ", &p.tm" << k << ", (int)(p.tx" << k
                 << " + tc * 64), (int)(p.ty" << k << " + tr * " << TR << "), bar);\n";
        }
    }
    body << "}\n";
    const int stage_bytes = static_cast<int>(tv.size()) * kTileBoxBytes;
    body << R"CUDA(__device__ __forceinline__ void bh_main(const P &p) {
    if (!p.tma_ok) {
        for (bh_i64 w = blockIdx.x; w < p.work; w += gridDim.x) bh_tile<false>(p, w, nullptr);
        return;
    }
    extern __shared__ unsigned char bh_dyn[];
    // The 128-byte swizzle repeats every 1024 bytes: the ring starts on a 1024-byte boundary.
    unsigned char *ring = bh_dyn + ((1024u - (bh_saddr(bh_dyn) & 1023u)) & 1023u);
    __shared__ alignas(8) unsigned long long bar[)CUDA" << stages << R"CUDA(];
    __shared__ int fail;
    const bh_i64 first = blockIdx.x, step = gridDim.x;
    const int mine = first < p.work ? (int)((p.work - 1 - first) / step + 1) : 0;
    if (threadIdx.x == 0) {
        for (int s = 0; s < )CUDA" << stages << R"CUDA(; ++s) bh_mbar_init(&bar[s], 1u);
        bh_mbar_fence_init();
        fail = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int it = 0; it < )CUDA" << stages << R"CUDA( && it < mine; ++it)
            bh_tile_issue(p, first + it * step, ring + it * )CUDA" << stage_bytes << R"CUDA(, &bar[it]);
    int it = 0;
    for (; it < mine; ++it) {
        const int s = it % )CUDA" << stages << R"CUDA(;
        if (!bh_mbar_wait(&bar[s], (unsigned)((it / )CUDA" << stages << R"CUDA() & 1))) fail = 1;
        __syncthreads();
        if (fail) break;
        bh_tile<true>(p, first + it * step, ring + s * )CUDA" << stage_bytes << R"CUDA();
        __syncthreads();  // every thread is done with the stage
        if (threadIdx.x == 0 && it + )CUDA" << stages << R"CUDA( < mine)
            bh_tile_issue(p, first + (it + )CUDA" << stages << R"CUDA() * step, ring + s * )CUDA" << stage_bytes << R"CUDA(, &bar[s]);
    }
    if (fail && threadIdx.x == 0) {
        // A tile load never completed: record it, and let the copies already issued into the
        // ring land (bounded) before the CTA leaves.
        atomicCAS(p.err, 0ull, 0xC000000000000000ull | (unsigned long long)blockIdx.x);
        for (int j = it; j < mine && j < it + )CUDA" << stages << R"CUDA(; ++j)
            bh_mbar_wait(&bar[j % )CUDA" << stages << R"CUDA(], (unsigned)((j / )CUDA" << stages << R"CUDA() & 1));
    }
}
)CUDA";
    body << kBatchWork << kKernels;
    u.fields = pl.fields;
    u.algorithmic_bytes = unit_bytes(sym, vector<const Block *>{&holder});
    u.elements = u.rows * u.cols;
    finish_source(u, pl.decl.str(), body.str(), opt);
    return true;
}

// Parallel points below which an inner reduction is split along its swept axis, and the number of
// (point, chunk) threads the split aims at. Both are fixed constants so that the summation order
// depends on the array shapes only.
constexpr int64_t kSplitTargetThreads = 600000;
constexpr int64_t kSplitMinChunk = 16;
// Points from which LANE_REDUCE (C lanes of one CTA per point) fills the GPU well enough to be
// preferred over SPLIT_REDUCE when the swept axis is contiguous.
constexpr int64_t kLaneMinPoints = 148;
// (point, lane) threads LANE_REDUCE aims at when it picks the lanes per point (fewer lanes per
// point, with each CTA holding several neighbouring points, measured slower on the 4096^2 heat
// stencil: 16-64 lanes took 1.6-2.1x the time of 256).
constexpr int64_t kLaneTargetThreads = 600000;

// The swept sub-loop of `inner` when `inner` is [identity instructions] [swept innermost sub-loop]
// [instructions], and the sub-loop's sweeps are reductions; nullptr otherwise.
const LoopB *split_candidate(const LoopB &inner) {
    const LoopB *sub = nullptr;
    bool after = false;
    for (const Block &b : inner._block_list) {
        if (b.isInstr()) {
            if (!after) {
                const bh_instruction &i = *b.getInstr();
                if (!(i.opcode == BH_IDENTITY && i.operand.size() == 2 && i.operand[1].isConstant())) return nullptr;
            }
            continue;
        }
        if (sub != nullptr) return nullptr;
        sub = &b.getLoop();
        after = true;
    }
    if (sub == nullptr || sub->_sweeps.empty() || !sub->isInnermost()) return nullptr;
    for (const InstrPtr &s : sub->_sweeps)
        if (!bh_opcode_is_reduction(s->opcode) || !jitk::sweeping_innermost_axis(s)) return nullptr;
    // The identities must initialise outputs of these sweeps.
    set<ViewKey> outs;
    for (const InstrPtr &s : sub->_sweeps) outs.insert(ViewKey(s->operand[0]));
    for (const Block &b : inner._block_list) {
        if (!b.isInstr()) break;
        if (!outs.count(ViewKey(b.getInstr()->operand[0]))) return nullptr;
    }
    return sub;
}

int64_t split_chunks(int64_t points, int64_t len) {
    if (points <= 0 || len <= 0) return 1;
    const int64_t want = (kSplitTargetThreads + points - 1) / points;
    const int64_t most = max<int64_t>(1, len / kSplitMinChunk);
    return max<int64_t>(1, min(want, most));
}

int ilog2(int64_t x) {
    int r = 0;
    while ((int64_t(1) << (r + 1)) <= x) ++r;
    return r;
}

// Lanes per point of LANE_REDUCE: a power of two up to a CTA (256) chosen from the shapes alone.
int64_t lane_count(int64_t points, int64_t len) {
    int64_t c = 1;
    while (c < kThreads && points * c < kLaneTargetThreads && c * 4 <= len) c *= 2;
    return c;
}

// True when every array the swept sub-loop (at `rank`) reads walks that axis with unit stride (or
// broadcasts along it), and at least one does: C consecutive lanes then read adjacent elements.
bool swept_axis_contiguous(const LoopB &sub, int rank) {
    bool unit = false;
    for (const InstrPtr &ip : jitk::all_instr(sub)) {
        for (size_t o = 1; o < ip->operand.size(); ++o) {
            const bh_view &v = ip->operand[o];
            if (v.isConstant() || v.ndim <= rank) continue;
            const int64_t st = v.stride[rank];
            if (st == 1) {
                unit = true;
            } else if (st != 0 && v.shape[rank] > 1) {
                return false;
            }
        }
    }
    return unit;
}

// LANE_REDUCE: the SPLIT_REDUCE structure ([identities] [swept innermost sub-loop] [instructions]
// inside P threaded ranks) when the swept axis is contiguous in memory. C lanes of one CTA share a
// point: lane c folds elements c, c+C, c+2C, ... in order (adjacent lanes read adjacent elements),
// then the C lane partials are combined by a fixed shuffle tree (xor C/2 .. 1 within a warp; for
// C > 32 the warp sums are folded in warp order), and lane 0 runs the instructions that follow.
// No scratch memory and no counters: one pass.
// Stencil groups for LANE_REDUCE with one point axis and a CTA per point: read-only 2-D views of
// one base with equal strides, unit column stride and a row stride of at least 64 elements, whose
// starts differ by dk whole rows and dm (|dm| <= 8) columns, e.g. x[i-1, j], x[i, j-1], x[i, j],
// x[i, j+1], x[i+1, j]. Member i reads, at point i0 and column j, element
// s0 + (i0 + dk_i) * S0 + dm_i + j of the base, so the rows a CTA needs for consecutive points
// overlap and can be staged once in shared memory.
// Rows a staging CTA keeps in flight beyond the ones the current point reads (on the 4096^2
// heat stencil, 2 and 3 took 3 % longer than 1 -- fewer CTAs fit in shared memory -- and 0 took
// 8 % longer although four CTAs fit).
constexpr int64_t kStagePrefetch = 1;

struct StencilMember {
    size_t view;  // index in the view list
    int64_t dk, dm;
};
struct StencilGroup {
    vector<StencilMember> m;
    int64_t kmin = 0, kspan = 0, mmin = 0, mspan = 0;
};

StencilGroup stencil_group(const vector<bh_view> &views, const Symbols &sym) {
    StencilGroup best;
    for (size_t a = 0; a < views.size(); ++a) {
        const bh_view &va = views[a];
        if (va.ndim != 2 || va.stride[1] != 1 || va.stride[0] < 64 || va.hasSlide()) continue;
        const int ga = sym.view_group.at(static_cast<size_t>(sym.view_id.at(va)));
        const int64_t S0 = va.stride[0];
        StencilGroup g;
        for (size_t b = 0; b < views.size(); ++b) {
            const bh_view &vb = views[b];
            if (vb.base != va.base || vb.ndim != 2 || vb.hasSlide() ||
                sym.view_group.at(static_cast<size_t>(sym.view_id.at(vb))) != ga)
                continue;
            const int64_t d = vb.start - va.start;
            const int64_t dk = d >= 0 ? (d + S0 / 2) / S0 : -((-d + S0 / 2) / S0);
            const int64_t dm = d - dk * S0;
            if (dm < -8 || dm > 8) continue;
            g.m.push_back({b, dk, dm});
        }
        int64_t kmax = g.m[0].dk, mmax = g.m[0].dm;
        g.kmin = kmax;
        g.mmin = mmax;
        for (const StencilMember &x : g.m) {
            g.kmin = min(g.kmin, x.dk);
            kmax = max(kmax, x.dk);
            g.mmin = min(g.mmin, x.dm);
            mmax = max(mmax, x.dm);
        }
        g.kspan = kmax - g.kmin;
        g.mspan = mmax - g.mmin;
        if (g.kspan < 1 || g.kspan > 4) continue;  // no row shared between points, or too many rows
        if (g.m.size() > best.m.size()) best = g;
    }
    return best;
}

// Asynchronous global -> shared copies (cp.async, completed in commit groups) for staged rows.
const char *kStagePrelude = R"CUDA(
__device__ __forceinline__ void bh_cp16(void *s, const void *g) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"((unsigned)__cvta_generic_to_shared(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void bh_cp8(void *s, const void *g) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" :: "r"((unsigned)__cvta_generic_to_shared(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void bh_cp4(void *s, const void *g) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" :: "r"((unsigned)__cvta_generic_to_shared(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void bh_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void bh_cp_wait() { asm volatile("cp.async.wait_group %0;" :: "n"(N) : "memory"); }
__device__ __forceinline__ void bh_cp_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
// Stage `nelem` elements starting at `src` into dst[pre ...] (dst 16-byte aligned, src - pre a
// 16-byte boundary): whole 16-byte chunks in one copy, the partial chunks at either end element
// by element. Nothing outside [src, src + nelem) is read.
template <typename T> __device__ __forceinline__ void bh_stage_row(T *dst, const T *src, bh_i64 nelem, int pre) {
    const char *g = (const char *)src - pre * (int)sizeof(T);
    char *d = (char *)dst;
    const bh_i64 b_lo = (bh_i64)pre * (bh_i64)sizeof(T), b_hi = b_lo + nelem * (bh_i64)sizeof(T);
    const bh_i64 nchunks = (b_hi + 15) / 16;
    for (bh_i64 c = threadIdx.x; c < nchunks; c += blockDim.x) {
        const bh_i64 b0 = c * 16;
        if (b0 >= b_lo && b0 + 16 <= b_hi) {
            bh_cp16(d + b0, g + b0);
        } else {
            for (bh_i64 b = b0 > b_lo ? b0 : b_lo; b < b0 + 16 && b < b_hi; b += (bh_i64)sizeof(T)) {
                if (sizeof(T) == 4) bh_cp4(d + b, g + b);
                else bh_cp8(d + b, g + b);
            }
        }
    }
}
)CUDA";

LaunchUnit lower_lane_reduce(const LoopB &loop, unsigned P, const CodegenOptions &opt) {
    LaunchUnit u;
    u.sched = Sched::LANE_REDUCE;
    const Block holder(loop);
    const LoopB &L = holder.getLoop();
    const vector<const LoopB *> chain = jitk::get_first_loop_blocks(L);
    const LoopB &inner = *chain[P - 1];
    const LoopB &sub = *split_candidate(inner);
    set<const bh_instruction *> folded;
    for (const Block &b : inner._block_list) {
        if (!b.isInstr()) break;
        folded.insert(b.getInstr().get());
    }
    Symbols sym = build_symbols({&holder}, folded);
    vector<InstrPtr> reds(sub._sweeps.begin(), sub._sweeps.end());
    sort(reds.begin(), reds.end(), [](const InstrPtr &a, const InstrPtr &b) { return a->origin_id < b->origin_id; });
    u.nred = static_cast<int>(reds.size());
    int64_t rows = 1;
    for (unsigned r = 0; r + 1 < P; ++r) rows *= chain[r]->size;
    u.rows = rows;
    u.cols = inner.size;
    const int64_t points = rows * inner.size;
    const int64_t C = lane_count(points, sub.size);
    u.chunks = C;
    for (const InstrPtr &r : reds)
        u.red_orders.emplace_back(r->origin_id, "lanes:" + to_string(C) + ":" + to_string(sub.size));
    ParamLayout pl;
    add_common_fields(sym, pl, opt);
    pl.add(work_field(points), "bh_i64", "points");
    pl.add(work_field(u.work_items()), "bh_i64", "work");

    stringstream body;
    Emitter em(sym, body, opt);
    vector<string> ctypes, idents;
    for (size_t k = 0; k < reds.size(); ++k) {
        const bh_type t = reds[k]->operand[0].base->dtype();
        ctypes.push_back(cuda_type(t));
        idents.push_back(constant_literal(jitk::sweep_identity(reds[k]->opcode, t)));
        em.external_acc[ViewKey(reds[k]->operand[0])] = "pacc" + to_string(k);
    }
    const int sub_lid = sym.loop_id.at(&sub);
    const int64_t per_cta = kThreads / C;


    body << "__device__ void bh_work(const P &p, bh_i64 w) {\n";
    body << pointer_locals(sym);
    if (C > 32) {
        for (size_t k = 0; k < reds.size(); ++k)
            body << "    __shared__ " << ctypes[k] << " wsum" << k << "[" << kThreads / 32 << "];\n";
    }
    body << "    const int lane = threadIdx.x & " << (C - 1) << ";\n";
    body << "    const bh_i64 pt = w * " << per_cta << " + (threadIdx.x >> " << ilog2(C) << ");\n";
    for (size_t k = 0; k < reds.size(); ++k) body << "    " << ctypes[k] << " pacc" << k << " = " << idents[k] << ";\n";
    auto decompose = [&](int ind) {
        const string sp(static_cast<size_t>(ind), ' ');
        body << sp << "bh_i64 rem = pt;\n";
        for (int r = static_cast<int>(P) - 1; r >= 0; --r) {
            const int lid = sym.loop_id.at(chain[r]);
            if (r == 0) {
                body << sp << "const bh_i64 i0 = rem;\n";
            } else {
                body << sp << "const bh_i64 i" << r << " = rem % p.n" << lid << "; rem /= p.n" << lid << ";\n";
            }
        }
        body << sp << "(void)rem;\n";
    };
    body << "    if (pt < p.points) {\n";
    decompose(8);
    {
        Scope scope;
        declare_chain_temps(em, sym, scope, chain, P, body, 8);
        // Inputs that this kernel does not write are loaded for U strided iterations at once
        // before any of them computes or stores: a store may alias a later load as far as the
        // compiler can tell, so without this each iteration's loads wait for the previous one.
        // Every lane still folds its elements in increasing order.
        const vector<bh_view> pre = preloadable_views(sub, L, sym);
        const int64_t U = pre.empty() ? 1 : (pre.size() <= 8 ? 4 : 2);
        const string iv = "i" + to_string(P), nv = "p.n" + to_string(sub_lid);
        hoist_views(em, sub, static_cast<int>(P), body, 8);
        if (U > 1 && sub.size / C >= U) {
            body << "/*@unroll@*/\n";
            body << "        for (bh_i64 ib = lane; ib < " << nv << "; ib += " << C * U << ") {\n";
            body << "            if (ib + " << C * (U - 1) << " < " << nv << ") {\n";
            for (size_t k = 0; k < pre.size(); ++k)
                body << "                " << cuda_type(pre[k].base->dtype()) << " pl" << k << "[" << U << "];\n";
            body << "#pragma unroll\n";
            body << "                for (int j = 0; j < " << U << "; ++j) {\n";
            body << "                    const bh_i64 " << iv << " = ib + j * " << C << ";\n";
            for (size_t k = 0; k < pre.size(); ++k)
                body << "                    pl" << k << "[j] = " << em.array_ref(pre[k]) << ";\n";
            body << "                }\n";
            body << "#pragma unroll\n";
            body << "                for (int j = 0; j < " << U << "; ++j) {\n";
            body << "                    const bh_i64 " << iv << " = ib + j * " << C << ";\n";
            Scope s1;
            s1.parent = &scope;
            for (size_t k = 0; k < pre.size(); ++k) s1.repl[ViewKey(pre[k])] = "pl" + to_string(k) + "[j]";
            em.write_body(sub, s1, 20);
            body << "                }\n";
            body << "            } else {\n";
            body << "                for (bh_i64 " << iv << " = ib; " << iv << " < " << nv << "; " << iv << " += " << C
                 << ") {\n";
            Scope s2;
            s2.parent = &scope;
            em.write_body(sub, s2, 20);
            body << "                }\n";
            body << "            }\n";
            body << "        }\n";
        } else {
            body << "/*@unroll@*/\n";
            body << "        for (bh_i64 " << iv << " = lane; " << iv << " < " << nv << "; " << iv << " += " << C << ") {\n";
            Scope s1;
            s1.parent = &scope;
            em.write_body(sub, s1, 12);
            body << "        }\n";
        }
        em.hoisted.clear();
        em.hoist_axis = -1;
    }
    body << "    }\n";
    // Combine the C lanes of each point (every lane of the warp takes part; lanes of points past
    // the end hold the identity).
    const int64_t in_warp = C < 32 ? C : 32;
    for (size_t k = 0; k < reds.size(); ++k) {
        body << "#pragma unroll\n";
        body << "    for (int m = " << in_warp / 2 << "; m >= 1; m >>= 1) { const " << ctypes[k]
             << " o = bh_shfl_xor(pacc" << k << ", m); pacc" << k << " = "
             << reduce_expr(reds[k]->opcode, "pacc" + to_string(k), "o") << "; }\n";
    }
    if (C > 32) {
        const int64_t nw = C / 32;
        for (size_t k = 0; k < reds.size(); ++k) body << "    if ((threadIdx.x & 31) == 0) wsum" << k << "[threadIdx.x >> 5] = pacc" << k << ";\n";
        body << "    __syncthreads();\n";
        body << "    if (lane == 0) {\n";
        body << "        const int w0 = threadIdx.x >> 5;\n";
        for (size_t k = 0; k < reds.size(); ++k) {
            body << "        pacc" << k << " = wsum" << k << "[w0];\n";
            body << "        for (int j = 1; j < " << nw << "; ++j) pacc" << k << " = "
                 << reduce_expr(reds[k]->opcode, "pacc" + to_string(k), "wsum" + to_string(k) + "[w0 + j]") << ";\n";
        }
        body << "    }\n";
        body << "    __syncthreads();  // wsum is rewritten by the next work item of this CTA\n";
    }
    body << "    if (lane != 0 || pt >= p.points) return;\n";
    {
        decompose(4);
        Scope scope;
        declare_chain_temps(em, sym, scope, chain, P - 1, body, 4);
        for (const bh_base *b : em.sorted_temps(inner)) {
            if (sym.temps.count(b) && !scope.is_tmp(b)) {
                scope.tmps.insert(b);
                body << "    " << cuda_type(b->dtype()) << " t" << sym.base_index(b) << ";\n";
            }
        }
        bool after = false;
        for (const Block &b : inner._block_list) {
            if (!b.isInstr()) {
                after = true;
                continue;
            }
            if (after) em.write_instr(*b.getInstr(), scope, 4);
        }
        for (size_t k = 0; k < reds.size(); ++k) {
            if (sym.temps.count(reds[k]->operand[0].base)) continue;
            body << "    " << em.array_ref(reds[k]->operand[0], reds[k]->sweep_axis()) << " = pacc" << k << ";\n";
        }
    }
    body << "}\n";

    // Staged rows: with one point axis, a CTA per point and a stencil group among the read-only
    // views, each CTA walks a contiguous range of points (rows) and keeps the group's rows in a
    // ring of shared-memory buffers filled by asynchronous copies one row ahead, so every base
    // row is read once per CTA and the copies overlap the computation. The lanes fold the same
    // elements in the same order as bh_work. A kernel-side check (layout, view offsets, bounds)
    // falls back to bh_work for launches the staging does not fit.
    bool staged = false;
    if (P == 1 && C == kThreads && !opt.bounds_check) {
        const vector<bh_view> pre = preloadable_views(sub, L, sym);
        const StencilGroup g = stencil_group(pre, sym);
        const bh_view *v0 = g.m.empty() ? nullptr : &pre[g.m[0].view];
        const int64_t es = v0 ? bh_type_size(v0->base->dtype()) : 0;
        const int64_t n = sub.size, U = (n + C - 1) / C, F = n / C;
        const int64_t nrow = n + g.mspan, CE = es > 0 ? 16 / es : 1, NB = g.kspan + 1 + kStagePrefetch;
        const int64_t RS = (nrow + CE - 1 + CE - 1) / CE * CE;
        const int64_t smem = NB * RS * es;
        if (v0 != nullptr && (es == 4 || es == 8) && U <= 16 && smem <= 160 * 1024) {
            staged = true;
            const string T = cuda_type(v0->base->dtype());
            const int gid = sym.view_group.at(static_cast<size_t>(sym.view_id.at(*v0)));
            const int vid0 = sym.view_id.at(*v0);
            const int pid = sym.param_id.at(v0->base);
            const string nv = "p.n" + to_string(sub_lid), S0 = "p.g" + to_string(gid) + "_s0";
            ParamField fe{ParamField::I64};
            fe.i64 = v0->base->nelem();
            pl.add(fe, "bh_i64", "stage_nelem");
            if (opt.stage_bulk) {
                ParamField fok{ParamField::TMA_OK};  // bulk copies allowed (not in grouped launches)
                pl.add(fok, "bh_i64", "tma_ok");
                ParamField ferr{ParamField::SCRATCH};
                ferr.i64 = -1;  // the engine's error record
                pl.add(ferr, "unsigned long long*", "err");
            }
            body << "// bh_dynamic_shared_bytes: " << smem << "\n";
            body << kStagePrelude;
            // Launch-time check: the layout the staging assumes holds for these parameters, and
            // every staged row lies inside the base.
            body << "__device__ __forceinline__ bool bh_stage_ok(const P &p, bh_i64 lo, bh_i64 hi) {\n";
            body << "    const bh_i64 S0 = " << S0 << ";\n";
            body << "    if (S0 < " << nrow << " || (S0 * " << es << ") % 16 != 0 || " << nv << " != " << n
                 << ") return false;\n";
            for (const StencilMember &x : g.m) {
                const int vid = sym.view_id.at(pre[x.view]);
                body << "    if (p.v" << vid << "_o - p.v" << vid0 << "_o != " << x.dk << "LL * S0 + (" << x.dm
                     << "LL)) return false;\n";
            }
            body << "    const bh_i64 first = p.v" << vid0 << "_o + (lo + (" << g.kmin << "LL)) * S0 + (" << g.mmin
                 << "LL);\n";
            body << "    const bh_i64 last = p.v" << vid0 << "_o + (hi - 1 + (" << g.kmin + g.kspan << "LL)) * S0 + ("
                 << g.mmin << "LL) + " << nrow << ";\n";
            body << "    return first >= 0 && last <= p.stage_nelem;\n";
            body << "}\n";
            // The bulk form copies each row from the 16-byte boundary at or below its first element
            // to the 16-byte boundary at or above its end: that span must lie inside the base.
            body << "__device__ __forceinline__ bool bh_bulk_ok(const P &p, bh_i64 lo, bh_i64 hi) {\n";
            body << "    const bh_i64 S0 = " << S0 << ";\n";
            body << "    if (((unsigned long long)p.a" << pid << " & 15ULL) != 0) return false;\n";
            body << "    const bh_i64 first = p.v" << vid0 << "_o + (lo + (" << g.kmin << "LL)) * S0 + (" << g.mmin << "LL);\n";
            body << "    const bh_i64 pre = first % " << CE << ";\n";
            body << "    const bh_i64 span = (pre + " << nrow << " + " << CE - 1 << ") / " << CE << " * " << CE << ";\n";
            body << "    const bh_i64 last = p.v" << vid0 << "_o + (hi - 1 + (" << g.kmin + g.kspan << "LL)) * S0 + (" << g.mmin
                 << "LL) - pre + span;\n";
            body << "    return span <= " << RS << " && last <= p.stage_nelem;\n";
            body << "}\n";
            // Two forms of the staged walk: `bulk` fills each ring row with one cp.async.bulk copy
            // (the TMA engine, issued by one thread, completion counted on the row slot's
            // mbarrier; waits bounded), the other with 16-byte cp.async copies by every thread
            // (commit groups). Grouped launches (no error-record check) take the cp.async form.
            auto emit_staged = [&](bool bulk) {
            const string fname = bulk ? "bh_work_bulk" : "bh_work_staged";
            body << "__device__ void " << fname << "(const P &p, bh_i64 lo, bh_i64 hi) {\n";
            body << "    extern __shared__ __align__(16) unsigned char bh_dyn[];\n";
            body << "    " << T << "* ring = (" << T << "*)bh_dyn;\n";
            body << pointer_locals(sym);
            for (size_t k = 0; k < reds.size(); ++k)
                body << "    __shared__ " << ctypes[k] << " wsum" << k << "[2][" << kThreads / 32 << "];\n";
            body << "    const int lane = threadIdx.x;\n";
            body << "    const bh_i64 S0 = " << S0 << ";\n";
            body << "    const " << T << "* rows0 = a" << pid << " + (p.v" << vid0 << "_o + (" << g.kmin << "LL) * S0 + ("
                 << g.mmin << "LL));\n";
            body << "    const int pre = (int)(((unsigned long long)(rows0 + lo * S0) & 15ULL) / " << es << ");\n";
            body << "    const bh_i64 rend = hi + " << g.kspan << ";\n";
            if (bulk) {
                // Row r (relative index r - lo) lives in slot (r - lo) % NB; its copy is the
                // ((r - lo) / NB)-th completion of that slot's barrier.
                body << "    const unsigned row_bytes = (unsigned)(((pre + " << nrow << ") * " << es << " + 15) / 16 * 16);\n";
                body << "    __shared__ alignas(8) unsigned long long bar[" << NB << "];\n";
                body << "    __shared__ int fail;\n";
                body << "    if (threadIdx.x == 0) {\n";
                body << "        for (int b = 0; b < " << NB << "; ++b) bh_mbar_init(&bar[b], 1u);\n";
                body << "        bh_mbar_fence_init();\n";
                body << "        fail = 0;\n";
                body << "    }\n";
                body << "    __syncthreads();\n";
                body << "    bh_i64 issued = lo, waited = lo;  // rows [lo, issued) copied, [lo, waited) arrived (thread 0)\n";
                body << "    if (threadIdx.x == 0) {\n";
                body << "        for (; issued < rend && issued < lo + " << NB << "; ++issued) {\n";
                body << "            const int b = (int)(issued - lo);\n";
                body << "            bh_mbar_expect_tx(&bar[b], row_bytes);\n";
                body << "            bh_bulk_row(ring + b * " << RS << ", (const char *)(rows0 + issued * S0) - pre * " << es
                     << ", row_bytes, &bar[b]);\n";
                body << "        }\n";
                body << "    }\n";
            } else {
                body << "    for (int b = 0; b < " << NB << "; ++b) {\n";
                body << "        const bh_i64 r = lo + b;\n";
                body << "        if (r < rend) bh_stage_row(ring + (r % " << NB << ") * " << RS << ", rows0 + r * S0, (bh_i64)"
                     << nrow << ", pre);\n";
                body << "        bh_cp_commit();\n";
                body << "    }\n";
            }
            body << "    for (bh_i64 pt = lo; pt < hi; ++pt) {\n";
            if (bulk) {
                // Rows pt .. pt + kspan are read; all but the newest arrived by earlier points.
                body << "        for (bh_i64 r = (pt == lo ? lo : pt + " << g.kspan << "); r <= pt + " << g.kspan << "; ++r) {\n";
                body << "            const int b = (int)((r - lo) % " << NB << ");\n";
                body << "            if (!bh_mbar_wait(&bar[b], (unsigned)(((r - lo) / " << NB << ") & 1))) fail = 1;\n";
                body << "            else if (threadIdx.x == 0) waited = r + 1;\n";
                body << "        }\n";
                body << "        __syncthreads();\n";
                body << "        if (fail) break;\n";
            } else {
                body << "        bh_cp_wait<" << kStagePrefetch << ">();  // all but the newest prefetched rows have landed\n";
                body << "        __syncthreads();\n";
            }
            body << "        const bh_i64 i0 = pt;\n";
            for (size_t k = 0; k < reds.size(); ++k)
                body << "        " << ctypes[k] << " pacc" << k << " = " << idents[k] << ";\n";
            for (size_t k = 0; k < g.m.size(); ++k) {
                if (bulk) {
                    body << "        const " << T << "* sr" << k << " = ring + ((pt - lo + " << g.m[k].dk - g.kmin << ") % " << NB
                         << ") * " << RS << " + pre + " << g.m[k].dm - g.mmin << ";\n";
                } else {
                    body << "        const " << T << "* sr" << k << " = ring + ((pt + " << g.m[k].dk - g.kmin << ") % " << NB
                         << ") * " << RS << " + pre + " << g.m[k].dm - g.mmin << ";\n";
                }
            }
            {
                Scope scope;
                declare_chain_temps(em, sym, scope, chain, P, body, 8);
                body << (U <= 16 ? "#pragma unroll\n" : "#pragma unroll 4\n");
                body << "        for (int j = 0; j < " << U << "; ++j) {\n";
                body << "            const bh_i64 i1 = lane + j * " << C << ";\n";
                body << "            if (j < " << F << " || i1 < " << nv << ") {\n";
                Scope s1;
                s1.parent = &scope;
                for (size_t k = 0; k < g.m.size(); ++k) s1.repl[ViewKey(pre[g.m[k].view])] = "sr" + to_string(k) + "[i1]";
                em.write_body(sub, s1, 16);
                body << "            }\n";
                body << "        }\n";
            }
            for (size_t k = 0; k < reds.size(); ++k) {
                body << "#pragma unroll\n";
                body << "        for (int m = 16; m >= 1; m >>= 1) { const " << ctypes[k] << " o = bh_shfl_xor(pacc" << k
                     << ", m); pacc" << k << " = " << reduce_expr(reds[k]->opcode, "pacc" + to_string(k), "o") << "; }\n";
                body << "        if ((threadIdx.x & 31) == 0) wsum" << k << "[pt & 1][threadIdx.x >> 5] = pacc" << k << ";\n";
            }
            body << "        __syncthreads();  // also: every thread is done with the oldest row's buffer\n";
            body << "        const bh_i64 rnext = pt + " << NB << ";\n";
            if (bulk) {
                body << "        if (threadIdx.x == 0 && rnext < rend) {\n";
                body << "            const int b = (int)((rnext - lo) % " << NB << ");\n";
                body << "            bh_mbar_expect_tx(&bar[b], row_bytes);\n";
                body << "            bh_bulk_row(ring + b * " << RS << ", (const char *)(rows0 + rnext * S0) - pre * " << es
                     << ", row_bytes, &bar[b]);\n";
                body << "            issued = rnext + 1;\n";
                body << "        }\n";
            } else {
                body << "        if (rnext < rend) bh_stage_row(ring + (rnext % " << NB << ") * " << RS
                     << ", rows0 + rnext * S0, (bh_i64)" << nrow << ", pre);\n";
                body << "        bh_cp_commit();\n";
            }
            body << "        if (lane == 0) {\n";
            for (size_t k = 0; k < reds.size(); ++k) {
                body << "            pacc" << k << " = wsum" << k << "[pt & 1][0];\n";
                body << "            for (int j = 1; j < " << kThreads / 32 << "; ++j) pacc" << k << " = "
                     << reduce_expr(reds[k]->opcode, "pacc" + to_string(k), "wsum" + to_string(k) + "[pt & 1][j]")
                     << ";\n";
            }
            {
                Scope scope;
                declare_chain_temps(em, sym, scope, chain, P - 1, body, 12);
                for (const bh_base *b : em.sorted_temps(inner)) {
                    if (sym.temps.count(b) && !scope.is_tmp(b)) {
                        scope.tmps.insert(b);
                        body << "            " << cuda_type(b->dtype()) << " t" << sym.base_index(b) << ";\n";
                    }
                }
                bool after = false;
                for (const Block &b : inner._block_list) {
                    if (!b.isInstr()) {
                        after = true;
                        continue;
                    }
                    if (after) em.write_instr(*b.getInstr(), scope, 12);
                }
                for (size_t k = 0; k < reds.size(); ++k) {
                    if (sym.temps.count(reds[k]->operand[0].base)) continue;
                    body << "            " << em.array_ref(reds[k]->operand[0], reds[k]->sweep_axis()) << " = pacc" << k
                         << ";\n";
                }
            }
            body << "        }\n";
            body << "    }\n";
            if (bulk) {
                body << "    if (fail && threadIdx.x == 0) {\n";
                body << "        // A row copy never completed: record it, and let the copies still in flight into\n";
                body << "        // the ring land (bounded) before the CTA leaves.\n";
                body << "        atomicCAS(p.err, 0ull, 0xC000000000000000ull | (unsigned long long)blockIdx.x);\n";
                body << "        for (bh_i64 r = waited; r < issued; ++r)\n";
                body << "            bh_mbar_wait(&bar[(r - lo) % " << NB << "], (unsigned)(((r - lo) / " << NB << ") & 1));\n";
                body << "    }\n";
            } else {
                body << "    bh_cp_wait0();  // no copy in flight when the CTA leaves\n";
            }
            body << "}\n";
            };
            emit_staged(false);
            if (opt.stage_bulk) emit_staged(true);
            string wrappers = kWrappers;
            const string loop = "    for (bh_i64 w = blockIdx.x; w < p.work; w += gridDim.x) bh_work(p, w);\n";
            const size_t at = wrappers.find(loop);
            if (at == string::npos) throw runtime_error("lower_lane_reduce(): wrapper template changed");
            wrappers.replace(at, loop.size(),
                             "    // a contiguous range of points (rows) per CTA\n"
                             "    const bh_i64 lo = (bh_i64)blockIdx.x * p.work / gridDim.x;\n"
                             "    const bh_i64 hi = ((bh_i64)blockIdx.x + 1) * p.work / gridDim.x;\n"
                             "    if (lo < hi && bh_stage_ok(p, lo, hi)) {\n" +
                             string(opt.stage_bulk ? "        if (p.tma_ok && bh_bulk_ok(p, lo, hi)) bh_work_bulk(p, lo, hi);\n"
                                                     "        else bh_work_staged(p, lo, hi);\n"
                                                   : "        bh_work_staged(p, lo, hi);\n") +
                             "    } else {\n"
                             "        for (bh_i64 w = lo; w < hi; ++w) bh_work(p, w);\n"
                             "    }\n");
            body << wrappers;
        }
    }
    if (!staged) body << kWrappers;
    u.fields = pl.fields;
    u.algorithmic_bytes = unit_bytes(sym, vector<const Block *>{&holder});
    u.elements = points * sub.size;
    finish_source(u, pl.decl.str(), body.str(), opt);
    return u;
}

LaunchUnit lower_split_reduce(const LoopB &loop, unsigned P, const CodegenOptions &opt) {
    LaunchUnit u;
    u.sched = Sched::SPLIT_REDUCE;
    const Block holder(loop);
    const LoopB &L = holder.getLoop();
    const vector<const LoopB *> chain = jitk::get_first_loop_blocks(L);
    const LoopB &inner = *chain[P - 1];
    const LoopB &sub = *split_candidate(inner);
    set<const bh_instruction *> folded;
    for (const Block &b : inner._block_list) {
        if (!b.isInstr()) break;
        folded.insert(b.getInstr().get());
    }
    Symbols sym = build_symbols({&holder}, folded);
    vector<InstrPtr> reds(sub._sweeps.begin(), sub._sweeps.end());
    sort(reds.begin(), reds.end(), [](const InstrPtr &a, const InstrPtr &b) { return a->origin_id < b->origin_id; });
    u.nred = static_cast<int>(reds.size());
    int64_t rows = 1;
    for (unsigned r = 0; r + 1 < P; ++r) rows *= chain[r]->size;
    u.rows = rows;
    u.cols = inner.size;
    const int64_t points = rows * inner.size;
    u.chunks = split_chunks(points, sub.size);
    const int64_t chunk_len = (sub.size + u.chunks - 1) / u.chunks;
    for (const InstrPtr &r : reds)
        u.red_orders.emplace_back(r->origin_id, "split:" + to_string(u.chunks) + ":" + to_string(chunk_len) + ":" +
                                                    to_string(sub.size));
    ParamLayout pl;
    add_common_fields(sym, pl, opt);
    pl.add(work_field(points), "bh_i64", "points");
    pl.add(work_field(u.chunks), "bh_i64", "chunks");
    pl.add(work_field(chunk_len), "bh_i64", "chunk_len");
    pl.add(work_field(u.work_items()), "bh_i64", "work");
    ParamField fs{ParamField::SCRATCH};
    pl.add(fs, "unsigned char*", "scratch");
    ParamField fc{ParamField::COUNTER};
    pl.add(fc, "unsigned int*", "counter");

    stringstream body;
    Emitter em(sym, body, opt);
    vector<string> ctypes, idents;
    for (size_t k = 0; k < reds.size(); ++k) {
        const bh_type t = reds[k]->operand[0].base->dtype();
        ctypes.push_back(cuda_type(t));
        idents.push_back(constant_literal(jitk::sweep_identity(reds[k]->opcode, t)));
        em.external_acc[ViewKey(reds[k]->operand[0])] = "pacc" + to_string(k);
    }
    const int sub_lid = sym.loop_id.at(&sub);
    body << "__device__ void bh_work(const P &p, bh_i64 w) {\n";
    body << pointer_locals(sym);
    body << "    __shared__ bool am_last;\n";
    body << "    const bh_i64 pb = w / p.chunks, chunk = w - pb * p.chunks;\n";
    body << "    const bh_i64 pt = pb * " << kThreads << " + threadIdx.x;\n";
    u.slot_bytes = red_slot_bytes(reds);
    for (size_t k = 0; k < reds.size(); ++k)
        body << "    " << ctypes[k] << "* part" << k << " = (" << ctypes[k] << "*)(p.scratch + " << u.slot_bytes * k
             << " * p.chunks * p.points);\n";
    // Decompose the point into the threaded indices i0..i{P-1}.
    auto decompose = [&](int ind) {
        const string sp(static_cast<size_t>(ind), ' ');
        body << sp << "bh_i64 rem = pt;\n";
        for (int r = static_cast<int>(P) - 1; r >= 0; --r) {
            const int lid = sym.loop_id.at(chain[r]);
            if (r == 0) {
                body << sp << "const bh_i64 i0 = rem;\n";
            } else {
                body << sp << "const bh_i64 i" << r << " = rem % p.n" << lid << "; rem /= p.n" << lid << ";\n";
            }
        }
        body << sp << "(void)rem;\n";
    };
    body << "    if (pt < p.points) {\n";
    decompose(8);
    {
        Scope scope;
        declare_chain_temps(em, sym, scope, chain, P, body, 8);
        for (size_t k = 0; k < reds.size(); ++k) body << "        " << ctypes[k] << " pacc" << k << " = " << idents[k] << ";\n";
        body << "        const bh_i64 lo = chunk * p.chunk_len;\n";
        body << "        const bh_i64 hi = min(lo + p.chunk_len, (bh_i64)p.n" << sub_lid << ");\n";
        body << "/*@unroll@*/\n";  // the autotuner may put an unroll pragma here
        body << "        for (bh_i64 i" << P << " = lo; i" << P << " < hi; ++i" << P << ") {\n";
        Scope s1;
        s1.parent = &scope;
        em.write_body(sub, s1, 12);
        body << "        }\n";
        for (size_t k = 0; k < reds.size(); ++k)
            body << "        part" << k << "[chunk * p.points + pt] = pacc" << k << ";\n";
    }
    body << "    }\n";
    body << "    __syncthreads();\n";
    body << "    if (threadIdx.x == 0) {\n";
    body << "        am_last = bh_arrive((unsigned*)(p.counter + pb)) == (unsigned)(p.chunks - 1);\n";
    body << "    }\n";
    body << "    __syncthreads();\n";
    body << "    if (!am_last) return;\n";
    body << "    bh_acquire();\n";
    body << "    if (threadIdx.x == 0) p.counter[pb] = 0u;\n";
    body << "    if (pt >= p.points) return;\n";
    {
        decompose(4);
        Scope scope;
        declare_chain_temps(em, sym, scope, chain, P - 1, body, 4);
        // The chunk partials were written by other CTAs (made visible by the fence and the
        // counter): read them through L2 (ld.global.cg), eight loads in flight, folded in chunk
        // order.
        for (size_t k = 0; k < reds.size(); ++k) {
            const string acc = "pacc" + to_string(k), T = ctypes[k];
            body << "    " << T << " " << acc << " = " << idents[k] << ";\n";
            body << "    {\n";
            body << "        bh_i64 c = 0;\n";
            body << "        for (; c + 8 <= p.chunks; c += 8) {\n";
            body << "            " << T << " x[8];\n";
            body << "#pragma unroll\n";
            body << "            for (int j = 0; j < 8; ++j) x[j] = bh_ldcg(part" << k << " + (c + j) * p.points + pt);\n";
            body << "#pragma unroll\n";
            body << "            for (int j = 0; j < 8; ++j) " << acc << " = " << reduce_expr(reds[k]->opcode, acc, "x[j]")
                 << ";\n";
            body << "        }\n";
            body << "        for (; c < p.chunks; ++c) {\n";
            body << "            const " << T << " x = bh_ldcg(part" << k << " + c * p.points + pt);\n";
            body << "            " << acc << " = " << reduce_expr(reds[k]->opcode, acc, "x") << ";\n";
            body << "        }\n";
            body << "    }\n";
        }
        // Instructions after the swept sub-loop, then the reduction outputs.
        for (const bh_base *b : em.sorted_temps(inner)) {
            if (sym.temps.count(b) && !scope.is_tmp(b)) {
                scope.tmps.insert(b);
                body << "    " << cuda_type(b->dtype()) << " t" << sym.base_index(b) << ";\n";
            }
        }
        bool after = false;
        for (const Block &b : inner._block_list) {
            if (!b.isInstr()) {
                after = true;
                continue;
            }
            if (after) em.write_instr(*b.getInstr(), scope, 4);
        }
        for (size_t k = 0; k < reds.size(); ++k) {
            if (sym.temps.count(reds[k]->operand[0].base)) continue;
            body << "    " << em.array_ref(reds[k]->operand[0], reds[k]->sweep_axis()) << " = pacc" << k << ";\n";
        }
    }
    body << "}\n" << kWrappers;
    u.fields = pl.fields;
    u.algorithmic_bytes = unit_bytes(sym, vector<const Block *>{&holder});
    u.elements = points * sub.size;
    finish_source(u, pl.decl.str(), body.str(), opt);
    return u;
}

// CTA-wide deterministic tree reduction of `v` (fixed xor-shuffle butterfly, then warp 0); the
// result is valid in thread 0.
string block_reduce_fn(const string &ctype, const string &fname, bh_opcode op, const string &identity) {
    stringstream ss;
    ss << "__device__ __forceinline__ " << ctype << " " << fname << "(" << ctype << " v, " << ctype << " *sm) {\n";
    ss << "#pragma unroll\n";
    ss << "    for (int m = 16; m >= 1; m >>= 1) { const " << ctype << " o = bh_shfl_xor(v, m); v = "
       << reduce_expr(op, "v", "o") << "; }\n";
    ss << "    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;\n";
    ss << "    __syncthreads();\n";
    ss << "    if (lane == 0) sm[warp] = v;\n";
    ss << "    __syncthreads();\n";
    ss << "    if (warp == 0) {\n";
    ss << "        v = lane < " << (kThreads / 32) << " ? sm[lane] : " << identity << ";\n";
    ss << "#pragma unroll\n";
    ss << "        for (int m = 16; m >= 1; m >>= 1) { const " << ctype << " o = bh_shfl_xor(v, m); v = "
       << reduce_expr(op, "v", "o") << "; }\n";
    ss << "    }\n";
    ss << "    return v;\n}\n";
    return ss.str();
}

// Block reduction of K values per thread for several reductions at once: every reduction gets
// the tree of bh_block_reduce_k, but all share one pair of barriers (each has its own region of
// `sm`, at `offsets` bytes).
string block_reduce_all_fn(const vector<string> &ctypes, const vector<bh_opcode> &ops, const vector<string> &idents,
                           const vector<int64_t> &offsets, int K) {
    stringstream ss;
    ss << "__device__ __forceinline__ void bh_block_reduce_all(";
    for (size_t r = 0; r < ctypes.size(); ++r) ss << ctypes[r] << " (&v" << r << ")[" << K << "], ";
    ss << "unsigned char *sm) {\n";
    for (size_t r = 0; r < ctypes.size(); ++r)
        ss << "    " << ctypes[r] << " *s" << r << " = (" << ctypes[r] << " *)(sm + " << offsets[r] << ");\n";
    ss << "#pragma unroll\n";
    ss << "    for (int k = 0; k < " << K << "; ++k) {\n";
    for (size_t r = 0; r < ctypes.size(); ++r) {
        ss << "#pragma unroll\n";
        ss << "        for (int m = 16; m >= 1; m >>= 1) { const " << ctypes[r] << " o = bh_shfl_xor(v" << r << "[k], m); v"
           << r << "[k] = " << reduce_expr(ops[r], "v" + to_string(r) + "[k]", "o") << "; }\n";
    }
    ss << "    }\n";
    ss << "    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;\n";
    ss << "    __syncthreads();\n";
    ss << "    if (lane == 0) {\n";
    ss << "#pragma unroll\n";
    ss << "        for (int k = 0; k < " << K << "; ++k) {\n";
    for (size_t r = 0; r < ctypes.size(); ++r) ss << "            s" << r << "[warp * " << K << " + k] = v" << r << "[k];\n";
    ss << "        }\n";
    ss << "    }\n";
    ss << "    __syncthreads();\n";
    ss << "    if (warp == 0) {\n";
    ss << "#pragma unroll\n";
    ss << "        for (int k = 0; k < " << K << "; ++k) {\n";
    for (size_t r = 0; r < ctypes.size(); ++r) {
        ss << "            v" << r << "[k] = lane < " << (kThreads / 32) << " ? s" << r << "[lane * " << K << " + k] : "
           << idents[r] << ";\n";
        ss << "#pragma unroll\n";
        ss << "            for (int m = 16; m >= 1; m >>= 1) { const " << ctypes[r] << " o = bh_shfl_xor(v" << r
           << "[k], m); v" << r << "[k] = " << reduce_expr(ops[r], "v" + to_string(r) + "[k]", "o") << "; }\n";
    }
    ss << "        }\n";
    ss << "    }\n";
    ss << "}\n";
    return ss.str();
}

// GRID_REDUCE: `loop` is a 1-D innermost loop whose rank-0 sweeps are reductions to scalars.
// `identities` are the kernel-level identity instructions of those reductions (folded). Work item
// = one tile of kReduceTile elements; the CTA that completes the last tile of a unit folds the
// unit's tile partials in tile order and writes the results.
// Tiles per GRID_REDUCE work item: with many tiles a CTA takes K consecutive tiles at once so that
// K x 8 loads per thread are in flight together. Every tile keeps its own partial, reduced in the
// same order, so the result does not depend on K; K only depends on the tile count.
// The element body of GRID_REDUCE's full tiles written for two elements at once: every line
// (one statement or declaration per instruction) is followed by its copy for the next element, with
// temporaries t<N> renamed t<N>_1, the index i0 renamed i0_1 and preloaded slots [k * 8 + j] moved
// to [k * 8 + j + 1]. Accumulator updates keep their order: element j's before element j + 1's.
string interleave_second_element(const string &block) {
    static const regex tmp("\\bt([0-9]+)\\b"), idx("\\bi0\\b");
    const string slot = "[k * " + to_string(kReduceV) + " + j]", slot1 = "[k * " + to_string(kReduceV) + " + j + 1]";
    stringstream in(block), out;
    string line;
    while (getline(in, line)) {
        string second = regex_replace(regex_replace(line, tmp, "t$1_1"), idx, "i0_1");
        for (size_t at = second.find(slot); at != string::npos; at = second.find(slot, at + slot1.size()))
            second.replace(at, slot.size(), slot1);
        out << line << "\n" << second << "\n";
    }
    return out.str();
}

int grid_tiles_per_item(int64_t ntiles, const LoopB &L) {
    // Only light element code is memory-latency bound; a heavy body (many instructions, float64
    // math) is compute bound and would only lose occupancy to the extra registers.
    int n = 0, heavy = 0;
    for (const InstrPtr &i : jitk::all_instr(L)) {
        ++n;
        const bh_opcode op = i->opcode;
        const bool f64 = !i->operand.empty() && !i->operand[0].isConstant() &&
                         i->operand[0].base->dtype() == bh_type::FLOAT64;
        if (f64 && (op == BH_DIVIDE || op == BH_EXP || op == BH_LOG || op == BH_SQRT || op == BH_POWER ||
                    op == BH_SIN || op == BH_COS || op == BH_TANH))
            ++heavy;
    }
    if (n > 24 || heavy > 0) return 1;
    const int64_t resident = 148 * 4;
    if (ntiles >= 4 * 4 * resident) return 4;
    if (ntiles >= 2 * 2 * resident) return 2;
    return 1;
}

// Tiles per work item in a grouped launch: small light kernels (at most 64 tiles) take 4, so that
// in a launch of many small arrays through the same kernel every work item keeps 4 tiles of loads
// in flight and pays one block reduction and one counter update for the 4. Launched alone they
// keep 1 tile per item (more CTAs: a launch of a few tiles is latency-bound).
int grid_tiles_per_item_grouped(int64_t ntiles, const LoopB &L) {
    const int plain = grid_tiles_per_item(ntiles, L);
    if (plain == 1 && ntiles <= 64 && grid_tiles_per_item(int64_t{1} << 40, L) == 4) return 4;
    return plain;
}

// Block reduction of K values per thread at once (one shared-memory round for all K): the same
// tree as bh_block_reduce for every k.
string block_reduce_k_fn(const string &ctype, const string &fname, bh_opcode op, const string &identity, int K) {
    stringstream ss;
    ss << "__device__ __forceinline__ void " << fname << "(" << ctype << " (&v)[" << K << "], " << ctype << " *sm) {\n";
    ss << "#pragma unroll\n";
    ss << "    for (int k = 0; k < " << K << "; ++k) {\n";
    ss << "#pragma unroll\n";
    ss << "        for (int m = 16; m >= 1; m >>= 1) { const " << ctype << " o = bh_shfl_xor(v[k], m); v[k] = "
       << reduce_expr(op, "v[k]", "o") << "; }\n";
    ss << "    }\n";
    ss << "    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;\n";
    ss << "    __syncthreads();\n";
    ss << "    if (lane == 0) {\n";
    ss << "#pragma unroll\n";
    ss << "        for (int k = 0; k < " << K << "; ++k) sm[warp * " << K << " + k] = v[k];\n";
    ss << "    }\n";
    ss << "    __syncthreads();\n";
    ss << "    if (warp == 0) {\n";
    ss << "#pragma unroll\n";
    ss << "        for (int k = 0; k < " << K << "; ++k) {\n";
    ss << "            v[k] = lane < " << (kThreads / 32) << " ? sm[lane * " << K << " + k] : " << identity << ";\n";
    ss << "#pragma unroll\n";
    ss << "            for (int m = 16; m >= 1; m >>= 1) { const " << ctype << " o = bh_shfl_xor(v[k], m); v[k] = "
       << reduce_expr(op, "v[k]", "o") << "; }\n";
    ss << "        }\n";
    ss << "    }\n";
    ss << "}\n";
    return ss.str();
}

LaunchUnit lower_grid_reduce(const LoopB &loop, const vector<InstrPtr> &identities, const CodegenOptions &opt,
                             int forceK = 0) {
    LaunchUnit u;
    u.sched = Sched::GRID_REDUCE;
    u.V = kReduceV;
    const Block holder(loop);
    set<const bh_instruction *> folded;
    for (const InstrPtr &i : identities) folded.insert(i.get());
    Symbols sym = build_symbols({&holder}, folded);
    const LoopB &L = holder.getLoop();
    vector<InstrPtr> reds(L._sweeps.begin(), L._sweeps.end());
    sort(reds.begin(), reds.end(), [](const InstrPtr &a, const InstrPtr &b) { return a->origin_id < b->origin_id; });
    u.nred = static_cast<int>(reds.size());
    u.cols = L.size;
    const int64_t ntiles = (L.size + kReduceTile - 1) / kReduceTile;
    // Tiles per work item: Kp for plain launches, Kg for grouped ones. When they differ the unit's
    // source holds the device code twice, compiled for each (bh_work and bh_batch_work); results
    // do not depend on it (every tile keeps its own partial).
    const int Kp = grid_tiles_per_item(ntiles, L), Kg = grid_tiles_per_item_grouped(ntiles, L);
    if (forceK == 0 && Kp != Kg) {
        LaunchUnit up = lower_grid_reduce(loop, identities, opt, Kp);
        const LaunchUnit ug = lower_grid_reduce(loop, identities, opt, Kg);
        if (up.body_core.empty() || ug.body_core.empty()) throw runtime_error("lower_grid_reduce(): no body core");
        stringstream both;
        both << "namespace bh_kp {\n" << up.body_core << "} // namespace bh_kp\n";
        both << "namespace bh_kg {\n" << ug.body_core << "} // namespace bh_kg\n";
        both << "__device__ __forceinline__ void bh_work(const P &p, bh_i64 w) { bh_kp::bh_work(p, w); }\n";
        both << "__device__ __forceinline__ void bh_batch_work(const P &p, bh_i64 w) { bh_kg::bh_work(p, w); }\n";
        if (up.tail_capable) both << "__device__ __forceinline__ void bh_tail(const P &p) { bh_kp::bh_tail(p); }\n";
        both << kMainWrapper << kKernels;
        LaunchUnit u2 = up;
        u2.batch_chunks = Kg;
        finish_source(u2, up.params_decl, both.str(), opt);
        return u2;
    }
    const int K = forceK > 0 ? forceK : Kp;
    const string KT = to_string(K);
    u.chunks = K;
    ParamLayout pl;
    add_common_fields(sym, pl, opt);
    pl.add(work_field(ntiles), "bh_i64", "ntiles");
    pl.add(work_field((ntiles + K - 1) / K), "bh_i64", "work");
    ParamField fs{ParamField::SCRATCH};
    pl.add(fs, "unsigned char*", "scratch");
    ParamField fc{ParamField::COUNTER};
    pl.add(fc, "unsigned int*", "counter");

    stringstream helpers, body;
    Emitter em(sym, body, opt);
    vector<string> ctypes, idents, accs;
    for (size_t k = 0; k < reds.size(); ++k) {
        const InstrPtr &r = reds[k];
        const bh_type t = r->operand[0].base->dtype();
        ctypes.push_back(cuda_type(t));
        idents.push_back(constant_literal(jitk::sweep_identity(r->opcode, t)));
        accs.push_back("tacc" + to_string(k));
        helpers << block_reduce_fn(ctypes[k], "bh_block_reduce" + to_string(k), r->opcode, idents[k]);
        helpers << block_reduce_k_fn(ctypes[k], "bh_block_reduce_k" + to_string(k), r->opcode, idents[k], K);
    }
    u.slot_bytes = red_slot_bytes(reds);
    u.scratch_bytes_per_tile = u.slot_bytes * static_cast<int64_t>(reds.size());
    for (const InstrPtr &r : reds) u.red_orders.emplace_back(r->origin_id, "tree:" + to_string(L.size));
    // Several reductions share the tile's block-reduction barriers (each keeps its own tree).
    int64_t sm_bytes = (kThreads / 32) * K * u.slot_bytes;
    if (reds.size() > 1) {
        vector<int64_t> offsets;
        vector<bh_opcode> ops;
        int64_t off = 0;
        for (const InstrPtr &r : reds) {
            offsets.push_back(off);
            ops.push_back(r->opcode);
            off += ((kThreads / 32) * K * bh_type_size(r->operand[0].base->dtype()) + 15) / 16 * 16;
        }
        sm_bytes = max(sm_bytes, off);
        helpers << block_reduce_all_fn(ctypes, ops, idents, offsets, K);
    }
    body << helpers.str();
    body << "__device__ void bh_work(const P &p, bh_i64 w) {\n";
    body << pointer_locals(sym);
    body << "    __shared__ alignas(16) unsigned long long sm_raw[" << (sm_bytes + 7) / 8 << "];\n";
    body << "    __shared__ bool am_last;\n";
    for (size_t k = 0; k < reds.size(); ++k)
        body << "    " << ctypes[k] << "* part" << k << " = (" << ctypes[k] << "*)(p.scratch + p.ntiles * "
             << u.slot_bytes * k << ");\n";
    for (size_t k = 0; k < reds.size(); ++k) {
        body << "    " << ctypes[k] << " " << accs[k] << "[" << K << "];\n";
        body << "#pragma unroll\n";
        body << "    for (int k = 0; k < " << K << "; ++k) " << accs[k] << "[k] = " << idents[k] << ";\n";
    }
    body << "    const bh_i64 tile0 = w * " << KT << ";\n";
    body << "    const int ktiles = (int)min((bh_i64)" << KT << ", p.ntiles - tile0);\n";
    // Full items (K full tiles) run without bounds checks, after loading the read-only inputs of
    // all K x 8 elements of the thread; the last item checks every index. Tile k accumulates into
    // slot k, elements j = 0..7 in order, in both paths.
    const string n0 = "p.n" + to_string(sym.loop_id.at(&L));
    const bool heavy = heavy_body(L);
    // Loading every element's inputs up front keeps K x 8 loads in flight. A heavy body pays for
    // them in registers (Black-Scholes: 80 and 3 CTAs per SM with them, 48 and 5 without) and is
    // still faster with them (0.174 vs 0.188 ms per 10M options on a B200), so `preload_heavy`
    // is on by default.
    const vector<bh_view> pre = heavy && !opt.preload_heavy ? vector<bh_view>{} : preloadable_views(L, L, sym);
    map<ViewKey, string> acc_k;
    for (size_t k = 0; k < reds.size(); ++k) acc_k[ViewKey(reds[k]->operand[0])] = accs[k] + "[k]";
    // Element j (0..7) of a thread's part of tile k: 4 consecutive elements at 4t and 4 at 1024 + 4t
    // of the tile, so a view with unit stride is two 4-element words per thread; the thread folds
    // them in that order, on every path.
    const string elem_index = "(tile0 + k) * " + to_string(kReduceTile) + " + (j >> 2) * " + to_string(kReduceTile / 2) +
                              " + threadIdx.x * 4 + (j & 3)";
    // Views moved as words on full tiles: read-only inputs and arrays written by the element code
    // with unit stride (see emit_flat_vector).
    const bool vectorized = opt.vector_access && !opt.bounds_check && !(heavy && opt.interleave == 2);
    vector<bool> vec_pre(pre.size());
    for (size_t v = 0; v < pre.size(); ++v) vec_pre[v] = vectorized && unit_stride_view(pre[v], 0, sym);
    vector<bh_view> wouts;
    if (vectorized) {
        map<const bh_base *, set<ViewKey>> touched;
        for (const InstrPtr &i : jitk::all_instr(L))
            for (const bh_view &v : i->operand)
                if (!v.isConstant()) touched[v.base].insert(ViewKey(v));
        set<ViewKey> seen;
        for (const InstrPtr &i : jitk::all_instr(L)) {
            const bh_opcode op = i->opcode;
            if (bh_opcode_is_system(op) || bh_opcode_is_sweep(op) || op == BH_GATHER || op == BH_SCATTER ||
                op == BH_COND_SCATTER || i->operand.empty())
                continue;
            const bh_view &v = i->operand[0];
            if (!unit_stride_view(v, 0, sym) || sym.always_array.count(v.base) || touched[v.base].size() != 1) continue;
            if (acc_k.count(ViewKey(v))) continue;
            if (seen.insert(ViewKey(v)).second) wouts.push_back(v);
        }
    }
    // Code pieces of the two paths. `k` is the (unrolled) tile index in the generated code.
    auto emit_vec_check = [&](Emitter &eb) {
        // Word alignment of every word-moved view: the same for every group of 4 elements of
        // every tile, since a tile and a half-tile are whole multiples of 16 bytes.
        body << "        bool vec = true;\n";
        body << "        {\n";
        body << "            const bh_i64 i0 = tile0 * " << kReduceTile << " + threadIdx.x * 4;\n";
        for (size_t v = 0; v < pre.size(); ++v) {
            if (!vec_pre[v]) continue;
            const int bytes = min(16, 4 * static_cast<int>(bh_type_size(pre[v].base->dtype())));
            body << "            vec = vec && (((unsigned long long)&" << eb.array_ref(pre[v]) << ") & " << bytes - 1
                 << "ull) == 0;\n";
        }
        for (const bh_view &v : wouts) {
            const int bytes = min(16, 4 * static_cast<int>(bh_type_size(v.base->dtype())));
            body << "            vec = vec && (((unsigned long long)&" << eb.array_ref(v) << ") & " << bytes - 1
                 << "ull) == 0;\n";
        }
        body << "        }\n";
    };
    auto emit_pl_decls = [&]() {
        for (size_t v = 0; v < pre.size(); ++v)
            body << "        " << cuda_type(pre[v].base->dtype()) << " pl" << v << "[" << K * kReduceV << "];\n";
    };
    // The read-only inputs of tile k's 8 elements per thread into pl*[k * 8 ...].
    auto emit_preload_tile = [&](Emitter &eb, int ind) {
        const string sp(static_cast<size_t>(ind), ' ');
        if (vectorized) {
            // Two words of 4 elements per view and tile: elements 4t..4t+3 and 1024+4t..1024+4t+3.
            body << "#pragma unroll\n";
            body << sp << "for (int g = 0; g < 2; ++g) {\n";
            body << sp << "    const bh_i64 i0 = (tile0 + k) * " << kReduceTile << " + g * " << kReduceTile / 2
                 << " + threadIdx.x * 4;\n";
            for (size_t v = 0; v < pre.size(); ++v) {
                const string dst = "&pl" + to_string(v) + "[k * " + to_string(kReduceV) + " + g * 4]";
                const int bytes = 4 * static_cast<int>(bh_type_size(pre[v].base->dtype()));
                if (vec_pre[v]) {
                    body << sp << "    if (vec) { " << word_copy(dst, "&" + eb.array_ref(pre[v]), bytes) << "} else {\n";
                } else {
                    body << sp << "    {\n";
                }
                body << "#pragma unroll\n";
                body << sp << "        for (int e = 0; e < 4; ++e) {\n";
                body << sp << "            const bh_i64 i0e = i0 + e;\n";
                body << sp << "            pl" << v << "[k * " << kReduceV << " + g * 4 + e] = "
                     << regex_replace(eb.array_ref(pre[v]), regex("\\bi0\\b"), "i0e") << ";\n";
                body << sp << "        }\n";
                body << sp << "    }\n";
            }
            body << sp << "}\n";
        } else {
            body << "#pragma unroll\n";
            body << sp << "for (int j = 0; j < " << kReduceV << "; ++j) {\n";
            body << sp << "    const bh_i64 i0 = " << elem_index << ";\n";
            for (size_t v = 0; v < pre.size(); ++v)
                body << sp << "    pl" << v << "[k * " << kReduceV << " + j] = " << eb.array_ref(pre[v]) << ";\n";
            body << sp << "}\n";
        }
    };
    // Tile k's 8 elements per thread without bounds checks (inputs from pl*, written words through
    // so*), then the written words.
    auto emit_full_tile = [&](Emitter &eb, Scope &scope, int ind) {
        const string sp(static_cast<size_t>(ind), ' ');
        if (vectorized)
            for (size_t m = 0; m < wouts.size(); ++m)
                body << sp << cuda_type(wouts[m].base->dtype()) << " so" << m << "[" << kReduceV << "];\n";
        body << "#pragma unroll\n";
        body << sp << "for (int j = 0; j < " << kReduceV << "; ++j) {\n";
        body << sp << "    const bh_i64 i0 = " << elem_index << ";\n";
        eb.write_body(L, scope, ind + 4);
        body << sp << "}\n";
        if (vectorized) {
            // The written arrays' words: 4 elements at 4t and 4 at 1024 + 4t.
            body << "#pragma unroll\n";
            body << sp << "for (int g = 0; g < 2; ++g) {\n";
            body << sp << "    const bh_i64 i0 = (tile0 + k) * " << kReduceTile << " + g * " << kReduceTile / 2
                 << " + threadIdx.x * 4;\n";
            for (size_t m = 0; m < wouts.size(); ++m) {
                const int bytes = 4 * static_cast<int>(bh_type_size(wouts[m].base->dtype()));
                body << sp << "    if (vec) { " << word_copy("&" + eb.array_ref(wouts[m]), "&so" + to_string(m) + "[g * 4]", bytes)
                     << "} else {\n";
                body << "#pragma unroll\n";
                body << sp << "        for (int e = 0; e < 4; ++e) {\n";
                body << sp << "            const bh_i64 i0e = i0 + e;\n";
                body << sp << "            " << regex_replace(eb.array_ref(wouts[m]), regex("\\bi0\\b"), "i0e")
                     << " = so" << m << "[g * 4 + e];\n";
                body << sp << "        }\n";
                body << sp << "    }\n";
            }
            body << sp << "}\n";
        }
    };
    auto full_tile_scope = [&](Scope &scope) {
        for (size_t v = 0; v < pre.size(); ++v)
            scope.repl[ViewKey(pre[v])] = "pl" + to_string(v) + "[k * " + to_string(kReduceV) + " + j]";
        if (vectorized)
            for (size_t m = 0; m < wouts.size(); ++m) scope.repl[ViewKey(wouts[m])] = "so" + to_string(m) + "[j]";
    };
    // Path 0: all K tiles of the item are full. Every input of all K x 8 elements of the thread is
    // loaded first, then the tiles are computed.
    {
        body << "    if ((tile0 + " << KT << ") * " << kReduceTile << " <= " << n0 << ") {\n";
        Scope scope;
        Emitter eb(sym, body, opt);
        eb.external_acc = acc_k;
        if (vectorized) emit_vec_check(eb);
        if (!pre.empty()) {
            emit_pl_decls();
            body << "#pragma unroll\n";
            body << "        for (int k = 0; k < " << K << "; ++k) {\n";
            emit_preload_tile(eb, 12);
            body << "        }\n";
        }
        full_tile_scope(scope);
        // k always runs to the constant K (unrolled), so the accumulator slots stay registers.
        body << "#pragma unroll\n";
        body << "        for (int k = 0; k < " << K << "; ++k) {\n";
        if (heavy && opt.interleave == 2) {
            // Two elements per step, statement by statement (elements j and j + 1; reductions
            // still fold j before j + 1): independent chains side by side for the scheduler.
            body << "#pragma unroll\n";
            body << "            for (int j = 0; j < " << kReduceV << "; j += 2) {\n";
            body << "                const bh_i64 i0 = " << elem_index << ";\n";
            body << "                const bh_i64 i0_1 = " << regex_replace(elem_index, regex("\\bj\\b"), "(j + 1)") << ";\n";
            stringstream one;
            Emitter e1(sym, one, opt);
            e1.external_acc = acc_k;
            e1.write_body(L, scope, 16);
            body << interleave_second_element(one.str());
            body << "            }\n";
        } else {
            emit_full_tile(eb, scope, 12);
        }
        body << "        }\n";
    }
    // Path 1: the last work item. Its full tiles (kfull of them) take the same code as path 0,
    // one tile at a time; the partial tile checks every index. Both fold elements j = 0..7 of
    // tile k into slot k in order, as path 0 does.
    {
        body << "    } else {\n";
        Emitter eb(sym, body, opt);
        eb.external_acc = acc_k;
        if (K > 1) {
            body << "        const bh_i64 nfull = " << n0 << " / " << kReduceTile << " - tile0;\n";
            body << "        const int kfull = (int)(nfull < 0 ? 0 : (nfull < ktiles ? nfull : ktiles));\n";
            if (vectorized) emit_vec_check(eb);
            if (!pre.empty()) emit_pl_decls();
        }
        body << "#pragma unroll\n";
        body << "        for (int k = 0; k < " << K << "; ++k) {\n";
        body << "            if (k >= ktiles) break;\n";
        int ind = 12;
        if (K > 1) {
            body << "            if (k < kfull) {\n";
            Scope fscope;
            full_tile_scope(fscope);
            if (!pre.empty()) emit_preload_tile(eb, 16);
            emit_full_tile(eb, fscope, 16);
            body << "                continue;\n";
            body << "            }\n";
        }
        Scope scope;
        body << string(static_cast<size_t>(ind), ' ') << "for (int j = 0; j < " << kReduceV << "; ++j) {\n";
        body << string(static_cast<size_t>(ind), ' ') << "    const bh_i64 i0 = " << elem_index << ";\n";
        body << string(static_cast<size_t>(ind), ' ') << "    if (i0 >= " << n0 << ") break;\n";
        eb.write_body(L, scope, ind + 4);
        body << string(static_cast<size_t>(ind), ' ') << "}\n";
        body << "        }\n";
    }
    body << "    }\n";
    if (reds.size() > 1) {
        body << "    bh_block_reduce_all(";
        for (size_t k = 0; k < reds.size(); ++k) body << accs[k] << ", ";
        body << "(unsigned char*)sm_raw);\n";
    } else {
        body << "    bh_block_reduce_k0(" << accs[0] << ", (" << ctypes[0] << "*)sm_raw);\n";
    }
    for (size_t k = 0; k < reds.size(); ++k) {
        body << "    if (threadIdx.x == 0) {\n";
        body << "#pragma unroll\n";
        body << "        for (int k = 0; k < " << K << "; ++k)\n";
        body << "            if (k < ktiles) part" << k << "[tile0 + k] = " << accs[k] << "[k];\n";
        body << "    }\n";
    }
    body << "    if (threadIdx.x == 0) {\n";
    body << "        am_last = bh_arrive_n((unsigned*)p.counter, (unsigned)ktiles) + (unsigned)ktiles == (unsigned)p.ntiles;\n";
    body << "    }\n";
    body << "    __syncthreads();\n";
    body << "    if (!am_last) return;\n";
    body << "    bh_acquire();\n";
    for (size_t k = 0; k < reds.size(); ++k) {
        const InstrPtr &r = reds[k];
        body << "    {\n";
        body << "        " << ctypes[k] << " acc = " << idents[k] << ";\n";
        body << "        for (bh_i64 t = threadIdx.x; t < p.ntiles; t += " << kThreads << ") {\n";
        body << "            const " << ctypes[k] << " x = bh_ldcg(part" << k << " + t);\n";
        body << "            acc = " << reduce_expr(r->opcode, "acc", "x") << ";\n";
        body << "        }\n";
        body << "        acc = bh_block_reduce" << k << "(acc, (" << ctypes[k] << "*)sm_raw);\n";
        if (!sym.temps.count(r->operand[0].base)) {
            body << "        if (threadIdx.x == 0) " << em.array_ref(r->operand[0]) << " = acc;\n";
        }
        body << "    }\n";
    }
    body << "    if (threadIdx.x == 0) *p.counter = 0u;\n";
    body << "}\n";
    // The whole reduction in one CTA, for another kernel's tail (fuse_tails): only for small
    // arrays and order-free reductions, where the fold order does not change the result.
    bool order_free = !opt.bounds_check && ntiles <= 4;
    for (const InstrPtr &r : reds) {
        const bh_type t = r->operand[0].base->dtype();
        const bool exact_arith = (r->opcode == BH_ADD_REDUCE || r->opcode == BH_MULTIPLY_REDUCE) &&
                                 (bh_type_is_integer(t) || t == bh_type::BOOL);
        const bool cmp_or_bits = r->opcode == BH_MAXIMUM_REDUCE || r->opcode == BH_MINIMUM_REDUCE ||
                                 r->opcode == BH_LOGICAL_AND_REDUCE || r->opcode == BH_LOGICAL_OR_REDUCE ||
                                 r->opcode == BH_LOGICAL_XOR_REDUCE || r->opcode == BH_BITWISE_AND_REDUCE ||
                                 r->opcode == BH_BITWISE_OR_REDUCE || r->opcode == BH_BITWISE_XOR_REDUCE;
        if (!(exact_arith || (cmp_or_bits && !bh_type_is_complex(t)))) order_free = false;
    }
    if (order_free) {
        u.tail_capable = true;
        body << "__device__ void bh_tail(const P &p) {\n";
        body << pointer_locals(sym);
        body << "    __shared__ alignas(16) unsigned long long tail_sm[" << (kThreads / 32) * 2 << "];\n";
        map<ViewKey, string> acc1;
        for (size_t k = 0; k < reds.size(); ++k) {
            body << "    " << ctypes[k] << " tacc" << k << " = " << idents[k] << ";\n";
            acc1[ViewKey(reds[k]->operand[0])] = "tacc" + to_string(k);
        }
        body << "#pragma unroll 4\n";
        body << "    for (bh_i64 i0 = threadIdx.x; i0 < " << n0 << "; i0 += " << kThreads << ") {\n";
        {
            Scope scope;
            Emitter et(sym, body, opt);
            et.external_acc = acc1;
            et.write_body(L, scope, 8);
        }
        body << "    }\n";
        for (size_t k = 0; k < reds.size(); ++k) {
            body << "    tacc" << k << " = bh_block_reduce" << k << "(tacc" << k << ", (" << ctypes[k] << "*)tail_sm);\n";
            if (!sym.temps.count(reds[k]->operand[0].base))
                body << "    if (threadIdx.x == 0) " << em.array_ref(reds[k]->operand[0]) << " = tacc" << k << ";\n";
        }
        body << "}\n";
    }
    body << kWrappers;
    u.fields = pl.fields;
    u.algorithmic_bytes = unit_bytes(sym, vector<const Block *>{&holder});
    u.elements = L.size;
    finish_source(u, pl.decl.str(), body.str(), opt);
    return u;
}

// ------------------------------------------------------------------------------------- SCAN1D
// A 1-D innermost loop with one accumulate (cumulative sum/product) among elementwise
// instructions. Three launch units, in a fixed order that depends on the length only:
//   A  per chunk of 2048 elements: the accumulate's inputs are computed on the fly at coalesced
//      positions and staged in shared memory; thread t folds elements 8t..8t+7 of the chunk in
//      order from there, and a fixed block scan of the 256 thread totals gives the chunk total;
//   B  per group of 2048 chunk totals: the same per-thread fold and block scan -> each chunk's
//      exclusive prefix within its group, and the group total; the CTA that finishes last folds
//      the group totals in order -> the carry into every group. A chunk's carry is its group's
//      carry op its prefix within the group;
//   C  per chunk: the same staging, per-thread fold and block scan; element value = carry op
//      (exclusive thread prefix op running thread prefix), staged again and written out at
//      coalesced positions, where the instructions after the accumulate run on it.
// The fold order is the same whatever the staging, so results depend on the length only.
constexpr int kScanPerThread = 8;
constexpr int64_t kScanTile = kThreads * kScanPerThread;

bh_opcode scan_reduce_op(bh_opcode acc) { return acc == BH_MULTIPLY_ACCUMULATE ? BH_MULTIPLY_REDUCE : BH_ADD_REDUCE; }

// Deterministic block scan helper: returns the exclusive prefix of `v` over the CTA's threads in
// thread order and writes the CTA total to `total` (all threads).
string block_scan_fn(const string &T, const string &fname, bh_opcode op, const string &ident) {
    stringstream ss;
    ss << "__device__ __forceinline__ " << T << " " << fname << "(" << T << " v, " << T << " &total, " << T
       << " *sm) {\n";
    ss << "    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;\n";
    ss << "    " << T << " x = v;\n";
    ss << "#pragma unroll\n";
    ss << "    for (int d = 1; d < 32; d <<= 1) {\n";
    ss << "        " << T << " y = x;\n";
    ss << "        y = bh_shfl_up(y, d);\n";
    ss << "        if (lane >= d) x = " << reduce_expr(op, "y", "x") << ";\n";
    ss << "    }\n";
    ss << "    " << T << " ex = x;\n";
    ss << "    ex = bh_shfl_up(ex, 1);\n";
    ss << "    if (lane == 0) ex = " << ident << ";\n";
    ss << "    __syncthreads();\n";
    ss << "    if (lane == 31) sm[warp] = x;\n";
    ss << "    __syncthreads();\n";
    ss << "    if (threadIdx.x == 0) {\n";
    ss << "        " << T << " run = " << ident << ";\n";
    ss << "        for (int w = 0; w < " << kThreads / 32 << "; ++w) { const " << T << " t = sm[w]; sm[" << kThreads / 32
       << " + w] = run; run = " << reduce_expr(op, "run", "t") << "; }\n";
    ss << "        sm[" << 2 * (kThreads / 32) << "] = run;\n";
    ss << "    }\n";
    ss << "    __syncthreads();\n";
    ss << "    total = sm[" << 2 * (kThreads / 32) << "];\n";
    ss << "    const " << T << " wo = sm[" << kThreads / 32 << " + warp];\n";
    ss << "    return " << reduce_expr(op, "wo", "ex") << ";\n";
    ss << "}\n";
    return ss.str();
}

// True when `loop` can be lowered as SCAN1D; `acc` receives the accumulate.
bool scan1d_applicable(const LoopB &loop, InstrPtr &acc) {
    if (loop.rank != 0 || !loop.isInnermost() || loop._sweeps.size() != 1) return false;
    acc = *loop._sweeps.begin();
    if (acc->opcode != BH_ADD_ACCUMULATE && acc->opcode != BH_MULTIPLY_ACCUMULATE) return false;
    if (acc->operand[0].ndim != 1 || acc->operand[1].isConstant()) return false;
    for (const Block &b : loop._block_list) {
        if (!b.isInstr()) return false;
        const bh_opcode op = b.getInstr()->opcode;
        if (b.getInstr() == acc || bh_opcode_is_system(op)) continue;
        if (bh_opcode_is_sweep(op) || op == BH_GATHER || op == BH_SCATTER || op == BH_COND_SCATTER) return false;
    }
    // The accumulate's output is only read by instructions after it, at the same element.
    bool after = false;
    for (const Block &b : loop._block_list) {
        const InstrPtr &i = b.getInstr();
        if (i == acc) {
            after = true;
            continue;
        }
        for (size_t o = 1; o < i->operand.size(); ++o) {
            const bh_view &v = i->operand[o];
            if (v.isConstant() || v.base != acc->operand[0].base) continue;
            if (!after || !(v == acc->operand[0])) return false;
        }
        if (!i->operand.empty() && !i->operand[0].isConstant() && i->operand[0].base == acc->operand[0].base)
            return false;
    }
    return true;
}

vector<LaunchUnit> lower_scan1d(const LoopB &loop, const InstrPtr &acc, const CodegenOptions &opt) {
    const Block holder(loop);
    const LoopB &L = holder.getLoop();
    const int64_t n = L.size;
    const int64_t nchunks = (n + kScanTile - 1) / kScanTile;
    const int64_t ngroups = (nchunks + kScanTile - 1) / kScanTile;  // groups of chunk totals
    const bh_type t = acc->operand[0].base->dtype();
    const string T = cuda_type(t);
    const bh_opcode rop = scan_reduce_op(acc->opcode);
    const string ident = constant_literal(jitk::sweep_identity(rop, t));
    // Windowed (scan_windows, off by default): one group of chunks at a time, unit A then unit C,
    // so that the re-scan finds the group's inputs still in L2 (a group is 2048 chunks, 4M
    // elements: 32 MB of float64) and each input element crosses HBM once. On a B200 it measured
    // slower than the whole-length units (0.52 against 0.28 ms for 5e7 float64: two launches and
    // a group scan on every CTA's critical path per 32 MB window). Every CTA of the windowed unit C repeats
    // unit B's scan of its group's chunk totals (16 KB, read from L2) and takes its own chunk's
    // carry from it; the CTA of the group's first chunk stores the group's total and carry, which
    // the next group's launch reads. The operations and their association are those of the three
    // units, so the results are bit-identical.
    const bool windowed = opt.scan_windows;
    struct Step {
        int phase;
        int64_t first, work;  // first work item (chunk, or group for unit B) and item count
    };
    vector<Step> steps;
    if (windowed) {
        for (int64_t g = 0; g < ngroups; ++g) {
            const int64_t first = g * kScanTile, cnt = min<int64_t>(kScanTile, nchunks - first);
            steps.push_back({0, first, cnt});
            steps.push_back({2, first, cnt});
        }
    } else {
        steps = {{0, 0, nchunks}, {1, 0, ngroups}, {2, 0, nchunks}};
    }
    vector<LaunchUnit> units;
    for (const Step &st : steps) {
        const int phase = st.phase;
        LaunchUnit u;
        u.sched = Sched::SCAN1D;
        u.cols = n;
        u.chunks = st.work;  // work items
        Symbols sym = build_symbols({&holder}, {});
        ParamLayout pl;
        add_common_fields(sym, pl, opt);
        pl.add(work_field(nchunks), "bh_i64", "nchunks");
        pl.add(work_field(st.work), "bh_i64", "work");
        pl.add(work_field(st.first), "bh_i64", "first");
        ParamField fs{ParamField::SCRATCH};
        pl.add(fs, "unsigned char*", "scratch");
        if (phase == 1) {
            ParamField fc{ParamField::COUNTER};
            pl.add(fc, "unsigned int*", "counter");
            u.scan_gate = true;
        }
        // Prefetch (scan_prefetch): the streaming units read their unit-stride read-only inputs
        // from a two-slot shared-memory ring per CTA, each full chunk filled by TMA bulk copies
        // (one thread, one mbarrier per slot, bounded waits) while the CTA works on the chunk before.
        vector<bh_view> pfv;
        vector<int64_t> pf_off;
        int64_t pf_bytes = 0;
        if (phase != 1 && opt.scan_prefetch && !opt.bounds_check) {
            vector<bh_view> cand = preloadable_views(L, L, sym);
            const bh_view &in = acc->operand[1];
            bool in_written = false;
            for (const InstrPtr &i : jitk::all_instr(L))
                if (!i->operand.empty() && !i->operand[0].isConstant() && i->operand[0].base == in.base) in_written = true;
            if (!in.isConstant() && !sym.temps.count(in.base) && !in_written &&
                find_if(cand.begin(), cand.end(), [&](const bh_view &v) { return v == in; }) == cand.end())
                cand.push_back(in);
            for (const bh_view &v : cand) {
                if (!unit_stride_view(v, 0, sym)) continue;
                pfv.push_back(v);
                pf_off.push_back(pf_bytes);
                pf_bytes += 2 * kScanTile * static_cast<int64_t>(bh_type_size(v.base->dtype()));
            }
            if (pf_bytes > 64 * 1024) {
                pfv.clear();
                pf_off.clear();
                pf_bytes = 0;
            }
        }
        const bool pf = !pfv.empty();
        if (pf) {
            ParamField fok{ParamField::TMA_OK};  // bulk copies allowed (not in grouped launches)
            pl.add(fok, "bh_i64", "tma_ok");
            ParamField ferr{ParamField::SCRATCH};
            ferr.i64 = -1;  // the engine's error record
            pl.add(ferr, "unsigned long long*", "err");
        }
        stringstream body;
        Emitter em(sym, body, opt);
        body << block_scan_fn(T, "bh_block_scan", rop, ident);
        if (pf) {
            body << "// bh_dynamic_shared_bytes: " << pf_bytes << "\n";
            body << "__device__ void bh_work_x(const P &p, bh_i64 w, int slot, const unsigned char *ring) {\n";
        } else {
            body << "__device__ void bh_work(const P &p, bh_i64 w) {\n";
        }
        body << "    const bh_i64 c = p.first + w;\n";
        body << pointer_locals(sym);
        for (size_t k = 0; k < pfv.size(); ++k) {
            const string Tv = cuda_type(pfv[k].base->dtype());
            body << "    const " << Tv << "* rv" << k << " = (const " << Tv << "*)(ring + " << pf_off[k] << " + slot * "
                 << kScanTile * static_cast<int64_t>(bh_type_size(pfv[k].base->dtype())) << ");\n";
        }
        body << "    __shared__ " << T << " sm[" << 2 * (kThreads / 32) + 1 << "];\n";
        body << "    " << T << "* totals = (" << T << "*)p.scratch;\n";
        body << "    " << T << "* carries = totals + p.nchunks;\n";
        const string n0 = "p.n" + to_string(sym.loop_id.at(&L));
        // The accumulate's input at element i0 (computed by the instructions before it).
        auto emit_inputs = [&](Scope &scope, int ind) {
            for (const Block &b : L._block_list) {
                const InstrPtr &i = b.getInstr();
                if (i == acc) break;
                if (bh_opcode_is_system(i->opcode)) continue;
                em.write_instr(*i, scope, ind);
            }
        };
        auto declare_temps = [&](Scope &scope, int ind) {
            for (const bh_base *b : em.sorted_temps(L)) {
                if (sym.temps.count(b) && !scope.is_tmp(b)) {
                    scope.tmps.insert(b);
                    body << string(static_cast<size_t>(ind), ' ') << cuda_type(b->dtype()) << " t" << sym.base_index(b)
                         << ";\n";
                }
            }
        };
        if (phase == 1) {
            // Work item g scans chunk totals 2048g..2048g+2047 into carries local to the group
            // and stores the group total; the CTA that finishes last folds the group totals in
            // group order into the carry of every group.
            body << "    " << T << "* gtot = carries + p.nchunks;\n";
            body << "    " << T << "* grun = gtot + (p.nchunks + " << kScanTile - 1 << ") / " << kScanTile << ";\n";
            body << "    __shared__ bool am_last;\n";
            body << "    const bh_i64 base = c * " << kScanTile << ";\n";
            body << "    " << T << " v[" << kScanPerThread << "];\n";
            body << "    " << T << " s = " << ident << ";\n";
            body << "#pragma unroll\n";
            body << "    for (int k = 0; k < " << kScanPerThread << "; ++k) {\n";
            body << "        const bh_i64 j = base + threadIdx.x * " << kScanPerThread << " + k;\n";
            body << "        v[k] = s;\n";  // exclusive running prefix
            body << "        if (j < p.nchunks) { const " << T << " x = totals[j]; s = " << reduce_expr(rop, "s", "x")
                 << "; }\n";
            body << "    }\n";
            body << "    " << T << " total;\n";
            body << "    const " << T << " e = bh_block_scan(s, total, sm);\n";
            body << "#pragma unroll\n";
            body << "    for (int k = 0; k < " << kScanPerThread << "; ++k) {\n";
            body << "        const bh_i64 j = base + threadIdx.x * " << kScanPerThread << " + k;\n";
            body << "        if (j < p.nchunks) carries[j] = " << reduce_expr(rop, "e", "v[k]") << ";\n";
            body << "    }\n";
            body << "    if (threadIdx.x == 0) {\n";
            body << "        gtot[c] = total;\n";
            body << "        am_last = bh_arrive(p.counter) == (unsigned)(p.work - 1);\n";
            body << "    }\n";
            body << "    __syncthreads();\n";
            body << "    if (!am_last) return;\n";
            body << "    bh_acquire();\n";
            body << "    if (threadIdx.x == 0) {\n";
            body << "        " << T << " run = " << ident << ";\n";
            body << "        for (bh_i64 g = 0; g < p.work; ++g) {\n";
            body << "            grun[g] = run;\n";
            body << "            const " << T << " t = bh_ldcg(gtot + g);\n";
            body << "            run = " << reduce_expr(rop, "run", "t") << ";\n";
            body << "        }\n";
            body << "        *p.counter = 0u;\n";
            body << "    }\n";
            body << "}\n" << kWrappers;
        } else {
            // Pass 1: the accumulate's inputs, computed at coalesced positions (element k*256 + t
            // of the chunk in thread t) and staged in shared memory; stage slot of element q is
            // q + q/8, so the per-thread reads of 8 consecutive elements below hit distinct banks.
            body << "    __shared__ " << T << " stage[" << kScanTile + kScanTile / kScanPerThread << "];\n";
            body << "    const bh_i64 cbase = c * " << kScanTile << ";\n";
            auto stage_pass_one = [&](bool with_inputs, const string &what, bool from_ring) {
                Scope scope;
                if (from_ring)
                    for (size_t k = 0; k < pfv.size(); ++k) scope.repl[ViewKey(pfv[k])] = "rv" + to_string(k) + "[q]";
                body << "#pragma unroll\n";
                body << "    for (int k = 0; k < " << kScanPerThread << "; ++k) {\n";
                body << "        const int q = k * " << kThreads << " + (int)threadIdx.x;\n";
                body << "        const bh_i64 i0 = cbase + q;\n";
                if (what == "in") body << "        " << T << " x = " << ident << ";\n";
                body << "        if (i0 < " << n0 << ") {\n";
                declare_temps(scope, 12);
                if (with_inputs) emit_inputs(scope, 12);
                if (what == "in") {
                    body << "            x = " << em.name(acc->operand[1], scope) << ";\n";
                    body << "        }\n";
                    body << "        stage[q + (q >> 3)] = x;\n";
                    body << "    }\n";
                    return;
                }
                // Pass 2: the scanned values back at coalesced positions, then the instructions
                // after the accumulate.
                body << "            const " << T << " out = stage[q + (q >> 3)];\n";
                if (sym.temps.count(acc->operand[0].base)) {
                    body << "            t" << sym.base_index(acc->operand[0].base) << " = out;\n";
                } else {
                    body << "            " << em.array_ref(acc->operand[0]) << " = out;\n";
                    scope.repl[ViewKey(acc->operand[0])] = "out";
                }
                bool after = false;
                for (const Block &b : L._block_list) {
                    const InstrPtr &i = b.getInstr();
                    if (i == acc) {
                        after = true;
                        continue;
                    }
                    if (after && !bh_opcode_is_system(i->opcode)) em.write_instr(*i, scope, 12);
                }
                body << "        }\n";
                body << "    }\n";
            };
            // With the ring, a full chunk (slot >= 0) reads the prefetched inputs from it.
            auto stage_pass = [&](bool with_inputs, const string &what) {
                if (!pf) {
                    stage_pass_one(with_inputs, what, false);
                    return;
                }
                body << "    if (slot >= 0) {\n";
                stage_pass_one(with_inputs, what, true);
                body << "    } else {\n";
                stage_pass_one(with_inputs, what, false);
                body << "    }\n";
            };
            stage_pass(true, "in");
            body << "    __syncthreads();\n";
            // Thread t folds elements 8t..8t+7 of the chunk in order. The re-scan keeps them in
            // registers across the block scan: reading them back from the stage instead cut the
            // float64 re-scan from 64 to 48 registers but measured 4 % slower per flush.
            body << "    " << T << " s = " << ident << ";\n";
            body << "    " << T << " xs[" << kScanPerThread << "];\n";
            body << "#pragma unroll\n";
            body << "    for (int k = 0; k < " << kScanPerThread << "; ++k) {\n";
            body << "        const int q = (int)threadIdx.x * " << kScanPerThread << " + k;\n";
            body << "        xs[k] = stage[q + (q >> 3)];\n";
            body << "        if (cbase + q < " << n0 << ") s = " << reduce_expr(rop, "s", "xs[k]") << ";\n";
            body << "    }\n";
            // The block scan's first barrier orders these stage reads before any later stage write.
            body << "    " << T << " total;\n";
            body << "    const " << T << " e = bh_block_scan(s, total, sm);\n";
            // The kernel wrappers: with the ring, bh_main runs the prefetch walk.
            auto wrappers = [&]() -> string {
                if (!pf) return kWrappers;
                stringstream ws;
                ws << "__device__ __forceinline__ void bh_work(const P &p, bh_i64 w) { bh_work_x(p, w, -1, nullptr); }\n";
                ws << "__device__ __forceinline__ bool bh_pf_full(const P &p, bh_i64 w) { return (p.first + w + 1) * "
                   << kScanTile << " <= " << n0 << "; }\n";
                ws << "__device__ __forceinline__ bool bh_pf_ok(const P &p) {\n";
                ws << pointer_locals(sym);
                ws << "    const bh_i64 i0 = 0;\n";
                ws << "    bool ok = p.tma_ok != 0;\n";
                for (const bh_view &v : pfv) ws << "    ok = ok && (((unsigned long long)&" << em.array_ref(v) << ") & 15ull) == 0;\n";
                ws << "    return ok;\n";
                ws << "}\n";
                ws << "__device__ __forceinline__ void bh_pf_issue(const P &p, bh_i64 w, int slot, unsigned char *ring, "
                      "unsigned long long *bar) {\n";
                ws << pointer_locals(sym);
                int64_t chunk_bytes = 0;
                for (const bh_view &v : pfv) chunk_bytes += kScanTile * static_cast<int64_t>(bh_type_size(v.base->dtype()));
                ws << "    const bh_i64 i0 = (p.first + w) * " << kScanTile << ";\n";
                ws << "    bh_mbar_expect_tx(bar, " << chunk_bytes << "u);\n";
                for (size_t k = 0; k < pfv.size(); ++k) {
                    const int64_t vb = kScanTile * static_cast<int64_t>(bh_type_size(pfv[k].base->dtype()));
                    ws << "    bh_bulk_row(ring + " << pf_off[k] << " + slot * " << vb << ", &" << em.array_ref(pfv[k]) << ", "
                       << vb << "u, bar);\n";
                }
                ws << "}\n";
                ws << R"CUDA(__device__ void bh_main(const P &p) {
    extern __shared__ __align__(16) unsigned char bh_dyn[];
    if (!bh_pf_ok(p)) {
        for (bh_i64 w = blockIdx.x; w < p.work; w += gridDim.x) bh_work(p, w);
        return;
    }
    // Item i of this CTA is work item blockIdx.x + i * gridDim.x; its chunk (when full) is the
    // (i / 2)-th copy into slot i % 2.
    __shared__ alignas(8) unsigned long long pf_bar[2];
    __shared__ int pf_fail;
    if (threadIdx.x == 0) {
        bh_mbar_init(&pf_bar[0], 1u);
        bh_mbar_init(&pf_bar[1], 1u);
        bh_mbar_fence_init();
        pf_fail = 0;
    }
    __syncthreads();
    const bh_i64 step = gridDim.x;
    bh_i64 issued = 0, waited = 0;  // items [0, issued) copied, [0, waited) arrived (thread 0)
    if (threadIdx.x == 0) {
        for (; issued < 2; ++issued) {
            const bh_i64 w = blockIdx.x + issued * step;
            if (w >= p.work || !bh_pf_full(p, w)) break;
            bh_pf_issue(p, w, (int)issued, bh_dyn, &pf_bar[issued]);
        }
    }
    for (bh_i64 i = 0;; ++i) {
        const bh_i64 w = blockIdx.x + i * step;
        if (w >= p.work) break;
        const int slot = (int)(i & 1);
        const bool full = bh_pf_full(p, w);
        if (full) {
            if (!bh_mbar_wait(&pf_bar[slot], (unsigned)((i >> 1) & 1))) pf_fail = 1;
            else if (threadIdx.x == 0) waited = i + 1;
        }
        __syncthreads();
        if (pf_fail) break;
        bh_work_x(p, w, full ? slot : -1, bh_dyn);
        __syncthreads();  // every thread is done with the slot
        const bh_i64 wn = w + 2 * step;
        if (threadIdx.x == 0 && full && wn < p.work && bh_pf_full(p, wn)) {
            bh_pf_issue(p, wn, slot, bh_dyn, &pf_bar[slot]);
            issued = i + 3;
        }
    }
    if (pf_fail && threadIdx.x == 0) {
        // A chunk copy never completed: record it, and let the copies still in flight into the
        // ring land (bounded) before the CTA leaves.
        atomicCAS(p.err, 0ull, 0xC000000000000000ull | (unsigned long long)blockIdx.x);
        for (bh_i64 j = waited; j < issued; ++j) bh_mbar_wait(&pf_bar[j & 1], (unsigned)((j >> 1) & 1));
    }
}
)CUDA";
                ws << kBatchWork << kKernels;
                return ws.str();
            };
            if (phase == 0) {
                body << "    if (threadIdx.x == 0) totals[c] = total;\n";
                body << "}\n" << wrappers();
            } else {
                if (!windowed) {
                    body << "    const " << T << "* grun = carries + p.nchunks + (p.nchunks + " << kScanTile - 1 << ") / "
                         << kScanTile << ";\n";
                    body << "    const " << T << " carry = " << reduce_expr(rop, "grun[c / " + to_string(kScanTile) + "]", "carries[c]")
                         << ";\n";
                } else {
                    // Unit B's steps for this chunk's group: thread t folds chunk totals 8t..8t+7 of
                    // the group (v: its exclusive running prefixes), a block scan of the thread sums,
                    // and the group's carry from the previous group's carry and total.
                    body << "    " << T << "* gtot = carries + p.nchunks;\n";
                    body << "    " << T << "* grun = gtot + (p.nchunks + " << kScanTile - 1 << ") / " << kScanTile << ";\n";
                    body << "    __shared__ " << T << " chunk_carry;\n";
                    body << "    const bh_i64 g = c / " << kScanTile << ", gbase = g * " << kScanTile << ";\n";
                    body << "    " << T << " gv[" << kScanPerThread << "];\n";
                    body << "    " << T << " gs = " << ident << ";\n";
                    body << "#pragma unroll\n";
                    body << "    for (int k = 0; k < " << kScanPerThread << "; ++k) {\n";
                    body << "        const bh_i64 j = gbase + threadIdx.x * " << kScanPerThread << " + k;\n";
                    body << "        gv[k] = gs;\n";
                    body << "        if (j < p.nchunks) { const " << T << " x = totals[j]; gs = " << reduce_expr(rop, "gs", "x")
                         << "; }\n";
                    body << "    }\n";
                    body << "    " << T << " gtotal;\n";
                    body << "    const " << T << " ge = bh_block_scan(gs, gtotal, sm);\n";
                    body << "    const " << T << " run = g == 0 ? " << ident << " : " << reduce_expr(rop, "grun[g - 1]", "gtot[g - 1]")
                         << ";\n";
                    body << "    {\n";
                    body << "        const int own = (int)(c - gbase);\n";
                    body << "        if ((int)threadIdx.x == own / " << kScanPerThread << ") {\n";
                    body << "            " << T << " v = gv[0];\n";
                    body << "#pragma unroll\n";
                    body << "            for (int k = 1; k < " << kScanPerThread << "; ++k) if (k == own % " << kScanPerThread
                         << ") v = gv[k];\n";
                    body << "            chunk_carry = " << reduce_expr(rop, "run", "(" + reduce_expr(rop, "ge", "v") + ")") << ";\n";
                    body << "        }\n";
                    body << "        if (c == gbase && threadIdx.x == 0) {\n";
                    body << "            gtot[g] = gtotal;\n";
                    body << "            grun[g] = run;\n";
                    body << "        }\n";
                    body << "    }\n";
                    body << "    __syncthreads();\n";
                    body << "    const " << T << " carry = chunk_carry;\n";
                }
                body << "    " << T << " r = " << ident << ";\n";
                body << "#pragma unroll\n";
                body << "    for (int k = 0; k < " << kScanPerThread << "; ++k) {\n";
                body << "        const int j = (int)threadIdx.x * " << kScanPerThread << " + k;\n";
                body << "        if (cbase + j < " << n0 << ") {\n";
                body << "            r = " << reduce_expr(rop, "r", "xs[k]") << ";\n";
                body << "            const " << T << " inner = " << reduce_expr(rop, "e", "r") << ";\n";
                body << "            stage[j + (j >> 3)] = " << reduce_expr(rop, "carry", "inner") << ";\n";
                body << "        }\n";
                body << "    }\n";
                body << "    __syncthreads();\n";
                // Instructions after the accumulate that read values computed before it get them
                // recomputed (same thread and element as in pass 1, so stores repeat their values).
                bool reread = false, after = false;
                for (const Block &b : L._block_list) {
                    const InstrPtr &i = b.getInstr();
                    if (i == acc) {
                        after = true;
                        continue;
                    }
                    if (!after || bh_opcode_is_system(i->opcode)) continue;
                    for (size_t o = 1; o < i->operand.size(); ++o) {
                        const bh_view &v = i->operand[o];
                        if (!v.isConstant() && v.base != acc->operand[0].base) reread = true;
                    }
                }
                stage_pass(reread, "out");
                // Stage reads of this work item before the next item's pass 1 writes.
                body << "    __syncthreads();\n";
                body << "}\n" << wrappers();
            }
        }
        u.fields = pl.fields;
        u.scratch_bytes_per_tile = 0;
        // chunk totals, chunk carries, group totals, group carries
        u.scan_bytes = 2 * (nchunks + ngroups) * static_cast<int64_t>(bh_type_size(t));
        // The whole scan's bytes go to its last unit; a window's units share them by elements.
        const int64_t all_bytes = phase == 2 ? unit_bytes(sym, vector<const Block *>{&holder}) : 0;
        const int64_t elems = phase == 1 ? st.work : min<int64_t>(n, (st.first + st.work) * kScanTile) - st.first * kScanTile;
        u.algorithmic_bytes = windowed ? static_cast<int64_t>(static_cast<double>(all_bytes) * elems / max<int64_t>(n, 1))
                                       : all_bytes;
        u.elements = elems;
        if (phase == 2) u.red_orders.emplace_back(acc->origin_id, "scan:" + to_string(kScanTile) + ":" + to_string(n));
        finish_source(u, pl.decl.str(), body.str(), opt);
        units.push_back(std::move(u));
    }
    return units;
}

// SCAN1D in one pass (single_pass): every CTA takes chunks by ticket (an atomic counter, so all
// lower chunks belong to CTAs that are already running), stages and folds its chunk as unit A
// does, publishes the chunk total behind a release flag, and then looks back with warp 0. In unit
// B's scan of the chunk totals, chunk c is entry k of thread t (lane l of warp w) of group g; the
// chunk that closes a thread (k = 7) publishes the thread's sum, the one that closes a warp
// (k = 7, l = 31) the warp's total from the same 32-lane shuffle scan, and the one that closes a
// group the carry into the next group. Chunk c waits for at most 7 chunk totals, 31 thread sums,
// 7 warp totals and its group's carry, and combines them with unit B's and C's operations in
// their order, so the result is bit-identical to the three units while each element is read from
// memory once.
// Waits poll a bounded number of times (`p.spin_cap`; negative: none); when one runs out, or
// another CTA gave up, the chunk is abandoned and an abort flag raised. The CTA that leaves last
// then recomputes the whole scan alone with the three units' steps, and resets the flags and
// counters for the next launch.
LaunchUnit lower_scan1d_single(const LoopB &loop, const InstrPtr &acc, const CodegenOptions &opt) {
    const Block holder(loop);
    const LoopB &L = holder.getLoop();
    const int64_t n = L.size;
    const int64_t nchunks = (n + kScanTile - 1) / kScanTile;
    const int64_t ngroups = (nchunks + kScanTile - 1) / kScanTile;
    const bh_type t = acc->operand[0].base->dtype();
    const string T = cuda_type(t);
    const bh_opcode rop = scan_reduce_op(acc->opcode);
    const string ident = constant_literal(jitk::sweep_identity(rop, t));
    // Parenthesised: nested uses must keep their association (a op (b op c) is not (a op b) op c).
    auto op = [&](const string &a, const string &b) { return "(" + reduce_expr(rop, a, b) + ")"; };
    LaunchUnit u;
    u.sched = Sched::SCAN1D;
    u.single_pass = true;
    u.no_batch = true;
    u.cols = n;
    u.chunks = nchunks;
    Symbols sym = build_symbols({&holder}, {});
    ParamLayout pl;
    add_common_fields(sym, pl, opt);
    pl.add(work_field(nchunks), "bh_i64", "nchunks");
    pl.add(work_field(ngroups), "bh_i64", "ngroups");
    pl.add(work_field(nchunks), "bh_i64", "work");
    ParamField cap{ParamField::I64};
    cap.i64 = opt.scan_spin_cap;
    pl.add(cap, "bh_i64", "spin_cap");
    ParamField fs{ParamField::SCRATCH};
    pl.add(fs, "unsigned char*", "scratch");
    ParamField fc{ParamField::COUNTER};
    pl.add(fc, "unsigned int*", "counter");
    stringstream body;
    Emitter em(sym, body, opt);
    body << block_scan_fn(T, "bh_block_scan", rop, ident);
    body << R"CUDA(__device__ __forceinline__ unsigned bh_ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void bh_st_release(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}
// Poll *flag until it is set: false when `cap` polls ran out (at once for a negative cap) or
// another CTA raised the abort flag.
__device__ __forceinline__ bool bh_await(const unsigned *flag, const unsigned *abort_flag, long long cap) {
    long long spins = 0;
    while (bh_ld_acquire(flag) == 0u) {
        if (cap < 0 || ++spins > cap || bh_ld_acquire(abort_flag) != 0u) return false;
        __nanosleep(32);  // fewer polls of L2 while the producer works
    }
    return true;
}
)CUDA";
    const string n0 = "p.n" + to_string(sym.loop_id.at(&L));
    auto emit_inputs = [&](Scope &scope, int ind) {
        for (const Block &b : L._block_list) {
            const InstrPtr &i = b.getInstr();
            if (i == acc) break;
            if (bh_opcode_is_system(i->opcode)) continue;
            em.write_instr(*i, scope, ind);
        }
    };
    auto declare_temps = [&](Scope &scope, int ind) {
        for (const bh_base *b : em.sorted_temps(L)) {
            if (sym.temps.count(b) && !scope.is_tmp(b)) {
                scope.tmps.insert(b);
                body << string(static_cast<size_t>(ind), ' ') << cuda_type(b->dtype()) << " t" << sym.base_index(b) << ";\n";
            }
        }
    };
    bool reread = false;
    {
        bool after = false;
        for (const Block &b : L._block_list) {
            const InstrPtr &i = b.getInstr();
            if (i == acc) {
                after = true;
                continue;
            }
            if (!after || bh_opcode_is_system(i->opcode)) continue;
            for (size_t o = 1; o < i->operand.size(); ++o) {
                const bh_view &v = i->operand[o];
                if (!v.isConstant() && v.base != acc->operand[0].base) reread = true;
            }
        }
    }
    // Chunk c's accumulate inputs, computed at coalesced positions and staged (as unit A).
    body << "__device__ __forceinline__ void bh_stage_in(const P &p, bh_i64 c, " << T << " *stage) {\n";
    body << pointer_locals(sym);
    body << "    const bh_i64 cbase = c * " << kScanTile << ";\n";
    {
        Scope scope;
        body << "#pragma unroll\n";
        body << "    for (int k = 0; k < " << kScanPerThread << "; ++k) {\n";
        body << "        const int q = k * " << kThreads << " + (int)threadIdx.x;\n";
        body << "        const bh_i64 i0 = cbase + q;\n";
        body << "        " << T << " x = " << ident << ";\n";
        body << "        if (i0 < " << n0 << ") {\n";
        declare_temps(scope, 12);
        emit_inputs(scope, 12);
        body << "            x = " << em.name(acc->operand[1], scope) << ";\n";
        body << "        }\n";
        body << "        stage[q + (q >> 3)] = x;\n";
        body << "    }\n";
    }
    body << "}\n";
    // Chunk c's scanned values from the stage to memory, then the instructions after the
    // accumulate (as unit C).
    body << "__device__ __forceinline__ void bh_stage_out(const P &p, bh_i64 c, const " << T << " *stage) {\n";
    body << pointer_locals(sym);
    body << "    const bh_i64 cbase = c * " << kScanTile << ";\n";
    {
        Scope scope;
        body << "#pragma unroll\n";
        body << "    for (int k = 0; k < " << kScanPerThread << "; ++k) {\n";
        body << "        const int q = k * " << kThreads << " + (int)threadIdx.x;\n";
        body << "        const bh_i64 i0 = cbase + q;\n";
        body << "        if (i0 < " << n0 << ") {\n";
        declare_temps(scope, 12);
        if (reread) emit_inputs(scope, 12);
        body << "            const " << T << " out = stage[q + (q >> 3)];\n";
        if (sym.temps.count(acc->operand[0].base)) {
            body << "            t" << sym.base_index(acc->operand[0].base) << " = out;\n";
        } else {
            body << "            " << em.array_ref(acc->operand[0]) << " = out;\n";
            scope.repl[ViewKey(acc->operand[0])] = "out";
        }
        bool after = false;
        for (const Block &b : L._block_list) {
            const InstrPtr &i = b.getInstr();
            if (i == acc) {
                after = true;
                continue;
            }
            if (after && !bh_opcode_is_system(i->opcode)) em.write_instr(*i, scope, 12);
        }
        body << "        }\n";
        body << "    }\n";
    }
    body << "}\n";
    // Thread t's fold of elements 8t..8t+7 (kept in xs) and the chunk's block scan (unit A/C).
    body << "__device__ __forceinline__ " << T << " bh_chunk_fold(const P &p, bh_i64 c, const " << T << " *stage, " << T
         << " (&xs)[" << kScanPerThread << "], " << T << " &total, " << T << " *sm) {\n";
    body << "    const bh_i64 cbase = c * " << kScanTile << ";\n";
    body << "    " << T << " s = " << ident << ";\n";
    body << "#pragma unroll\n";
    body << "    for (int k = 0; k < " << kScanPerThread << "; ++k) {\n";
    body << "        const int q = (int)threadIdx.x * " << kScanPerThread << " + k;\n";
    body << "        xs[k] = stage[q + (q >> 3)];\n";
    body << "        if (cbase + q < " << n0 << ") s = " << op("s", "xs[k]") << ";\n";
    body << "    }\n";
    body << "    return bh_block_scan(s, total, sm);\n";
    body << "}\n";
    // The carried values of chunk c into the stage (unit C).
    body << "__device__ __forceinline__ void bh_chunk_rescan(const P &p, bh_i64 c, " << T << " *stage, const " << T
         << " (&xs)[" << kScanPerThread << "], " << T << " e, " << T << " carry) {\n";
    body << "    const bh_i64 cbase = c * " << kScanTile << ";\n";
    body << "    " << T << " r = " << ident << ";\n";
    body << "#pragma unroll\n";
    body << "    for (int k = 0; k < " << kScanPerThread << "; ++k) {\n";
    body << "        const int j = (int)threadIdx.x * " << kScanPerThread << " + k;\n";
    body << "        if (cbase + j < " << n0 << ") {\n";
    body << "            r = " << op("r", "xs[k]") << ";\n";
    body << "            const " << T << " inner = " << op("e", "r") << ";\n";
    body << "            stage[j + (j >> 3)] = " << op("carry", "inner") << ";\n";
    body << "        }\n";
    body << "    }\n";
    body << "}\n";
    body << "__device__ void bh_work(const P &p, bh_i64 w) {}\n";  // never launched grouped
    body << "__device__ __forceinline__ void bh_main(const P &p) {\n";
    body << "    __shared__ " << T << " stage[" << kScanTile + kScanTile / kScanPerThread << "];\n";
    body << "    __shared__ " << T << " sm[" << 2 * (kThreads / 32) + 1 << "];\n";
    body << "    __shared__ " << T << " bcast;\n";
    body << "    __shared__ bh_i64 ticket;\n";
    body << "    __shared__ bool last;\n";
    // Published values (scan arena) and their flags (counters): chunk totals; thread sums (the fold
    // of 8 consecutive chunk totals, unit B's per-thread step); warp totals (unit B's shuffle scan
    // over 32 thread sums); group carries.
    body << "    const bh_i64 nthr = (p.nchunks + 7) / 8, nwarp = (p.nchunks + 255) / 256;\n";
    body << "    " << T << "* totals = (" << T << "*)p.scratch;\n";
    body << "    " << T << "* carries = totals + p.nchunks;\n";
    body << "    " << T << "* tsum = carries + p.nchunks;\n";
    body << "    " << T << "* wtot = tsum + nthr;\n";
    body << "    " << T << "* gcarry = wtot + nwarp;\n";
    body << "    unsigned* flags = p.counter;\n";
    body << "    unsigned* sflags = flags + p.nchunks;\n";
    body << "    unsigned* wflags = sflags + nthr;\n";
    body << "    unsigned* gflags = wflags + nwarp;\n";
    body << "    unsigned* ctr = gflags + p.ngroups + 1;  // ticket, CTAs that left, abort\n";
    body << "    __shared__ " << T << " lb_carry;\n";
    body << "    __shared__ int lb_ok;\n";
    body << "    " << T << " xs[" << kScanPerThread << "];\n";
    body << R"CUDA(    for (;;) {
        if (threadIdx.x == 0) ticket = bh_ld_acquire(ctr + 2) != 0u ? p.nchunks : (bh_i64)atomicAdd(ctr, 1u);
        __syncthreads();
        const bh_i64 c = ticket;
        if (c >= p.nchunks) break;
        bh_stage_in(p, c, stage);
        __syncthreads();
)CUDA";
    body << "        " << T << " total;\n";
    body << "        const " << T << " e = bh_chunk_fold(p, c, stage, xs, total, sm);\n";
    body << R"CUDA(        if (threadIdx.x == 0) {
            totals[c] = total;
            bh_st_release(flags + c, 1u);
        }
        // Look back (warp 0; the other warps wait at the barrier below). Chunk c is entry k of
        // thread t = lane l of warp w of group g in unit B's scan of the chunk totals.
        if (threadIdx.x < 32) {
            const int lane = threadIdx.x;
            const bh_i64 g = c / )CUDA" << kScanTile << R"CUDA(;
            const int q = (int)(c - g * )CUDA" << kScanTile << R"CUDA();
            const int k = q & 7, t = q >> 3, l = t & 31, w = t >> 5;
            const bh_i64 tg = c >> 3, wg = c >> 8;  // global thread and warp of c
            bool ok = true;
)CUDA";
    // Each value is published as soon as its own inputs are in, before the waits it does not
    // depend on: a thread sum needs only its 8 chunk totals, a warp total only its 32 thread
    // sums, the next group's carry only this group's warp totals and carry.
    body << "            " << T << " x1 = " << ident << ", x2 = " << ident << ", x3 = " << ident << ";\n";
    body << R"CUDA(            if (lane < k) {  // totals of the entries before k in thread t
                ok = bh_await(flags + c - k + lane, ctr + 2, p.spin_cap);
                if (ok) x1 = bh_ldcg(totals + c - k + lane);
            }
            ok = __all_sync(0xffffffffu, ok);
)CUDA";
    // v: unit B's exclusive running fold in thread t before entry k; sT: the thread's sum
    body << "            " << T << " v = " << ident << ";\n";
    body << "            for (int i = 0; i < k; ++i) { const " << T << " y = bh_shfl_idx(x1, i); v = " << op("v", "y") << "; }\n";
    body << "            const " << T << " sT = " << op("v", "total") << ";\n";
    body << R"CUDA(            if (ok && k == 7 && lane == 0) {
                tsum[tg] = sT;
                bh_st_release(sflags + tg, 1u);
            }
            if (ok && lane < l) {  // thread sums of the lanes before l in warp w
                ok = bh_await(sflags + tg - l + lane, ctr + 2, p.spin_cap);
                if (ok) x2 = bh_ldcg(tsum + tg - l + lane);
            }
            ok = __all_sync(0xffffffffu, ok);
)CUDA";
    // unit B's shuffle scan within warp w (lanes after l do not change lanes up to l)
    body << "            " << T << " xk = lane < l ? x2 : (lane == l && k == 7 ? sT : " << ident << ");\n";
    body << "#pragma unroll\n";
    body << "            for (int d = 1; d < 32; d <<= 1) {\n";
    body << "                " << T << " y = bh_shfl_up(xk, d);\n";
    body << "                if (lane >= d) xk = " << op("y", "xk") << ";\n";
    body << "            }\n";
    body << "            const " << T << " exv = bh_shfl_idx(xk, l > 0 ? l - 1 : 0);\n";
    body << "            const " << T << " ex = l > 0 ? exv : " << ident << ";\n";
    body << "            const " << T << " wt = bh_shfl_idx(xk, 31);\n";
    body << R"CUDA(            if (ok && k == 7 && l == 31 && lane == 0) {
                wtot[wg] = wt;
                bh_st_release(wflags + wg, 1u);
            }
            if (ok && lane < w) {  // totals of the warps before w in group g
                ok = bh_await(wflags + wg - w + lane, ctr + 2, p.spin_cap);
                if (ok) x3 = bh_ldcg(wtot + wg - w + lane);
            }
            ok = __all_sync(0xffffffffu, ok);
)CUDA";
    // warp offsets: serial run over the warp totals before w (and the group total's first 7)
    body << "            " << T << " wo = " << ident << ";\n";
    body << "            " << T << " gt = " << ident << ";\n";
    body << "            for (int i = 0; i < 8; ++i) {\n";
    body << "                const " << T << " y = bh_shfl_idx(x3, i);\n";
    body << "                if (i < w) wo = " << op("wo", "y") << ";\n";
    body << "                if (i < 7) gt = " << op("gt", "y") << ";\n";
    body << "            }\n";
    body << "            if (ok && lane == 0 && g > 0) ok = bh_await(gflags + g, ctr + 2, p.spin_cap);\n";
    body << "            ok = __all_sync(0xffffffffu, ok);\n";
    body << "            if (ok && lane == 0) {\n";
    body << "                const " << T << " grun = g > 0 ? bh_ldcg(gcarry + g) : " << ident << ";\n";
    body << "                lb_carry = " << op("grun", op(op("wo", "ex"), "v")) << ";\n";
    body << "                if (q == " << kScanTile - 1 << " && g + 1 < p.ngroups) {\n";
    body << "                    gt = " << op("gt", "wt") << ";\n";
    body << "                    gcarry[g + 1] = " << op("grun", "gt") << ";\n";
    body << "                    bh_st_release(gflags + g + 1, 1u);\n";
    body << "                }\n";
    body << "            }\n";
    body << "            if (lane == 0) lb_ok = ok ? 1 : 0;\n";
    body << "        }\n";
    body << R"CUDA(        __syncthreads();
        if (!lb_ok) {
            if (threadIdx.x == 0) atomicExch(ctr + 2, 1u);
            break;
        }
        bh_chunk_rescan(p, c, stage, xs, e, lb_carry);
)CUDA";

    body << R"CUDA(        __syncthreads();
        bh_stage_out(p, c, stage);
        __syncthreads();  // stage reads before the next chunk's writes
    }
    // The CTA that leaves last: the fallback if any CTA gave up, then the reset for the next launch.
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(ctr + 1, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    bh_acquire();
    if (bh_ld_acquire(ctr + 2) != 0u) {
        for (bh_i64 c = 0; c < p.nchunks; ++c) {
            bh_stage_in(p, c, stage);
            __syncthreads();
)CUDA";
    body << "            " << T << " total;\n";
    body << "            bh_chunk_fold(p, c, stage, xs, total, sm);\n";
    body << "            if (threadIdx.x == 0) totals[c] = total;\n";
    body << "            __syncthreads();\n";
    body << "        }\n";
    body << "        __threadfence_block();\n";
    body << "        __syncthreads();\n";
    body << "        " << T << " run = " << ident << ";\n";
    body << "        for (bh_i64 g = 0; g < p.ngroups; ++g) {\n";
    // unit B's per-group step, for every chunk of the group at once
    body << "            const bh_i64 base = g * " << kScanTile << ";\n";
    body << "            " << T << " v[" << kScanPerThread << "];\n";
    body << "            " << T << " s = " << ident << ";\n";
    body << "            for (int k = 0; k < " << kScanPerThread << "; ++k) {\n";
    body << "                const bh_i64 j = base + threadIdx.x * " << kScanPerThread << " + k;\n";
    body << "                v[k] = s;\n";
    body << "                if (j < p.nchunks) { const " << T << " x = totals[j]; s = " << op("s", "x") << "; }\n";
    body << "            }\n";
    body << "            " << T << " gt;\n";
    body << "            const " << T << " e = bh_block_scan(s, gt, sm);\n";
    body << "            for (int k = 0; k < " << kScanPerThread << "; ++k) {\n";
    body << "                const bh_i64 j = base + threadIdx.x * " << kScanPerThread << " + k;\n";
    body << "                if (j < p.nchunks) carries[j] = " << op("run", op("e", "v[k]")) << ";\n";
    body << "            }\n";
    body << "            run = " << op("run", "gt") << ";\n";
    body << "            __syncthreads();\n";
    body << "        }\n";
    body << "        __threadfence_block();\n";
    body << "        __syncthreads();\n";
    body << "        for (bh_i64 c = 0; c < p.nchunks; ++c) {\n";
    body << "            bh_stage_in(p, c, stage);\n";
    body << "            __syncthreads();\n";
    body << "            " << T << " total;\n";
    body << "            const " << T << " e = bh_chunk_fold(p, c, stage, xs, total, sm);\n";
    body << "            bh_chunk_rescan(p, c, stage, xs, e, carries[c]);\n";
    body << "            __syncthreads();\n";
    body << "            bh_stage_out(p, c, stage);\n";
    body << "            __syncthreads();\n";
    body << "        }\n";
    body << "    }\n";
    body << R"CUDA(    for (bh_i64 i = threadIdx.x; i < p.nchunks + nthr + nwarp + p.ngroups + 1; i += blockDim.x) flags[i] = 0u;
    if (threadIdx.x == 0) {
        ctr[0] = 0u;
        ctr[1] = 0u;
        ctr[2] = 0u;
    }
}
)CUDA";
    body << kBatchWork << kKernels;
    u.fields = pl.fields;
    u.scan_bytes = (2 * nchunks + (nchunks + 7) / 8 + (nchunks + 255) / 256 + ngroups + 1) *
                   static_cast<int64_t>(bh_type_size(t));
    u.algorithmic_bytes = unit_bytes(sym, vector<const Block *>{&holder});
    u.elements = n;
    u.red_orders.emplace_back(acc->origin_id, "scan:" + to_string(kScanTile) + ":" + to_string(n));
    finish_source(u, pl.decl.str(), body.str(), opt);
    return u;
}

// OUTER_REDUCE: rank 0 sweeps (reductions) with a single parallel sub-nest and no instructions
// directly at rank 0. Threads own points of the sub-nest and loop over the reduced axis in order.
bool outer_reduce_applicable(const LoopB &L) {
    if (L._sweeps.empty()) return false;
    for (const InstrPtr &s : L._sweeps)
        if (!bh_opcode_is_reduction(s->opcode)) return false;
    if (!jitk::all_local_instr(L).empty()) return false;
    if (L._block_list.size() != 1 || L._block_list[0].isInstr()) return false;
    const LoopB &sub = L._block_list[0].getLoop();
    return jitk::parallel_ranks(sub, 64).first > 0;
}

LaunchUnit lower_outer_reduce(const LoopB &loop, const vector<const Block *> &identity_loops,
                              const CodegenOptions &opt) {
    LaunchUnit u;
    u.sched = Sched::OUTER_REDUCE;
    const Block holder(loop);
    set<const bh_instruction *> folded;
    for (const Block *b : identity_loops)
        for (const InstrPtr &i : jitk::all_instr(*b)) folded.insert(i.get());
    Symbols sym = build_symbols({&holder}, folded);
    const LoopB &L = holder.getLoop();
    const LoopB &sub = L._block_list[0].getLoop();
    const unsigned P = static_cast<unsigned>(jitk::parallel_ranks(sub, 64).first);
    const vector<const LoopB *> chain = jitk::get_first_loop_blocks(sub);
    const LoopB &inner = *chain[P - 1];
    int64_t rows = 1;
    for (unsigned r = 0; r + 1 < P; ++r) rows *= chain[r]->size;
    u.rows = rows;
    u.cols = inner.size;
    ParamLayout pl;
    add_common_fields(sym, pl, opt);
    pl.add(work_field(rows * inner.size), "bh_i64", "points");
    pl.add(work_field((rows * inner.size + kThreads - 1) / kThreads), "bh_i64", "work");
    vector<InstrPtr> reds(L._sweeps.begin(), L._sweeps.end());
    sort(reds.begin(), reds.end(), [](const InstrPtr &a, const InstrPtr &b) { return a->origin_id < b->origin_id; });

    stringstream body;
    Emitter em(sym, body, opt);
    body << "__device__ __forceinline__ void bh_work(const P &p, bh_i64 w) {\n";
    body << pointer_locals(sym);
    body << "    const bh_i64 pt = w * " << kThreads << " + threadIdx.x;\n";
    body << "    if (pt >= p.points) return;\n";
    body << "    bh_i64 rem = pt;\n";
    for (int r = static_cast<int>(P) - 1; r >= 0; --r) {
        const int rank = r + 1;
        const int lid = sym.loop_id.at(chain[r]);
        if (r == 0) {
            body << "    const bh_i64 i" << rank << " = rem;\n";
        } else {
            body << "    const bh_i64 i" << rank << " = rem % p.n" << lid << "; rem /= p.n" << lid << ";\n";
        }
    }
    Scope scope;
    for (size_t k = 0; k < reds.size(); ++k) {
        const bh_type t = reds[k]->operand[0].base->dtype();
        const string nm = "oacc" + to_string(k);
        body << "    " << cuda_type(t) << " " << nm << " = " << constant_literal(jitk::sweep_identity(reds[k]->opcode, t))
             << ";\n";
        em.external_acc[ViewKey(reds[k]->operand[0])] = nm;
    }
    declare_chain_temps(em, sym, scope, chain, P - 1, body, 4);
    body << "    for (bh_i64 i0 = 0; i0 < p.n" << sym.loop_id.at(&L) << "; ++i0) {\n";
    Scope s0;
    s0.parent = &scope;
    for (const bh_base *b : em.sorted_temps(L)) {
        if (sym.temps.count(b) && !s0.is_tmp(b)) {
            s0.tmps.insert(b);
            body << "        " << cuda_type(b->dtype()) << " t" << sym.base_index(b) << ";\n";
        }
    }
    em.write_body(inner, s0, 8);
    body << "    }\n";
    for (size_t k = 0; k < reds.size(); ++k) {
        if (sym.temps.count(reds[k]->operand[0].base)) continue;
        body << "    " << em.array_ref(reds[k]->operand[0], 0) << " = oacc" << k << ";\n";
    }
    body << "}\n" << kWrappers;
    u.fields = pl.fields;
    u.algorithmic_bytes = unit_bytes(sym, vector<const Block *>{&holder});
    u.elements = rows * inner.size * L.size;
    finish_source(u, pl.decl.str(), body.str(), opt);
    return u;
}

bool is_foldable_identity(const Block &b) {
    if (!b.isInstr()) return false;
    const bh_instruction &i = *b.getInstr();
    return i.opcode == BH_IDENTITY && i.operand.size() == 2 && i.operand[1].isConstant();
}

bool identity_loop(const Block &b) {
    if (b.isInstr()) return false;
    const auto instrs = jitk::all_instr(b);
    return instrs.size() == 1 && instrs[0]->opcode == BH_IDENTITY && instrs[0]->operand[1].isConstant();
}

// The wrappers of a unit with a folded tail (see fuse_tails): the CTA that arrives last on the
// completion counter runs the tail -- per launch, or per item of a grouped launch.
const char *kTailWrappers = R"CUDA(
struct P {
    bh_u1::P a;
    bh_u2::P b;
    alignas(8) unsigned int* tail_counter;
};
// Every thread's writes are made visible device-wide, thread 0 arrives with an acquire-release
// atomic, and the tail's threads acquire before reading.
__device__ __forceinline__ bool bh_tail_gate(unsigned int *counter, unsigned int arrivals) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = bh_arrive(counter) == arrivals - 1u;
    __syncthreads();
    const bool l = last;
    if (l) {
        bh_acquire();
        if (threadIdx.x == 0) *counter = 0u;
    }
    return l;
}
extern "C" __global__ void __launch_bounds__(256) __KERNEL_NAME__(const __grid_constant__ P p) {
    bh_grid_dependency();
    bh_u1::bh_main(p.a);
    if (bh_tail_gate(p.tail_counter, gridDim.x)) bh_u2::bh_tail(p.b);
}
extern "C" __global__ void __launch_bounds__(256) __KERNEL_NAME___batch(const P* __restrict__ items,
        const bh_i64* __restrict__ prefix, int nitems, bh_i64 total) {
    // As the plain grouped wrapper; each item's tail runs after the item's last work item.
    bh_grid_dependency();
    __shared__ P sp;
    bh_i64 have_lo = 0, have_hi = 0;
    const bh_i64 g_lo = (bh_i64)blockIdx.x * total / gridDim.x;
    const bh_i64 g_hi = ((bh_i64)blockIdx.x + 1) * total / gridDim.x;
    for (bh_i64 g = g_lo; g < g_hi; ++g) {
        if (g < have_lo || g >= have_hi) {
            int lo = 0, hi = nitems - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (prefix[mid] <= g) lo = mid; else hi = mid - 1;
            }
            __syncthreads();
            for (int k = threadIdx.x; k < (int)(sizeof(P) / 8); k += blockDim.x)
                ((unsigned long long*)&sp)[k] = ((const unsigned long long*)(items + lo))[k];
            __syncthreads();
            have_lo = prefix[lo];
            have_hi = prefix[lo + 1];
        }
        bh_u1::bh_batch_work(sp.a, g - have_lo);
        if (bh_tail_gate(sp.tail_counter, (unsigned int)(have_hi - have_lo))) bh_u2::bh_tail(sp.b);
    }
}
)CUDA";

LaunchUnit fuse_tail(const LaunchUnit &u1, const LaunchUnit &u2) {
    LaunchUnit u = u1;
    u.tail = true;
    for (const ParamField &f : u2.fields) u.fields.push_back(f);  // its counter and scratch stay unused
    ParamField gate{ParamField::COUNTER};
    gate.off = u1.counters_needed();
    u.fields.push_back(gate);
    u.algorithmic_bytes = u1.algorithmic_bytes + u2.algorithmic_bytes;
    u.elements = u1.elements + u2.elements;
    u.red_orders.insert(u.red_orders.end(), u2.red_orders.begin(), u2.red_orders.end());
    stringstream src;
    src << kPrelude;
    auto uses = [&](const char *name) {
        for (const LaunchUnit *x : {&u1, &u2})
            if (x->params_decl.find(name) != string::npos || x->body_core.find(name) != string::npos) return true;
        return false;
    };
    if (uses("bh_c64") || uses("bh_c128")) src << kComplexPrelude;
    if (uses("bh_tmap") || uses("bh_mbar")) src << kTmaPrelude;
    src << "namespace bh_u1 {\nstruct P {\n" << u1.params_decl << "};\n" << u1.body_core << "} // namespace bh_u1\n";
    src << "namespace bh_u2 {\nstruct P {\n" << u2.params_decl << "};\n" << u2.body_core << "} // namespace bh_u2\n";
    src << kTailWrappers;
    const string without_name = src.str();
    stringstream nm;
    nm << "bh_" << sched_name(u1.sched) << "_tail_" << hex << fnv1a(without_name);
    u.name = nm.str();
    string text = without_name;
    const string placeholder = "__KERNEL_NAME__";
    for (size_t pos = text.find(placeholder); pos != string::npos; pos = text.find(placeholder))
        text.replace(pos, placeholder.size(), u.name);
    u.source = text;
    u.params_decl.clear();
    u.body_core.clear();
    u.tail_capable = false;
    return u;
}

} // namespace

vector<LaunchUnit> lower_kernel(const LoopB &kernel, const CodegenOptions &opt) {
    vector<const Block *> items;
    for (const Block &b : kernel._block_list)
        if (!b.isSystemOnly()) items.push_back(&b);
    if (items.empty()) return {};

    vector<LaunchUnit> units;
    vector<InstrPtr> pending_identities;     // kernel-level scalar identities
    vector<const Block *> pending_id_loops;  // kernel-level identity loops
    bool serial = false;
    for (size_t idx = 0; idx < items.size() && !serial; ++idx) {
        const Block &b = *items[idx];
        if (b.isInstr()) {
            if (is_foldable_identity(b)) {
                pending_identities.push_back(b.getInstr());
                continue;
            }
            serial = true;
            break;
        }
        const LoopB &L = b.getLoop();
        if (identity_loop(b) && idx + 1 < items.size()) {
            pending_id_loops.push_back(&b);
            continue;
        }
        const unsigned P = static_cast<unsigned>(jitk::parallel_ranks(L, 64).first);
        if (P >= 1) {
            if (!pending_identities.empty()) {
                serial = true;
                break;
            }
            for (const Block *il : pending_id_loops) {
                const unsigned Pi = static_cast<unsigned>(jitk::parallel_ranks(il->getLoop(), 64).first);
                units.push_back(lower_flat(il->getLoop(), Pi, opt));
            }
            pending_id_loops.clear();
            const vector<const LoopB *> chain = jitk::get_first_loop_blocks(L);
            const LoopB *sub = split_candidate(*chain[P - 1]);
            int64_t points = 1;
            for (unsigned r = 0; r < P; ++r) points *= chain[r]->size;
            if (sub != nullptr && points >= kLaneMinPoints && lane_count(points, sub->size) > 1 &&
                swept_axis_contiguous(*sub, static_cast<int>(P))) {
                units.push_back(lower_lane_reduce(L, P, opt));
            } else if (sub != nullptr && split_chunks(points, sub->size) > 1) {
                units.push_back(lower_split_reduce(L, P, opt));
            } else {
                LaunchUnit tu;
                if (P == 2 && lower_tile2d(L, opt, tu)) {
                    units.push_back(std::move(tu));
                } else {
                    units.push_back(lower_flat(L, P, opt));
                }
            }
            continue;
        }
        InstrPtr scan_acc;
        if (scan1d_applicable(L, scan_acc) && pending_identities.empty()) {
            // Identity loops that only seed the accumulate's output are subsumed by the scan.
            bool ok = true;
            for (const Block *il : pending_id_loops) {
                const bh_view &v = jitk::all_instr(*il)[0]->operand[0];
                ok = ok && v.base == scan_acc->operand[0].base;
            }
            if (ok) {
                pending_id_loops.clear();
                if (opt.scan_single_pass && !opt.bounds_check) {
                    units.push_back(lower_scan1d_single(L, scan_acc, opt));
                } else {
                    for (LaunchUnit &su : lower_scan1d(L, scan_acc, opt)) units.push_back(std::move(su));
                }
                continue;
            }
        }
        bool all_reduce = !L._sweeps.empty();
        for (const InstrPtr &s : L._sweeps) all_reduce = all_reduce && bh_opcode_is_reduction(s->opcode);
        if (all_reduce && L.isInnermost() && pending_id_loops.empty()) {
            // Every folded identity must belong to one of this loop's reductions.
            set<ViewKey> outs;
            for (const InstrPtr &s : L._sweeps) outs.insert(ViewKey(s->operand[0]));
            bool ok = true;
            for (const InstrPtr &i : pending_identities) ok = ok && outs.count(ViewKey(i->operand[0]));
            if (ok) {
                units.push_back(lower_grid_reduce(L, pending_identities, opt));
                pending_identities.clear();
                continue;
            }
        }
        if (all_reduce && outer_reduce_applicable(L) && pending_identities.empty()) {
            set<ViewKey> outs;
            for (const InstrPtr &s : L._sweeps) outs.insert(ViewKey(s->operand[0]));
            bool ok = true;
            for (const Block *il : pending_id_loops) ok = ok && outs.count(ViewKey(jitk::all_instr(*il)[0]->operand[0]));
            if (ok) {
                units.push_back(lower_outer_reduce(L, pending_id_loops, opt));
                pending_id_loops.clear();
                continue;
            }
        }
        serial = true;
    }
    if (!serial && (!pending_identities.empty() || !pending_id_loops.empty())) serial = true;
    if (serial) return {lower_serial(items, opt)};
    return units;
}

vector<int> fuse_tails(const vector<LoopB> &kernels, vector<vector<LaunchUnit>> &lowered, const CodegenOptions &opt) {
    vector<int> into(lowered.size(), -1);
    if (opt.bounds_check) return into;
    // Bases each kernel reads and writes (frees count as writes).
    const size_t n = kernels.size();
    vector<set<const bh_base *>> reads(n), writes(n);
    for (size_t k = 0; k < n; ++k) {
        for (const InstrPtr &ip : jitk::all_instr(kernels[k]))
            for (size_t o = 0; o < ip->operand.size(); ++o)
                if (!ip->operand[o].isConstant()) (o == 0 ? writes[k] : reads[k]).insert(ip->operand[o].base);
        for (bh_base *f : kernels[k].getAllFrees()) writes[k].insert(f);
    }
    auto meets = [](const set<const bh_base *> &a, const set<const bh_base *> &b) {
        for (const bh_base *x : a)
            if (b.count(x)) return true;
        return false;
    };
    for (size_t j = 1; j < n; ++j) {
        if (lowered[j].size() != 1 || !lowered[j][0].tail_capable || lowered[j][0].body_core.empty()) continue;
        // The producer: the last earlier kernel that writes an array this reduction reads. The
        // reduction moves up to the end of the producer's kernel, which keeps the program's
        // meaning when it commutes with every kernel in between (no array one writes and the other
        // reads or writes).
        size_t k = j;
        while (k > 0 && !meets(writes[k - 1], reads[j])) --k;
        if (k == 0) continue;
        --k;
        bool commutes = true;
        for (size_t m = k + 1; m < j && commutes; ++m)
            commutes = !meets(writes[m], reads[j]) && !meets(writes[m], writes[j]) && !meets(reads[m], writes[j]);
        if (!commutes || lowered[k].empty() || into[k] >= 0) continue;
        LaunchUnit &u1 = lowered[k].back();
        if (u1.tail || u1.sched == Sched::SCAN1D || u1.sched == Sched::SERIAL || u1.sched == Sched::TILE2D ||
            u1.body_core.empty())
            continue;
        u1 = fuse_tail(u1, lowered[j][0]);
        lowered[j].clear();
        into[j] = static_cast<int>(k);
        writes[k].insert(writes[j].begin(), writes[j].end());
        reads[k].insert(reads[j].begin(), reads[j].end());
    }
    return into;
}

} // namespace cuda
} // namespace bohrium
