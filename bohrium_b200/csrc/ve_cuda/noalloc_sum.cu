// Allocation-free float64 sum: a variant of the engine's GRID_REDUCE kernel (an ADD_REDUCE of a
// contiguous float64 array to one scalar) whose scratch memory is a fixed array in this library's
// device image instead of memory taken from the engine's stream-ordered pool.
//
// Callers that cannot allocate: a host framework that owns the device memory (its own caching
// allocator has reserved the HBM, so a cudaMalloc from a library fails or fragments its pool); a
// latency-bound loop, because cudaFree synchronises the whole device and cudaMalloc can block; and
// code that runs after a failed allocation and must still finish a reduction.
//
// Order of operations (the same as the GRID_REDUCE schedule, so the result equals the engine's
// ADD_REDUCE of the same array): tiles of 256 threads x 8 elements, thread x adds elements
// tile*2048 + (j/4)*1024 + 4x + j%4 for j = 0..7 in order (two 16-byte words), a warp-shuffle
// butterfly (xor 16, 8, 4, 2, 1) and
// the same butterfly over the 8 warp sums gives the tile partial; the CTA that completes the last
// tile folds the partials (thread t adds tiles t, t+256, ... in order) with the same CTA tree.
//
// Scratch: g_noalloc_scratch, a file-scope __device__ byte array of kScratchBytes (65,792 bytes):
// kMaxTiles float64 tile partials, then one 32-bit completion counter. Every call on a device
// shares it. The counter must start at zero; each call clears it on its stream before the kernel
// (and the kernel clears it again when it finishes); the partials are overwritten by every call.
// Calls whose kernels overlap on the GPU (on different streams, or from several host threads
// without ordering) race on the array and give wrong results; calls ordered on one stream are safe.
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <cuda_runtime.h>

extern "C" void bhb_set_last_error(const char *msg);

namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 8;
constexpr int64_t kTile = kThreads * kPerThread;
constexpr int64_t kMaxTiles = 8192;  // at most kMaxTiles * kTile = 16,777,216 elements
constexpr size_t kCounterOffset = kMaxTiles * sizeof(double);
constexpr size_t kScratchBytes = kCounterOffset + 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Per-device set-up, filled by the first call on each device. `scratch` is published with release
// order after `max_ctas` is written, so a thread that reads a non-null `scratch` (acquire) also
// sees `max_ctas`; concurrent first calls on one device serialise on g_setup_mutex.
struct DeviceSetup {
    std::atomic<unsigned char *> scratch{nullptr};  // device address of g_noalloc_scratch
    int64_t max_ctas = 0;                           // SMs x resident CTAs per SM of noalloc_sum_kernel
};
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mutex;

__device__ __forceinline__ double block_sum(double v, double *sm) {
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) {
        const double o = __shfl_xor_sync(0xffffffffu, v, m);
        v = v + o;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sm[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < kThreads / 32 ? sm[lane] : 0.0;
#pragma unroll
        for (int m = 16; m >= 1; m >>= 1) {
            const double o = __shfl_xor_sync(0xffffffffu, v, m);
            v = v + o;
        }
    }
    return v;
}

__global__ void __launch_bounds__(kThreads) noalloc_sum_kernel(const double *__restrict__ in, int64_t n,
                                                               double *__restrict__ out,
                                                               unsigned char *__restrict__ scratch) {
    __shared__ double sm[kThreads / 32];
    __shared__ bool am_last;
    double *partials = reinterpret_cast<double *>(scratch);
    unsigned int *counter = reinterpret_cast<unsigned int *>(scratch + kCounterOffset);
    const int64_t ntiles = (n + kTile - 1) / kTile;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        double acc = 0.0;
        if ((tile + 1) * kTile <= n) {
#pragma unroll
            for (int j = 0; j < kPerThread; ++j)
                acc = acc + in[tile * kTile + (j >> 2) * (kTile / 2) + threadIdx.x * 4 + (j & 3)];
        } else {
            for (int j = 0; j < kPerThread; ++j) {
                const int64_t i = tile * kTile + (j >> 2) * (kTile / 2) + threadIdx.x * 4 + (j & 3);
                if (i >= n) break;
                acc = acc + in[i];
            }
        }
        acc = block_sum(acc, sm);
        if (threadIdx.x == 0) {
            partials[tile] = acc;
            __threadfence();
            am_last = atomicAdd(counter, 1u) == static_cast<unsigned>(ntiles - 1);
        }
        __syncthreads();
        if (am_last) {  // every tile is done: this CTA has no further tile
            __threadfence();
            double total = 0.0;
            for (int64_t t = threadIdx.x; t < ntiles; t += kThreads) {
                const double x = reinterpret_cast<volatile double *>(partials)[t];
                total = total + x;
            }
            total = block_sum(total, sm);
            if (threadIdx.x == 0) {
                *out = total;
                *counter = 0u;
            }
        }
    }
}

int fail(const char *what, cudaError_t e) {
    char msg[256];
    snprintf(msg, sizeof msg, "bh_ve_cuda_sum_f64_noalloc: %s: %s", what, cudaGetErrorString(e));
    bhb_set_last_error(msg);
    return -1;
}

} // namespace

// Declared in include/bh_b200.h. Returns 0 on success, -1 with bhb_last_error() set on error.
extern "C" int bh_ve_cuda_sum_f64_noalloc(const double *in, int64_t n, double *out, void *stream) {
    char msg[256];
    if (n < 0 || (n > 0 && in == nullptr) || out == nullptr) {
        bhb_set_last_error("bh_ve_cuda_sum_f64_noalloc: bad arguments (n < 0 or a null pointer)");
        return -1;
    }
    const int64_t ntiles = (n + kTile - 1) / kTile;
    if (ntiles > kMaxTiles) {
        snprintf(msg, sizeof msg,
                 "bh_ve_cuda_sum_f64_noalloc: %lld elements exceed the maximum of %lld (static scratch of %lld "
                 "tile partials)",
                 static_cast<long long>(n), static_cast<long long>(kMaxTiles * kTile),
                 static_cast<long long>(kMaxTiles));
        bhb_set_last_error(msg);
        return -1;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail("cudaGetDevice", e);
    if (dev < 0 || dev >= kMaxDevices) {
        bhb_set_last_error("bh_ve_cuda_sum_f64_noalloc: device ordinal out of range");
        return -1;
    }
    // Set-up, once per device, with that device current: the device address of the static
    // scratch array and the persistent grid size. The first call on a device should come before
    // any stream capture on it.
    DeviceSetup &ds = g_setup[dev];
    unsigned char *scratch = ds.scratch.load(std::memory_order_acquire);
    if (scratch == nullptr) {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        scratch = ds.scratch.load(std::memory_order_acquire);
        if (scratch == nullptr) {
            void *ptr = nullptr;
            e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (e != cudaSuccess) return fail("cudaGetSymbolAddress", e);
            int sms = 0, occ = 0;
            e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (e != cudaSuccess) return fail("cudaDeviceGetAttribute", e);
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, noalloc_sum_kernel, kThreads, 0);
            if (e != cudaSuccess) return fail("cudaOccupancyMaxActiveBlocksPerMultiprocessor", e);
            ds.max_ctas = static_cast<int64_t>(sms) * (occ > 0 ? occ : 1);
            scratch = static_cast<unsigned char *>(ptr);
            ds.scratch.store(scratch, std::memory_order_release);
        }
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    e = cudaMemsetAsync(scratch + kCounterOffset, 0, sizeof(unsigned int), s);
    if (e != cudaSuccess) return fail("cudaMemsetAsync", e);
    if (n == 0) {  // the ADD identity
        e = cudaMemsetAsync(out, 0, sizeof(double), s);
        return e == cudaSuccess ? 0 : fail("cudaMemsetAsync", e);
    }
    const int64_t grid = ntiles < ds.max_ctas ? ntiles : ds.max_ctas;
    noalloc_sum_kernel<<<static_cast<unsigned>(grid), kThreads, 0, s>>>(in, n, out, scratch);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail("kernel launch", e);
    return 0;
}
