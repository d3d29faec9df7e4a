// The learned fusion cost model's network: an MLP F -> 64 -> 64 -> 1 (ReLU, float32) that maps the
// feature vector of a fused block to its predicted log device time. Inference and training run on
// the GPU with the kernels below; all reductions over rows are done in a fixed order, so training
// is deterministic (no floating-point atomics).
//
// Parameter layout (float32, one contiguous array of nparams):
//   W1[H][F]  b1[H]  W2[H][H]  b2[H]  W3[H]  b3
// Loss: mean squared error over the rows, L = (1/R) * sum_r (y_r - t_r)^2.
//
// Kernels:
//   mlp_forward      one thread per row, weights staged in shared memory (broadcast reads)
//   mlp_grad_chunk   a CTA per chunk of kRowsPerChunk rows: row-parallel forward/backward into
//                    shared memory, then parameter-parallel sums over the chunk's rows in row
//                    order -> one partial gradient per chunk
//   mlp_reduce_adam  parameter-parallel: sums the chunk partials in chunk order and applies Adam
//                    (or only writes the gradient)
// These are small, latency-bound kernels (5,313 parameters); tensor cores do not apply.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <random>
#include <vector>
#include <cuda_runtime.h>

extern "C" void bhb_set_last_error(const char *msg);

namespace {

constexpr int kF = 16;   // features
constexpr int kH = 64;   // hidden width
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kH * kF;
constexpr int kOffW2 = kOffB1 + kH;
constexpr int kOffB2 = kOffW2 + kH * kH;
constexpr int kOffW3 = kOffB2 + kH;
constexpr int kOffB3 = kOffW3 + kH;
constexpr int kParams = kOffB3 + 1;  // 5313
constexpr int kThreads = 256;
constexpr int kRowsPerChunk = 128;

__device__ __forceinline__ void load_params(const float *__restrict__ p, float *sp) {
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) sp[i] = p[i];
    __syncthreads();
}

// Forward of one row; h1/h2 receive the post-ReLU activations. Returns y.
__device__ __forceinline__ float row_forward(const float *sp, const float *x, float *h1, float *h2) {
#pragma unroll 4
    for (int i = 0; i < kH; ++i) {
        float a = sp[kOffB1 + i];
#pragma unroll
        for (int f = 0; f < kF; ++f) a = fmaf(sp[kOffW1 + i * kF + f], x[f], a);
        h1[i] = a > 0.f ? a : 0.f;
    }
    for (int i = 0; i < kH; ++i) {
        float a = sp[kOffB2 + i];
#pragma unroll 8
        for (int j = 0; j < kH; ++j) a = fmaf(sp[kOffW2 + i * kH + j], h1[j], a);
        h2[i] = a > 0.f ? a : 0.f;
    }
    float y = sp[kOffB3];
#pragma unroll 8
    for (int i = 0; i < kH; ++i) y = fmaf(sp[kOffW3 + i], h2[i], y);
    return y;
}

__global__ void __launch_bounds__(kThreads) mlp_forward(const float *__restrict__ params, const float *__restrict__ x,
                                                        int64_t rows, float *__restrict__ y) {
    extern __shared__ float sp[];
    load_params(params, sp);
    const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    float xr[kF], h1[kH], h2[kH];
#pragma unroll
    for (int f = 0; f < kF; ++f) xr[f] = x[r * kF + f];
    y[r] = row_forward(sp, xr, h1, h2);
}

// Shared memory of mlp_grad_chunk: the parameters, then one record per row of the chunk holding
// the input x, the activations h1 and h2, the pre-activation gradients dz1 and dz2, and dy.
// The record length (273 floats) is odd, so rows map to distinct banks.
constexpr int kRx = 0, kRh1 = kF, kRh2 = kRh1 + kH, kRdz1 = kRh2 + kH, kRdz2 = kRdz1 + kH, kRdy = kRdz2 + kH;
constexpr int kRowFloats = kRdy + 1;
constexpr size_t kGradSmem = (kParams + kRowsPerChunk * kRowFloats) * sizeof(float);

// rows_total: the number of rows the loss is averaged over (the minibatch). idx: optional row
// indices (nullptr: rows are x[first + i]).
__global__ void __launch_bounds__(kThreads) mlp_grad_chunk(const float *__restrict__ params, const float *__restrict__ x,
                                                           const float *__restrict__ t, const int32_t *__restrict__ idx,
                                                           int64_t first, int64_t nrows, int64_t rows_total,
                                                           float *__restrict__ partial, float *__restrict__ sqerr) {
    extern __shared__ float smem[];
    float *sp = smem;
    float *rowbuf = smem + kParams;
    load_params(params, sp);
    const int64_t c0 = static_cast<int64_t>(blockIdx.x) * kRowsPerChunk;
    const int nr = static_cast<int>(nrows - c0 < kRowsPerChunk ? nrows - c0 : kRowsPerChunk);
    // Row phase: one thread per row of the chunk.
    for (int lr = threadIdx.x; lr < nr; lr += blockDim.x) {
        const int64_t i = c0 + lr;
        const int64_t r = idx ? static_cast<int64_t>(idx[first + i]) : first + i;
        float *rb = rowbuf + lr * kRowFloats;
        float *xs = rb + kRx, *h1 = rb + kRh1, *h2 = rb + kRh2, *dz1 = rb + kRdz1, *dz2 = rb + kRdz2, *dy = rb + kRdy;
        for (int f = 0; f < kF; ++f) xs[f] = x[r * kF + f];
        const float y = row_forward(sp, xs, h1, h2);
        const float e = y - t[r];
        sqerr[i] = e * e;
        const float g = 2.f * e / static_cast<float>(rows_total);
        *dy = g;
        for (int k = 0; k < kH; ++k) dz2[k] = h2[k] > 0.f ? g * sp[kOffW3 + k] : 0.f;
        for (int j = 0; j < kH; ++j) {
            float a = 0.f;
            for (int k = 0; k < kH; ++k) a = fmaf(sp[kOffW2 + k * kH + j], dz2[k], a);
            dz1[j] = h1[j] > 0.f ? a : 0.f;
        }
    }
    __syncthreads();
    // Parameter phase: each parameter's sum over the chunk's rows, in row order.
    float *out = partial + static_cast<int64_t>(blockIdx.x) * kParams;
    for (int p = threadIdx.x; p < kParams; p += blockDim.x) {
        float acc = 0.f;
        if (p < kOffB1) {  // W1[i][f] += dz1[i] * x[f]
            const int i = p / kF, f = p % kF;
            for (int lr = 0; lr < nr; ++lr) {
                const float *rb = rowbuf + lr * kRowFloats;
                acc = fmaf(rb[kRdz1 + i], rb[kRx + f], acc);
            }
        } else if (p < kOffW2) {  // b1[i] += dz1[i]
            const int i = p - kOffB1;
            for (int lr = 0; lr < nr; ++lr) acc += rowbuf[lr * kRowFloats + kRdz1 + i];
        } else if (p < kOffB2) {  // W2[i][j] += dz2[i] * h1[j]
            const int i = (p - kOffW2) / kH, j = (p - kOffW2) % kH;
            for (int lr = 0; lr < nr; ++lr) {
                const float *rb = rowbuf + lr * kRowFloats;
                acc = fmaf(rb[kRdz2 + i], rb[kRh1 + j], acc);
            }
        } else if (p < kOffW3) {  // b2[i] += dz2[i]
            const int i = p - kOffB2;
            for (int lr = 0; lr < nr; ++lr) acc += rowbuf[lr * kRowFloats + kRdz2 + i];
        } else if (p < kOffB3) {  // W3[i] += dy * h2[i]
            const int i = p - kOffW3;
            for (int lr = 0; lr < nr; ++lr) {
                const float *rb = rowbuf + lr * kRowFloats;
                acc = fmaf(rb[kRdy], rb[kRh2 + i], acc);
            }
        } else {  // b3 += dy
            for (int lr = 0; lr < nr; ++lr) acc += rowbuf[lr * kRowFloats + kRdy];
        }
        out[p] = acc;
    }
}

struct AdamState {
    float lr, beta1, beta2, eps;
    int step;  // 1-based step of this update
};

// grad[p] = sum over chunks (in chunk order) of partial[c][p]; then Adam when `adam` is set.
__global__ void __launch_bounds__(kThreads) mlp_reduce_adam(const float *__restrict__ partial, int nchunks,
                                                            float *__restrict__ grad, float *__restrict__ params,
                                                            float *__restrict__ m, float *__restrict__ v, int adam,
                                                            AdamState st) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kParams) return;
    float g = 0.f;
    for (int c = 0; c < nchunks; ++c) g += partial[static_cast<int64_t>(c) * kParams + p];
    grad[p] = g;
    if (!adam) return;
    const float mp = st.beta1 * m[p] + (1.f - st.beta1) * g;
    const float vp = st.beta2 * v[p] + (1.f - st.beta2) * g * g;
    m[p] = mp;
    v[p] = vp;
    const float bc1 = 1.f - powf(st.beta1, static_cast<float>(st.step));
    const float bc2 = 1.f - powf(st.beta2, static_cast<float>(st.step));
    params[p] -= st.lr * (mp / bc1) / (sqrtf(vp / bc2) + st.eps);
}

// Sum of n values in a fixed order (one CTA; thread strided partials then a tree).
__global__ void __launch_bounds__(kThreads) sum_fixed(const float *__restrict__ in, int64_t n, float *__restrict__ out) {
    __shared__ float sm[kThreads];
    float acc = 0.f;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) acc += in[i];
    sm[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sm[threadIdx.x] += sm[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sm[0];
}

} // namespace

// --------------------------------------------------------------------------------- host side
struct bh_costmodel {
    int device = 0;
    cudaStream_t stream = nullptr;
    float *params = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr;
    float *partial = nullptr;  // [chunks][kParams]
    int64_t partial_chunks = 0;
    float *x = nullptr, *t = nullptr, *y = nullptr, *sqerr = nullptr, *scalar = nullptr;
    int64_t cap_rows = 0;
    int32_t *idx = nullptr;
    int adam_step = 0;
};

namespace {

bool ok(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return true;
    char msg[256];
    snprintf(msg, sizeof msg, "cost model: %s: %s", what, cudaGetErrorString(e));
    bhb_set_last_error(msg);
    return false;
}

bool ensure_rows(bh_costmodel *cm, int64_t rows) {
    if (rows <= cm->cap_rows) return true;
    cudaFree(cm->x);
    cudaFree(cm->t);
    cudaFree(cm->y);
    cudaFree(cm->sqerr);
    cudaFree(cm->idx);
    cm->x = cm->t = cm->y = cm->sqerr = nullptr;
    cm->idx = nullptr;
    cm->cap_rows = 0;
    const int64_t cap = rows < 1024 ? 1024 : rows;
    if (!ok(cudaMalloc(&cm->x, cap * kF * sizeof(float)), "cudaMalloc") ||
        !ok(cudaMalloc(&cm->t, cap * sizeof(float)), "cudaMalloc") ||
        !ok(cudaMalloc(&cm->y, cap * sizeof(float)), "cudaMalloc") ||
        !ok(cudaMalloc(&cm->sqerr, cap * sizeof(float)), "cudaMalloc") ||
        !ok(cudaMalloc(&cm->idx, cap * sizeof(int32_t)), "cudaMalloc"))
        return false;
    cm->cap_rows = cap;
    return true;
}

bool ensure_chunks(bh_costmodel *cm, int64_t chunks) {
    if (chunks <= cm->partial_chunks) return true;
    cudaFree(cm->partial);
    cm->partial = nullptr;
    cm->partial_chunks = 0;
    if (!ok(cudaMalloc(&cm->partial, chunks * kParams * sizeof(float)), "cudaMalloc")) return false;
    cm->partial_chunks = chunks;
    return true;
}

bool upload(bh_costmodel *cm, const float *x, const float *t, int64_t rows) {
    if (!ensure_rows(cm, rows)) return false;
    if (rows == 0) return true;
    if (!ok(cudaMemcpyAsync(cm->x, x, rows * kF * sizeof(float), cudaMemcpyHostToDevice, cm->stream), "H2D")) return false;
    if (t && !ok(cudaMemcpyAsync(cm->t, t, rows * sizeof(float), cudaMemcpyHostToDevice, cm->stream), "H2D")) return false;
    return true;
}

// Gradient (and optionally an Adam step) of the MSE over rows [first, first+n) of the uploaded
// data (through cm->idx when `use_idx`).
bool grad_step(bh_costmodel *cm, int64_t first, int64_t n, bool use_idx, bool adam, float lr) {
    const int64_t chunks = (n + kRowsPerChunk - 1) / kRowsPerChunk;
    if (!ensure_chunks(cm, chunks)) return false;
    mlp_grad_chunk<<<static_cast<unsigned>(chunks), kThreads, kGradSmem, cm->stream>>>(
        cm->params, cm->x, cm->t, use_idx ? cm->idx : nullptr, first, n, n, cm->partial, cm->sqerr);
    if (!ok(cudaGetLastError(), "mlp_grad_chunk")) return false;
    AdamState st{lr, 0.9f, 0.999f, 1e-8f, adam ? ++cm->adam_step : 0};
    mlp_reduce_adam<<<(kParams + kThreads - 1) / kThreads, kThreads, 0, cm->stream>>>(
        cm->partial, static_cast<int>(chunks), cm->grad, cm->params, cm->m, cm->v, adam ? 1 : 0, st);
    return ok(cudaGetLastError(), "mlp_reduce_adam");
}

void init_params(std::vector<float> &p, uint64_t seed) {
    std::mt19937_64 rng(seed);
    auto fill = [&](int off, int n, int fan_in) {
        std::normal_distribution<double> d(0.0, std::sqrt(2.0 / fan_in));  // He initialisation
        for (int i = 0; i < n; ++i) p[static_cast<size_t>(off + i)] = static_cast<float>(d(rng));
    };
    p.assign(kParams, 0.f);
    fill(kOffW1, kH * kF, kF);
    fill(kOffW2, kH * kH, kH);
    fill(kOffW3, kH, kH);
}

} // namespace

extern "C" {

int bh_ve_cuda_costmodel_nfeatures(void) { return kF; }
int64_t bh_ve_cuda_costmodel_nparams(void) { return kParams; }

bh_costmodel *bh_ve_cuda_costmodel_create(uint64_t seed) {
    bh_costmodel *cm = new (std::nothrow) bh_costmodel();
    if (!cm) return nullptr;
    if (!ok(cudaGetDevice(&cm->device), "cudaGetDevice") ||
        !ok(cudaStreamCreateWithFlags(&cm->stream, cudaStreamNonBlocking), "cudaStreamCreate") ||
        !ok(cudaMalloc(&cm->params, kParams * sizeof(float)), "cudaMalloc") ||
        !ok(cudaMalloc(&cm->m, kParams * sizeof(float)), "cudaMalloc") ||
        !ok(cudaMalloc(&cm->v, kParams * sizeof(float)), "cudaMalloc") ||
        !ok(cudaMalloc(&cm->grad, kParams * sizeof(float)), "cudaMalloc") ||
        !ok(cudaMalloc(&cm->scalar, sizeof(float)), "cudaMalloc") ||
        !ok(cudaFuncSetAttribute(mlp_grad_chunk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kGradSmem)), "cudaFuncSetAttribute") ||
        !ok(cudaFuncSetAttribute(mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kParams * sizeof(float))), "cudaFuncSetAttribute")) {
        delete cm;  // device memory of a failed create is released with the context
        return nullptr;
    }
    std::vector<float> p;
    init_params(p, seed);
    if (!ok(cudaMemcpy(cm->params, p.data(), kParams * sizeof(float), cudaMemcpyHostToDevice), "H2D") ||
        !ok(cudaMemset(cm->m, 0, kParams * sizeof(float)), "cudaMemset") ||
        !ok(cudaMemset(cm->v, 0, kParams * sizeof(float)), "cudaMemset")) {
        delete cm;
        return nullptr;
    }
    return cm;
}

void bh_ve_cuda_costmodel_destroy(bh_costmodel *cm) {
    if (!cm) return;
    cudaStreamSynchronize(cm->stream);
    for (float *p : {cm->params, cm->m, cm->v, cm->grad, cm->partial, cm->x, cm->t, cm->y, cm->sqerr, cm->scalar})
        cudaFree(p);
    cudaFree(cm->idx);
    cudaStreamDestroy(cm->stream);
    delete cm;
}

int bh_ve_cuda_costmodel_get_params(bh_costmodel *cm, float *out) {
    if (!ok(cudaMemcpyAsync(out, cm->params, kParams * sizeof(float), cudaMemcpyDeviceToHost, cm->stream), "D2H"))
        return -1;
    return ok(cudaStreamSynchronize(cm->stream), "sync") ? 0 : -1;
}

int bh_ve_cuda_costmodel_set_params(bh_costmodel *cm, const float *in) {
    cm->adam_step = 0;
    if (!ok(cudaMemcpyAsync(cm->params, in, kParams * sizeof(float), cudaMemcpyHostToDevice, cm->stream), "H2D") ||
        !ok(cudaMemsetAsync(cm->m, 0, kParams * sizeof(float), cm->stream), "cudaMemset") ||
        !ok(cudaMemsetAsync(cm->v, 0, kParams * sizeof(float), cm->stream), "cudaMemset"))
        return -1;
    return ok(cudaStreamSynchronize(cm->stream), "sync") ? 0 : -1;
}

// y[r] = network(x[r]) for `rows` rows of kF features (host arrays).
int bh_ve_cuda_costmodel_predict(bh_costmodel *cm, const float *x, int64_t rows, float *y) {
    if (rows < 0) return -1;
    if (rows == 0) return 0;
    if (!upload(cm, x, nullptr, rows)) return -1;
    const unsigned grid = static_cast<unsigned>((rows + kThreads - 1) / kThreads);
    mlp_forward<<<grid, kThreads, kParams * sizeof(float), cm->stream>>>(cm->params, cm->x, rows, cm->y);
    if (!ok(cudaGetLastError(), "mlp_forward")) return -1;
    if (!ok(cudaMemcpyAsync(y, cm->y, rows * sizeof(float), cudaMemcpyDeviceToHost, cm->stream), "D2H")) return -1;
    return ok(cudaStreamSynchronize(cm->stream), "sync") ? 0 : -1;
}

// Gradient of the mean squared error over all rows, and the loss (host arrays; no update).
int bh_ve_cuda_costmodel_gradient(bh_costmodel *cm, const float *x, const float *t, int64_t rows, float *grad,
                                  float *loss) {
    if (rows <= 0) return -1;
    if (!upload(cm, x, t, rows) || !grad_step(cm, 0, rows, false, false, 0.f)) return -1;
    sum_fixed<<<1, kThreads, 0, cm->stream>>>(cm->sqerr, rows, cm->scalar);
    if (!ok(cudaGetLastError(), "sum_fixed")) return -1;
    float s = 0.f;
    if (!ok(cudaMemcpyAsync(grad, cm->grad, kParams * sizeof(float), cudaMemcpyDeviceToHost, cm->stream), "D2H") ||
        !ok(cudaMemcpyAsync(&s, cm->scalar, sizeof(float), cudaMemcpyDeviceToHost, cm->stream), "D2H") ||
        !ok(cudaStreamSynchronize(cm->stream), "sync"))
        return -1;
    *loss = s / static_cast<float>(rows);
    return 0;
}

// Minibatch Adam training on `rows` samples for `epochs` passes; each epoch visits the rows in a
// seeded random order. `loss_out` (optional) receives the final mean squared error over all rows.
int bh_ve_cuda_costmodel_train(bh_costmodel *cm, const float *x, const float *t, int64_t rows, int epochs,
                               int batch, float lr, uint64_t seed, float *loss_out) {
    if (rows <= 0 || epochs < 0 || batch <= 0 || rows > INT32_MAX) return -1;
    if (!upload(cm, x, t, rows)) return -1;
    std::mt19937_64 rng(seed);
    std::vector<int32_t> order(static_cast<size_t>(rows));
    for (int64_t i = 0; i < rows; ++i) order[static_cast<size_t>(i)] = static_cast<int32_t>(i);
    int32_t *pinned = nullptr;
    if (!ok(cudaMallocHost(&pinned, rows * sizeof(int32_t)), "cudaMallocHost")) return -1;
    int rc = 0;
    for (int e = 0; e < epochs && rc == 0; ++e) {
        std::shuffle(order.begin(), order.end(), rng);
        // The previous epoch's copy has to finish before the staging buffer is rewritten.
        if (!ok(cudaStreamSynchronize(cm->stream), "sync")) {
            rc = -1;
            break;
        }
        memcpy(pinned, order.data(), rows * sizeof(int32_t));
        if (!ok(cudaMemcpyAsync(cm->idx, pinned, rows * sizeof(int32_t), cudaMemcpyHostToDevice, cm->stream), "H2D")) {
            rc = -1;
            break;
        }
        for (int64_t b0 = 0; b0 < rows; b0 += batch) {
            const int64_t n = rows - b0 < batch ? rows - b0 : batch;
            if (!grad_step(cm, b0, n, true, true, lr)) {
                rc = -1;
                break;
            }
        }
    }
    if (rc == 0 && !ok(cudaStreamSynchronize(cm->stream), "sync")) rc = -1;
    cudaFreeHost(pinned);
    if (rc == 0 && loss_out) {
        // Loss over all rows with the trained parameters (the data is still uploaded).
        if (!grad_step(cm, 0, rows, false, false, 0.f)) return -1;
        sum_fixed<<<1, kThreads, 0, cm->stream>>>(cm->sqerr, rows, cm->scalar);
        float s = 0.f;
        if (!ok(cudaGetLastError(), "sum_fixed") ||
            !ok(cudaMemcpyAsync(&s, cm->scalar, sizeof(float), cudaMemcpyDeviceToHost, cm->stream), "D2H") ||
            !ok(cudaStreamSynchronize(cm->stream), "sync"))
            return -1;
        *loss_out = s / static_cast<float>(rows);
    }
    return rc;
}

} // extern "C"
