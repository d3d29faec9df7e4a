// cuBLAS-backed BLAS extension methods for the cuda engine.
//
// Same method names and operand convention as the reference's BLAS extmethods
// (extmethods/blas/templates/methods.json and body.tpl): `blas_gemm` computes C = A * B and
// `blas_gemmt` computes C = A^T * B for row-major contiguous matrices, operand[0] = C,
// operand[1] = A, operand[2] = B, float32 or float64. The multiplication itself is cuBLAS
// (called, not restated), enqueued on the engine's stream on the engine's device buffers, so
// the operands never leave the GPU. Row-major products map onto cuBLAS's column-major ones by
// swapping the operands: C^T = B^T * A^T.
#include <cstdint>
#include <stdexcept>
#include <string>
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <bh_b200.h>
#include <bohrium/bh_extmethod.hpp>

using namespace std;
using namespace bohrium;

namespace {

void ck(cublasStatus_t s, const char *what) {
    if (s != CUBLAS_STATUS_SUCCESS) throw runtime_error(string("[cuBLAS] ") + what + " failed with status " + to_string(s));
}

const bh_ve_cuda_ext_context &context(void *arg) {
    const auto *ctx = static_cast<const bh_ve_cuda_ext_context *>(arg);
    if (ctx == nullptr || ctx->version != 1)
        throw runtime_error("cuBLAS extmethods need the cuda engine's extension context");
    return *ctx;
}

void require_matrix(const bh_view &v, const char *name) {
    if (v.isConstant() || v.ndim != 2 || !v.isContiguous())
        throw runtime_error(string("cuBLAS extmethod: ") + name + " must be a contiguous 2-D array");
}

class Gemm : public extmethod::ExtmethodImpl {
    cublasHandle_t handle = nullptr;
    bool transA;

public:
    explicit Gemm(bool trans_a) : transA(trans_a) { ck(cublasCreate(&handle), "cublasCreate"); }
    ~Gemm() override {
        if (handle) cublasDestroy(handle);
    }
    void execute(bh_instruction *instr, void *arg) override {
        const bh_ve_cuda_ext_context &ctx = context(arg);
        if (instr->operand.size() != 3) throw runtime_error("cuBLAS gemm: needs C, A and B");
        const bh_view &C = instr->operand[0], &A = instr->operand[1], &B = instr->operand[2];
        require_matrix(C, "C");
        require_matrix(A, "A");
        require_matrix(B, "B");
        const bh_type t = C.base->dtype();
        if (A.base->dtype() != t || B.base->dtype() != t)
            throw runtime_error("cuBLAS gemm: A, B and C must have the same type");
        // Row-major A is m x k (transA: k x m), B is k x n, C is m x n.
        const int64_t m = C.shape[0], n = C.shape[1];
        const int64_t k = transA ? A.shape[0] : A.shape[1];
        if ((transA ? A.shape[1] : A.shape[0]) != m || B.shape[0] != k || B.shape[1] != n)
            throw runtime_error("cuBLAS gemm: shapes do not match");
        ck(cublasSetStream(handle, static_cast<cudaStream_t>(ctx.stream)), "cublasSetStream");
        const size_t es = t == bh_type::FLOAT64 ? 8 : 4;
        char *a = static_cast<char *>(ctx.device_pointer(ctx.engine, A.base)) + A.start * es;
        char *b = static_cast<char *>(ctx.device_pointer(ctx.engine, B.base)) + B.start * es;
        char *c = static_cast<char *>(ctx.device_pointer(ctx.engine, C.base)) + C.start * es;
        // Column-major view: C^T (n x m) = B^T (n x k) * op(A)^T (k x m).
        const cublasOperation_t opA = transA ? CUBLAS_OP_T : CUBLAS_OP_N;
        const int lda = static_cast<int>(transA ? m : k);
        if (t == bh_type::FLOAT64) {
            const double one = 1.0, zero = 0.0;
            ck(cublasDgemm(handle, CUBLAS_OP_N, opA, static_cast<int>(n), static_cast<int>(m), static_cast<int>(k), &one,
                           reinterpret_cast<double *>(b), static_cast<int>(n), reinterpret_cast<double *>(a), lda, &zero,
                           reinterpret_cast<double *>(c), static_cast<int>(n)),
               "cublasDgemm");
        } else if (t == bh_type::FLOAT32) {
            const float one = 1.f, zero = 0.f;
            ck(cublasSgemm(handle, CUBLAS_OP_N, opA, static_cast<int>(n), static_cast<int>(m), static_cast<int>(k), &one,
                           reinterpret_cast<float *>(b), static_cast<int>(n), reinterpret_cast<float *>(a), lda, &zero,
                           reinterpret_cast<float *>(c), static_cast<int>(n)),
               "cublasSgemm");
        } else {
            throw runtime_error("cuBLAS gemm: only float32 and float64 are supported");
        }
        ctx.written(ctx.engine, C.base);
    }
};

} // namespace

extern "C" extmethod::ExtmethodImpl *blas_gemm_create() { return new Gemm(false); }
extern "C" void blas_gemm_destroy(extmethod::ExtmethodImpl *self) { delete self; }
extern "C" extmethod::ExtmethodImpl *blas_gemmt_create() { return new Gemm(true); }
extern "C" void blas_gemmt_destroy(extmethod::ExtmethodImpl *self) { delete self; }
