// Move-ordering MLP: tcgen05 GEMM and element-wise kernels (mlp_gemm.cu, mlp_kernels.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

namespace tdp {
namespace mlp {

constexpr int kFeatures = 1088;     // 32x32 adjacency bits + 64-bin cycle-length histogram
constexpr int kHidden = 256;
constexpr int kTriples = 4960;        // C(32,3)
constexpr int kTriplesPadded = 5120;  // 20 tiles of 256

struct GemmParams {
    int M, N, K;
    const float *bias;
    int relu;
    __nv_bfloat16 *outBf16;
    float *outF32;
    int ldo;
    int *error;
};

// One-time set-up of the GEMM (shared-memory attribute, tensor-map encoder); 0 on success.
int prepare(std::string &err);

// C = A[M x K] * B[N x K]^T (+ bias, ReLU); out is bf16 (outFp32 = 0) or fp32, row stride ldo.
int gemm_bf16(const void *A, const void *B, int M, int N, int K, const float *bias, int relu, void *out, int outFp32,
              int ldo, int *errorFlag, cudaStream_t stream, std::string &err);

// Features of `count` states (n <= 32) into X [count x 1088] bf16: state s reads spi/pi at
// spi + s*rowStride, pi + s*rowStride and its size at n[s*nStride].
void build_features(const uint8_t *spi, const uint8_t *pi, const uint8_t *n, int rowStride, int nStride, int count,
                    __nv_bfloat16 *X, cudaStream_t stream);
// Row-wise masked softmax cross-entropy over the first kTriples columns of logits
// [rows x ld] (columns whose triple has k >= n are masked); writes dlogits (bf16, already
// divided by rows) and per-row loss.
void softmax_xent(const float *logits, int ld, const uint8_t *n, const int32_t *target, int rows,
                  __nv_bfloat16 *dlogits, float *loss, cudaStream_t stream);
void transpose_bf16(const __nv_bfloat16 *in, int rows, int cols, __nv_bfloat16 *out, cudaStream_t stream);
void relu_backward(__nv_bfloat16 *grad, const __nv_bfloat16 *act, size_t count, cudaStream_t stream);
void column_sums(const __nv_bfloat16 *grad, int rows, int cols, float *out, cudaStream_t stream);
void adam_step(float *master, __nv_bfloat16 *weight, const float *grad, float *m, float *v, size_t count, float lr,
               float beta1, float beta2, float eps, int step, cudaStream_t stream);
// Per instance: the n-space lexicographic triple indices ordered by descending score.
void order_by_score(const float *scores, int ld, const uint8_t *n, int nStride, int count, uint16_t *order,
                    int orderStride, cudaStream_t stream);
// States after the first k1 children of each instance's root order: rows s*k1 + r of
// outSpi/outPi (64 bytes) and outN (0 when the root has fewer than r + 1 triples).
void level1_states(const uint8_t *spi, const uint8_t *pi, const uint8_t *n, int rowStride, int nStride, int count,
                   const uint16_t *order, int orderStride, int k1, uint8_t *outSpi, uint8_t *outPi, uint8_t *outN,
                   cudaStream_t stream);
// Per state: the k best-scoring n-space triple indices, best first (0xFFFF past the triples).
void top_k(const float *scores, int ld, const uint8_t *n, int nStride, int count, int k, uint16_t *out, int outStride,
           cudaStream_t stream);

}  // namespace mlp
}  // namespace tdp
