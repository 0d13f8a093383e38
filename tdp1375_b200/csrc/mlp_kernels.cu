// Element-wise and row kernels of the move-ordering MLP (features, loss, optimiser, order).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>

#include "mlp.h"
#include "tdp_math.cuh"

namespace tdp {
namespace mlp {
namespace {

// Lexicographic index of (i<j<k) among the triples of 32 positions.
__host__ __device__ __forceinline__ int lex32(int i, int j, int k) {
    // triples before first index i, then before second index j (given i), then k
    int idx = 0;
    for (int a = 0; a < i; ++a) idx += (31 - a) * (30 - a) / 2;
    for (int b = i + 1; b < j; ++b) idx += 31 - b;
    return idx + (k - j - 1);
}

__global__ void features_kernel(const uint8_t *spi, const uint8_t *pi, const uint8_t *nArr, int rowStride,
                                int nStride, int count, __nv_bfloat16 *X) {
    const int s = blockIdx.x;
    if (s >= count) return;
    __shared__ uint8_t sp[32], pp[32], pos[32];
    __shared__ int hist[64];
    const int n = min((int)nArr[(size_t)s * nStride], 32);
    const int t = threadIdx.x;
    if (t < 32) {
        sp[t] = t < n ? spi[(size_t)s * rowStride + t] : (uint8_t)t;
        pp[t] = t < n ? pi[(size_t)s * rowStride + t] : (uint8_t)t;
    }
    if (t < 64) hist[t] = 0;
    __syncthreads();
    if (t < 32) pos[pp[t]] = (uint8_t)t;
    __syncthreads();
    // adjacency in pi-position coordinates: row i = position of x, column j = position of spi(x)
    for (int e = t; e < 1024; e += blockDim.x) {
        const int i = e >> 5, j = e & 31;
        float v = 0.f;
        if (i < n && j < n && pos[sp[pp[i]]] == j) v = 1.f;
        X[(size_t)s * kFeatures + e] = __float2bfloat16_rn(v);
    }
    if (t < n) {
        // cycle length of symbol t, counted once at the cycle's smallest symbol
        int len = 1, m = t, cur = sp[t];
        while (cur != t && len < 64) {
            m = min(m, (int)cur);
            cur = sp[cur];
            ++len;
        }
        if (m == t) atomicAdd(&hist[len - 1], 1);
    }
    __syncthreads();
    if (t < 64) X[(size_t)s * kFeatures + 1024 + t] = __float2bfloat16_rn((float)hist[t]);
}

__device__ __forceinline__ float warp_max(float v) {
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
    return v;
}
__device__ __forceinline__ float warp_sum(float v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

__global__ void softmax_xent_kernel(const float *logits, int ld, const uint8_t *nArr, const int32_t *target, int rows,
                                    __nv_bfloat16 *dlogits, float *loss) {
    const int r = blockIdx.x;
    if (r >= rows) return;
    const int n = nArr[r];
    __shared__ float red[32];
    const float *row = logits + (size_t)r * ld;
    // column c = lex32(i,j,k) is valid when k < n; validity via a per-column decode is
    // costly, so decode once per column with the inverse walk below.
    float mx = -FLT_MAX;
    for (int c = threadIdx.x; c < kTriples; c += blockDim.x) {
        // decode c -> (i,j,k) by counting
        int rem = c, i = 0;
        while (i < 29 && rem >= (31 - i) * (30 - i) / 2) rem -= (31 - i) * (30 - i) / 2, ++i;
        int j = i + 1;
        while (j < 30 && rem >= 31 - j) rem -= 31 - j, ++j;
        const int k = j + 1 + rem;
        if (k < n) mx = fmaxf(mx, row[c]);
    }
    mx = warp_max(mx);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x < 32) {
        float v = threadIdx.x < blockDim.x / 32 ? red[threadIdx.x] : -FLT_MAX;
        v = warp_max(v);
        if (threadIdx.x == 0) red[0] = v;
    }
    __syncthreads();
    mx = red[0];
    __syncthreads();
    float sum = 0.f;
    for (int c = threadIdx.x; c < kTriples; c += blockDim.x) {
        int rem = c, i = 0;
        while (i < 29 && rem >= (31 - i) * (30 - i) / 2) rem -= (31 - i) * (30 - i) / 2, ++i;
        int j = i + 1;
        while (j < 30 && rem >= 31 - j) rem -= 31 - j, ++j;
        const int k = j + 1 + rem;
        if (k < n) sum += __expf(row[c] - mx);
    }
    sum = warp_sum(sum);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x < 32) {
        float v = threadIdx.x < blockDim.x / 32 ? red[threadIdx.x] : 0.f;
        v = warp_sum(v);
        if (threadIdx.x == 0) red[0] = v;
    }
    __syncthreads();
    sum = red[0];
    const int tgt = target[r];
    const float inv = 1.f / (float)rows;
    for (int c = threadIdx.x; c < ld; c += blockDim.x) {
        float g = 0.f;
        if (c < kTriples) {
            int rem = c, i = 0;
            while (i < 29 && rem >= (31 - i) * (30 - i) / 2) rem -= (31 - i) * (30 - i) / 2, ++i;
            int j = i + 1;
            while (j < 30 && rem >= 31 - j) rem -= 31 - j, ++j;
            const int k = j + 1 + rem;
            if (k < n) g = __expf(row[c] - mx) / sum - (c == tgt ? 1.f : 0.f);
        }
        dlogits[(size_t)r * ld + c] = __float2bfloat16_rn(g * inv);
    }
    if (threadIdx.x == 0) loss[r] = -(row[tgt] - mx - __logf(sum));
}

__global__ void transpose_kernel(const __nv_bfloat16 *in, int rows, int cols, __nv_bfloat16 *out) {
    __shared__ __nv_bfloat16 tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int r = by + y, c = bx + threadIdx.x;
        if (r < rows && c < cols) tile[y][threadIdx.x] = in[(size_t)r * cols + c];
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int r = bx + y, c = by + threadIdx.x;  // out is cols x rows
        if (r < cols && c < rows) out[(size_t)r * rows + c] = tile[threadIdx.x][y];
    }
}

__global__ void relu_backward_kernel(__nv_bfloat16 *grad, const __nv_bfloat16 *act, size_t count) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
        if (__bfloat162float(act[i]) <= 0.f) grad[i] = __float2bfloat16_rn(0.f);
}

__global__ void column_sums_kernel(const __nv_bfloat16 *grad, int rows, int cols, float *out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.f;
    for (int r = 0; r < rows; ++r) s += __bfloat162float(grad[(size_t)r * cols + c]);
    out[c] = s;
}

__global__ void adam_kernel(float *master, __nv_bfloat16 *weight, const float *grad, float *m, float *v, size_t count,
                            float lr, float b1, float b2, float eps, float c1, float c2) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
        const float g = grad[i];
        const float mi = b1 * m[i] + (1.f - b1) * g;
        const float vi = b2 * v[i] + (1.f - b2) * g * g;
        m[i] = mi;
        v[i] = vi;
        const float w = master[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        master[i] = w;
        weight[i] = __float2bfloat16_rn(w);
    }
}

// One block per instance: bitonic sort of (score, n-space index) pairs, 8192 slots.
__global__ void __launch_bounds__(1024) order_kernel(const float *scores, int ld, const uint8_t *nArr, int nStride,
                                                      int count, uint16_t *order, int orderStride) {
    const int s = blockIdx.x;
    if (s >= count) return;
    __shared__ float key[8192];
    __shared__ uint16_t val[8192];
    const int n = min((int)nArr[(size_t)s * nStride], 32);
    const int T = combinations3(n);
    int size = 1;
    while (size < T) size <<= 1;
    for (int t = threadIdx.x; t < size; t += blockDim.x) {
        float k = -FLT_MAX;
        uint16_t idx = 0xFFFF;
        if (t < T) {
            // n-space lexicographic index t -> (i, j, k)
            int rem = t, i = 0;
            while (i < n - 3 && rem >= (n - 1 - i) * (n - 2 - i) / 2) rem -= (n - 1 - i) * (n - 2 - i) / 2, ++i;
            int j = i + 1;
            while (j < n - 2 && rem >= n - 1 - j) rem -= n - 1 - j, ++j;
            const int kk = j + 1 + rem;
            k = scores[(size_t)s * ld + lex32(i, j, kk)];
            idx = (uint16_t)t;
        }
        key[t] = k;
        val[t] = idx;
    }
    __syncthreads();
    for (int len = 2; len <= size; len <<= 1) {
        for (int stride = len >> 1; stride > 0; stride >>= 1) {
            for (int t = threadIdx.x; t < size; t += blockDim.x) {
                const int partner = t ^ stride;
                if (partner > t) {
                    const bool desc = ((t & len) == 0);  // descending overall
                    const float a = key[t], b = key[partner];
                    const bool swap = desc ? (a < b || (a == b && val[t] > val[partner]))
                                           : (a > b || (a == b && val[t] < val[partner]));
                    if (swap) {
                        key[t] = b;
                        key[partner] = a;
                        const uint16_t u = val[t];
                        val[t] = val[partner];
                        val[partner] = u;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (int t = threadIdx.x; t < T; t += blockDim.x) order[(size_t)s * orderStride + t] = val[t];
}

// First-level states of the learned order: for instance s and rank r < K1 of its root
// order, the state after the root child order[r] (positions i<j<k of the root's pi array):
// spi' = spi o (a b c)^-1 with a, b, c = pi[i], pi[j], pi[k] (sorting_search.cu:543-555) and
// pi' = pi with [i,j) and [j,k) swapped (transposition.cuh:5-19).  Ranks past the root's
// triple count get n = 0.
__global__ void level1_states_kernel(const uint8_t *spi, const uint8_t *pi, const uint8_t *nArr, int rowStride,
                                     int nStride, int count, const uint16_t *order, int orderStride, int k1,
                                     uint8_t *outSpi, uint8_t *outPi, uint8_t *outN) {
    const int row = blockIdx.x;  // s * k1 + r
    const int s = row / k1, r = row % k1;
    if (s >= count) return;
    const int n = min((int)nArr[(size_t)s * nStride], 32);
    const int T = combinations3(n);
    const int p = threadIdx.x;  // 32 threads: one position / symbol each
    __shared__ int ijk[3];
    if (p == 0) {
        int rem = (r < T) ? (int)order[(size_t)s * orderStride + r] : 0, i = 0;
        while (i < n - 3 && rem >= (n - 1 - i) * (n - 2 - i) / 2) rem -= (n - 1 - i) * (n - 2 - i) / 2, ++i;
        int j = i + 1;
        while (j < n - 2 && rem >= n - 1 - j) rem -= n - 1 - j, ++j;
        ijk[0] = i;
        ijk[1] = j;
        ijk[2] = j + 1 + rem;
    }
    __syncthreads();
    const uint8_t *sp = spi + (size_t)s * rowStride, *pp = pi + (size_t)s * rowStride;
    uint8_t *os = outSpi + (size_t)row * 64, *op = outPi + (size_t)row * 64;
    const bool valid = r < T;
    if (p == 0) outN[row] = valid ? (uint8_t)n : (uint8_t)0;
    if (!valid || p >= n) {
        if (p < 32) os[p] = op[p] = 0;
        return;
    }
    const int i = ijk[0], j = ijk[1], k = ijk[2];
    const int a = pp[i], b = pp[j], c = pp[k];
    uint8_t v = sp[p];
    if (p == a) v = sp[c];
    if (p == b) v = sp[a];
    if (p == c) v = sp[b];
    os[p] = v;
    op[p] = pp[block_swap_src(p, i, j, k)];
}

// The K highest-scoring triples of each state (n-space lexicographic indices, ties to the
// smaller index, the order of order_kernel), by K rounds of a block arg-max; 0xFFFF pads
// states with fewer than K triples.
__global__ void __launch_bounds__(256) topk_kernel(const float *scores, int ld, const uint8_t *nArr, int nStride,
                                                   int count, int k, uint16_t *out, int outStride) {
    constexpr int kPer = 20;  // 256 * 20 >= C(32,3) = 4960
    const int s = blockIdx.x;
    if (s >= count) return;
    const int n = min((int)nArr[(size_t)s * nStride], 32);
    const int T = combinations3(n);
    float key[kPer];
#pragma unroll
    for (int e = 0; e < kPer; ++e) {
        const int t = threadIdx.x + 256 * e;
        key[e] = -FLT_MAX;
        if (t < T) {
            int rem = t, i = 0;
            while (i < n - 3 && rem >= (n - 1 - i) * (n - 2 - i) / 2) rem -= (n - 1 - i) * (n - 2 - i) / 2, ++i;
            int j = i + 1;
            while (j < n - 2 && rem >= n - 1 - j) rem -= n - 1 - j, ++j;
            key[e] = scores[(size_t)s * ld + lex32(i, j, j + 1 + rem)];
        }
    }
    unsigned taken = 0;
    __shared__ float bestKey[8];
    __shared__ int bestIdx[8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int round = 0; round < k; ++round) {
        float bk = -FLT_MAX;
        int bi = 0x7FFFFFFF;
#pragma unroll
        for (int e = 0; e < kPer; ++e) {
            const int t = threadIdx.x + 256 * e;
            if (t < T && !((taken >> e) & 1u) && (key[e] > bk || (key[e] == bk && t < bi))) {
                bk = key[e];
                bi = t;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float ok = __shfl_xor_sync(0xFFFFFFFFu, bk, o);
            const int oi = __shfl_xor_sync(0xFFFFFFFFu, bi, o);
            if (ok > bk || (ok == bk && oi < bi)) {
                bk = ok;
                bi = oi;
            }
        }
        if (lane == 0) {
            bestKey[warp] = bk;
            bestIdx[warp] = bi;
        }
        __syncthreads();
        bk = bestKey[0];
        bi = bestIdx[0];
        for (int w = 1; w < 8; ++w)
            if (bestKey[w] > bk || (bestKey[w] == bk && bestIdx[w] < bi)) {
                bk = bestKey[w];
                bi = bestIdx[w];
            }
        __syncthreads();
        if (threadIdx.x == 0) out[(size_t)s * outStride + round] = bi < T ? (uint16_t)bi : (uint16_t)0xFFFF;
        if (bi < T && (bi & 255) == (int)threadIdx.x) taken |= 1u << (bi >> 8);
    }
}

}  // namespace

void build_features(const uint8_t *spi, const uint8_t *pi, const uint8_t *n, int rowStride, int nStride, int count,
                    __nv_bfloat16 *X, cudaStream_t stream) {
    if (count > 0) features_kernel<<<count, 128, 0, stream>>>(spi, pi, n, rowStride, nStride, count, X);
}

void softmax_xent(const float *logits, int ld, const uint8_t *n, const int32_t *target, int rows,
                  __nv_bfloat16 *dlogits, float *loss, cudaStream_t stream) {
    if (rows > 0) softmax_xent_kernel<<<rows, 256, 0, stream>>>(logits, ld, n, target, rows, dlogits, loss);
}

void transpose_bf16(const __nv_bfloat16 *in, int rows, int cols, __nv_bfloat16 *out, cudaStream_t stream) {
    const dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
    transpose_kernel<<<grid, block, 0, stream>>>(in, rows, cols, out);
}

void relu_backward(__nv_bfloat16 *grad, const __nv_bfloat16 *act, size_t count, cudaStream_t stream) {
    relu_backward_kernel<<<1184, 256, 0, stream>>>(grad, act, count);
}

void column_sums(const __nv_bfloat16 *grad, int rows, int cols, float *out, cudaStream_t stream) {
    column_sums_kernel<<<(cols + 255) / 256, 256, 0, stream>>>(grad, rows, cols, out);
}

void adam_step(float *master, __nv_bfloat16 *weight, const float *grad, float *m, float *v, size_t count, float lr,
               float beta1, float beta2, float eps, int step, cudaStream_t stream) {
    const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
    adam_kernel<<<1184, 256, 0, stream>>>(master, weight, grad, m, v, count, lr, beta1, beta2, eps, c1, c2);
}

void order_by_score(const float *scores, int ld, const uint8_t *n, int nStride, int count, uint16_t *order,
                    int orderStride, cudaStream_t stream) {
    if (count > 0) order_kernel<<<count, 1024, 0, stream>>>(scores, ld, n, nStride, count, order, orderStride);
}

void level1_states(const uint8_t *spi, const uint8_t *pi, const uint8_t *n, int rowStride, int nStride, int count,
                   const uint16_t *order, int orderStride, int k1, uint8_t *outSpi, uint8_t *outPi, uint8_t *outN,
                   cudaStream_t stream) {
    if (count > 0 && k1 > 0)
        level1_states_kernel<<<count * k1, 32, 0, stream>>>(spi, pi, n, rowStride, nStride, count, order, orderStride,
                                                            k1, outSpi, outPi, outN);
}

void top_k(const float *scores, int ld, const uint8_t *n, int nStride, int count, int k, uint16_t *out, int outStride,
           cudaStream_t stream) {
    if (count > 0 && k > 0) topk_kernel<<<count, 256, 0, stream>>>(scores, ld, n, nStride, count, k, out, outStride);
}

}  // namespace mlp
}  // namespace tdp
