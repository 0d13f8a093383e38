// BF16 GEMM on the 5th-generation tensor cores (tcgen05 + TMEM + TMA) for the move-ordering
// MLP, and the small element-wise kernels of its training step.  No reference counterpart:
// the reference has no learned component.
//
//   C[M x N] (fp32 accumulate in TMEM) = A[M x K] * B[N x K]^T
//
// A and B are row-major bf16 with K contiguous (B has the torch.nn.Linear weight layout
// [out, in]).  One CTA computes one 128 x 256 tile:
//   warp 0 lane 0  TMA producer: 2-D tiled copies of 128x64 (A) and 256x64 (B) boxes with
//                  128-byte swizzle into a 4-stage shared-memory ring;
//   warp 1 lane 0  MMA issuer: four tcgen05.mma.kind::f16 (M=128, N=256, K=16) per stage,
//                  tcgen05.commit frees the stage, a final commit signals the epilogue;
//   warps 0-3      epilogue: tcgen05.ld 32 columns at a time from their TMEM lane quadrant,
//                  bias + ReLU, bf16 or fp32 stores.
// Every mbarrier wait is bounded by a 2 s deadline; on expiry the kernel records an error,
// skips the remaining tensor-core work and still frees its TMEM.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "mlp.h"

namespace tdp {
namespace mlp {
namespace {

constexpr int BM = 128, BN = 256, BK = 64, STAGES = 4;
constexpr int A_BYTES = BM * BK * 2;
constexpr int B_BYTES = BN * BK * 2;
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
constexpr unsigned long long kWaitNs = 2000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// Bounded wait for the completion of the phase with the given parity.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int *err) {
    const unsigned long long start = now_ns();
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        if (now_ns() - start > kWaitNs) {
            atomicExch(err, 1);
            return false;
        }
    }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);        // start address
    d |= (uint64_t)1u << 16;                        // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024u >> 4) << 32;              // stride byte offset
    d |= (uint64_t)1u << 46;                        // descriptor version (sm_100)
    d |= (uint64_t)2u << 61;                        // SWIZZLE_128B
    return d;
}

// Instruction descriptor: kind::f16, A/B bf16, D fp32, both K-major, M=128, N=256.
__host__ __device__ constexpr uint32_t instr_desc() {
    return (1u << 4)              // D format f32
           | (1u << 7)            // A format bf16
           | (1u << 10)           // B format bf16
           | ((uint32_t)(BN >> 3) << 17)
           | ((uint32_t)(BM >> 4) << 24);
}

__global__ void __launch_bounds__(128, 1)
    gemm_bf16_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                     const GemmParams p) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + STAGES * STAGE_BYTES);
    uint64_t *empty = full + STAGES;
    uint64_t *done = empty + STAGES;
    uint32_t *tmemSlot = reinterpret_cast<uint32_t *>(done + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tileN = blockIdx.x, tileM = blockIdx.y;
    const int kTiles = (p.K + BK - 1) / BK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(smem_u32(full + s), 1);
            mbar_init(smem_u32(empty + s), 1);
        }
        mbar_init(smem_u32(done), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmemSlot)),
                     "r"(BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmemSlot;

    if (warp == 0 && lane == 0) {
        for (int kt = 0; kt < kTiles; ++kt) {
            const int s = kt % STAGES, round = kt / STAGES;
            // a timed-out wait has set p.error; the later waits give up the same way
            if (round > 0 && !mbar_wait(smem_u32(empty + s), (uint32_t)((round - 1) & 1), p.error)) break;
            const uint32_t a = smem_u32(smem + s * STAGE_BYTES);
            const uint32_t b = a + A_BYTES;
            mbar_expect_tx(smem_u32(full + s), STAGE_BYTES);
            tma_load_2d(a, &tmA, kt * BK, tileM * BM, smem_u32(full + s));
            tma_load_2d(b, &tmB, kt * BK, tileN * BN, smem_u32(full + s));
        }
    } else if (warp == 1 && lane == 0) {
        constexpr uint32_t idesc = instr_desc();
        bool ok = true;
        for (int kt = 0; kt < kTiles && ok; ++kt) {
            const int s = kt % STAGES, round = kt / STAGES;
            if (!mbar_wait(smem_u32(full + s), (uint32_t)(round & 1), p.error)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a = smem_u32(smem + s * STAGE_BYTES);
            const uint32_t b = a + A_BYTES;
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk) {
                const uint64_t da = smem_desc(a + kk * 32);
                const uint64_t db = smem_desc(b + kk * 32);
                const uint32_t accumulate = (kt > 0 || kk > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(empty + s))
                         : "memory");
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(done))
                     : "memory");
    }
    __syncwarp();

    // Epilogue: every thread owns one row (TMEM lane) of the tile.
    const bool ready = mbar_wait(smem_u32(done), 0u, p.error);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int row = tileM * BM + warp * 32 + lane;
    if (ready) {
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 32) {
            uint32_t r[32];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                  "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                  "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < p.M) {
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int col = tileN * BN + c0 + j;
                    if (col < p.N) {
                        float v = __uint_as_float(r[j]);
                        if (p.bias) v += p.bias[col];
                        if (p.relu) v = fmaxf(v, 0.0f);
                        const size_t o = (size_t)row * (size_t)p.ldo + (size_t)col;
                        if (p.outF32) p.outF32[o] = v;
                        if (p.outBf16) p.outBf16[o] = __float2bfloat16_rn(v);
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN) : "memory");
    }
}

// ---------------------------------------------------------------- tensor maps
using EncodeFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                              const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encode_fn(std::string &err) {
    static std::mutex mu;
    static EncodeFn fn = nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!fn) {
        void *ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !ptr) {
            err = "cuTensorMapEncodeTiled is not available";
            return nullptr;
        }
        fn = reinterpret_cast<EncodeFn>(ptr);
    }
    return fn;
}

// rows x cols bf16 row-major (cols contiguous), box = boxRows x 64 columns, 128B swizzle.
bool make_map(CUtensorMap *map, const void *base, int rows, int cols, int boxRows, std::string &err) {
    EncodeFn fn = encode_fn(err);
    if (!fn) return false;
    if ((reinterpret_cast<uintptr_t>(base) & 15u) != 0 || (cols % 8) != 0) {
        err = "gemm operand must be 16-byte aligned with a row length that is a multiple of 8";
        return false;
    }
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
    const cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)boxRows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        err = "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")";
        return false;
    }
    return true;
}

}  // namespace

int prepare(std::string &err) {
    static std::once_flag attrOnce;
    static cudaError_t attrErr = cudaSuccess;
    std::call_once(attrOnce, [] {
        attrErr = cudaFuncSetAttribute(gemm_bf16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    });
    if (attrErr != cudaSuccess) {
        err = std::string("gemm set-up: ") + cudaGetErrorString(attrErr);
        return -3;
    }
    return encode_fn(err) ? 0 : -1;
}

int gemm_bf16(const void *A, const void *B, int M, int N, int K, const float *bias, int relu, void *out, int outFp32,
              int ldo, int *errorFlag, cudaStream_t stream, std::string &err) {
    if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !out || !errorFlag) {
        err = "gemm: bad arguments";
        return -1;
    }
    CUtensorMap ma, mb;
    if (!make_map(&ma, A, M, K, BM, err) || !make_map(&mb, B, N, K, BN, err)) return -1;
    if (prepare(err) != 0) return -3;
    GemmParams p{};
    p.M = M;
    p.N = N;
    p.K = K;
    p.bias = bias;
    p.relu = relu;
    p.outBf16 = outFp32 ? nullptr : static_cast<__nv_bfloat16 *>(out);
    p.outF32 = outFp32 ? static_cast<float *>(out) : nullptr;
    p.ldo = ldo > 0 ? ldo : N;
    p.error = errorFlag;
    const dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
    gemm_bf16_kernel<<<grid, 128, SMEM_BYTES, stream>>>(ma, mb, p);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        err = std::string("gemm launch: ") + cudaGetErrorString(e);
        return -3;
    }
    return 0;
}

}  // namespace mlp
}  // namespace tdp
