// Measurement helper (no counterpart in the reference): the L2 atomic throughput that bounds
// the transposition table's claims and depth updates.  Every thread issues returning 32-bit
// atomics (atomicCAS, as a table claim does, or atomicAdd) at pseudo-random 32-byte entries
// of a device buffer of `entries` entries, one atomic per entry touched, and the kernel is
// timed with CUDA events.  With entries * 32 bytes below the L2 size (126 MB on B200) every
// atomic resolves in L2; that rate is the atomic roof bench.py reports the engine against.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/tdp1375.h"

namespace {

__global__ void __launch_bounds__(256) l2_atomic_kernel(unsigned *buf, uint32_t mask, int iters, int useCas,
                                                        unsigned *sink) {
    uint32_t x = (blockIdx.x * blockDim.x + threadIdx.x) * 2654435761u + 0x9E3779B9u;
    unsigned acc = 0;
    for (int i = 0; i < iters; ++i) {
        x ^= x << 13;
        x ^= x >> 17;
        x ^= x << 5;
        unsigned *p = buf + (size_t)(x & mask) * 8u;  // the first word of a 32-byte entry
        acc += useCas ? atomicCAS(p, acc, acc + 1u) : atomicAdd(p, 1u);
    }
    if (acc == 0xFFFFFFFFu) *sink = acc;  // keeps the returned values live
}

thread_local std::string gMeasureError;

}  // namespace

extern "C" const char *tdp_measure_last_error(void) { return gMeasureError.c_str(); }

extern "C" int tdp_measure_atomics(int64_t entries, int use_cas, int iters, double *atomics_per_s) {
    if (entries < 1024 || (entries & (entries - 1)) != 0 || entries > (int64_t(1) << 31) || iters <= 0 ||
        !atomics_per_s) {
        gMeasureError = "tdp_measure_atomics: entries must be a power of two in [1024, 2^31], iters > 0";
        return TDP_ERR_ARGUMENT;
    }
    unsigned *buf = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int sms = 0, dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaMalloc(&buf, (size_t)entries * 32 + 64);
    if (e == cudaSuccess) e = cudaMemset(buf, 0, (size_t)entries * 32 + 64);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    float ms = 0.f;
    const int blocks = sms * 8;
    if (e == cudaSuccess) {
        unsigned *sink = buf + (size_t)entries * 8;
        l2_atomic_kernel<<<blocks, 256>>>(buf, (uint32_t)(entries - 1), iters, use_cas, sink);  // warm-up
        cudaEventRecord(e0);
        l2_atomic_kernel<<<blocks, 256>>>(buf, (uint32_t)(entries - 1), iters, use_cas, sink);
        cudaEventRecord(e1);
        e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (buf) cudaFree(buf);
    if (e != cudaSuccess) {
        gMeasureError = std::string("tdp_measure_atomics: ") + cudaGetErrorString(e);
        return TDP_ERR_CUDA;
    }
    *atomics_per_s = (double)blocks * 256.0 * (double)iters / ((double)ms * 1e-3);
    return 0;
}
