// Batched extension filter host entry (extension_filter.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace tdp {

// Candidates per base of n symbols: 2*C(n,3) + 2*C(n+3,3).
int extension_count(int n);
// Device buffers: bases (rows of 64 bytes), keep flags [count * extension_count(n)].
// 0 on success, -1 bad argument, -3 CUDA error.
int extension_filter_device(const uint8_t *spiDev, const uint8_t *piDev, int n, int count, uint8_t *keepDev,
                            cudaStream_t stream, std::string &err);

}  // namespace tdp
