// Batched canonical form of configurations (Configuration.getCanonical / hashCode).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

namespace tdp {

// Host-side check of rows (64-byte successor arrays, n[r] symbols each): n in 2..63 and
// spi a permutation of 0..n-1 without fixed points.  Returns 0 or -1 with err set.
int canonical_validate(const uint8_t *spi, const uint8_t *n, int count, std::string &err);

// Device buffers: spi rows (64 B), n (count bytes), sig rows (64 floats), hash, variant.
int canonical_device(const uint8_t *spiDev, const uint8_t *nDev, int count, float *sigDev, int32_t *hashDev,
                     int32_t *variantDev, cudaStream_t stream, std::string &err);

}  // namespace tdp
