// Permutation filter host entry (pi_filter.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace tdp {

// Returns the total number of hits (>= 0) or -1 bad argument, -3 CUDA error,
// -4 out of memory, -5 time limit; err receives the message.
int64_t pi_filter_run(const uint8_t *cycle, int cycleLen, const uint8_t *triple, int tripleLen, int n,
                      int skip2Move, uint8_t *out, int64_t maxRows, double timeLimitS, std::string &err);

// Device time (CUDA events around the kernels) of the calling thread's last pi_filter_run.
extern thread_local double gLastFilterKernelMs;

// Allocation-free variant (n <= 12): scratch is a static device array, rows go to a
// caller-provided device buffer, work runs on `stream`.  Same return convention.
int64_t pi_filter_noalloc_run(const uint8_t *cycle, int cycleLen, const uint8_t *triple, int tripleLen, int n,
                              int skip2Move, uint8_t *outDevice, int64_t maxRows, cudaStream_t stream,
                              std::string &err);

}  // namespace tdp
