// Device generator of the extend step's one-3-cycle insertions (Extensions.java:95-141,
// Type 1 and Type 2 extensions of SortOrExtend's proof generator).
//
// A configuration is spi over n symbols with pi = (0 1 ... n-1).  An extension inserts a new
// unoriented 3-cycle before old positions a <= b <= c (not a = b = c): old position p moves
// to p + [a <= p] + [b <= p] + [c <= p], the new symbols sit at a, b + 1 and c + 2, and the
// new cycle runs from the largest of them downwards, as Configuration.ofSignature builds an
// unoriented cycle (Configuration.java:106-145).  The old cycles keep their order, relabelled.
// The reference produces
//   Type 1 (the configuration has open gates): for every open gate g and every b <= c, the
//     insertion at {g, b, c} (Extensions.java:95-116);
//   Type 2 (no open gate): every insertion (Extensions.java:118-141);
// so as a set Type 1 is every insertion whose positions include an open gate.  Open gates
// follow CommonOperations.getOpenGates (CommonOperations.java:501-546): symbol a with
// b = spi(a) is closed when an edge (c, spi(c)) of another cycle makes a, c, b, spi(c) cyclic
// in pi^-1, or a c of a's own cycle makes a, b, c cyclic in pi.
//
// Layout: slot e of configuration r enumerates the multisets a <= b <= c over [0, maxN) in
// lexicographic order (C(maxN + 2, 3) slots per configuration); flag[e] = 1 (Type 1),
// 2 (Type 2) or 0 (not an extension of this configuration), and the extended spi goes to a
// 64-byte row.  One warp builds a configuration's gate mask; one thread per slot writes a row.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/tdp1375.h"

namespace tdp {
namespace {

constexpr int kMaxIn = 60;  // n + 3 <= 63

__device__ __forceinline__ bool cyclic_positions(const int *p, int count) {
    int leaps = 0;
    for (int i = 0; i < count; ++i) leaps += p[i] > p[(i + 1) % count] ? 1 : 0;
    return leaps <= 1;
}

// One warp per configuration: bit a of gates[r] = symbol a is an open gate.
__global__ void open_gates_kernel(const uint8_t *spi, const uint8_t *nArr, int count, unsigned long long *gates) {
    const int r = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= count) return;
    const int n = nArr[r];
    const uint8_t *s = spi + (size_t)r * 64;
    __shared__ int leaderOf[8][64];
    int *leader = leaderOf[threadIdx.x >> 5];
    // cycle leader (smallest symbol) of every symbol, by walking the cycle (bounded by n)
    for (int x = lane; x < n; x += 32) {
        int m = x, cur = s[x];
        for (int it = 0; it < n && cur != x; ++it) {
            m = min(m, cur);
            cur = s[cur];
        }
        leader[x] = m;
    }
    __syncwarp();
    unsigned long long mask = 0;
    for (int a = lane; a < n; a += 32) {
        const int b = s[a];
        if (b == a) continue;  // only symbols of cycles of length > 1 can be gates
        bool closed = false;
        for (int c = 0; c < n && !closed; ++c) {
            if (s[c] == c) continue;
            if (leader[c] != leader[a]) {
                // another cycle's edge (c, spi(c)): a, c, b, spi(c) cyclic in pi^-1
                const int q[4] = {n - 1 - a, n - 1 - c, n - 1 - b, n - 1 - s[c]};
                closed = cyclic_positions(q, 4);
            } else if (c != a && c != b) {
                const int q[3] = {a, b, c};
                closed = cyclic_positions(q, 3);
            }
        }
        if (!closed) mask |= 1ull << a;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mask |= __shfl_xor_sync(0xFFFFFFFFu, mask, o);
    if (lane == 0) gates[r] = mask;
}

__global__ void insertion_kernel(const uint8_t *spi, const uint8_t *nArr, int count, int maxN,
                                 const unsigned long long *gates, uint8_t *flags, uint8_t *out) {
    const long long slots = (long long)(maxN + 2) * (maxN + 1) * maxN / 6;
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= slots * count) return;
    const int r = (int)(g / slots);
    int e = (int)(g - (long long)r * slots);
    // slot e -> multiset a <= b <= c over [0, maxN), lexicographic
    int a = 0;
    while (true) {
        const int m = maxN - a;  // multisets with this a: C(m + 1, 2)
        const int cnt = m * (m + 1) / 2;
        if (e < cnt) break;
        e -= cnt;
        ++a;
    }
    int b = a;
    while (e >= maxN - b) {
        e -= maxN - b;
        ++b;
    }
    const int c = b + e;
    const int n = nArr[r];
    uint8_t flag = 0;
    if (c < n && !(a == b && b == c)) {
        const unsigned long long gm = gates[r];
        if (gm == 0ull) {
            flag = 2;
        } else if (((gm >> a) | (gm >> b) | (gm >> c)) & 1ull) {
            flag = 1;
        }
    }
    flags[g] = flag;
    if (!flag) return;
    const uint8_t *s = spi + (size_t)r * 64;
    uint8_t *o = out + (size_t)g * 64;
    for (int p = 0; p < n; ++p) {
        const int q = s[p];
        const int mp = p + (a <= p) + (b <= p) + (c <= p);
        const int mq = q + (a <= q) + (b <= q) + (c <= q);
        o[mp] = (uint8_t)mq;
    }
    const int x = a, y = b + 1, z = c + 2;
    o[z] = (uint8_t)y;
    o[y] = (uint8_t)x;
    o[x] = (uint8_t)z;
    for (int p = n + 3; p < 64; ++p) o[p] = 0;
}

thread_local std::string gError;

}  // namespace
}  // namespace tdp

extern "C" const char *tdp_insertion_extensions_error(void) { return tdp::gError.c_str(); }

extern "C" int64_t tdp_insertion_extension_slots(int max_n) {
    if (max_n < 0) return 0;
    return (int64_t)(max_n + 2) * (max_n + 1) * max_n / 6;
}

extern "C" int tdp_insertion_extensions_device(const uint8_t *spi, const uint8_t *n, int count, int max_n,
                                               uint64_t *gates, uint8_t *flags, uint8_t *out, void *stream) {
    if (count < 0 || max_n < 1 || max_n > tdp::kMaxIn || (count > 0 && (!spi || !n || !gates || !flags || !out))) {
        tdp::gError = "tdp_insertion_extensions_device: need 1 <= max_n <= 60 and device buffers";
        return TDP_ERR_ARGUMENT;
    }
    if (count == 0) return 0;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    tdp::open_gates_kernel<<<(count + 7) / 8, 256, 0, s>>>(spi, n, count,
                                                          reinterpret_cast<unsigned long long *>(gates));
    const long long total = tdp_insertion_extension_slots(max_n) * (long long)count;
    const int threads = 256;
    tdp::insertion_kernel<<<(unsigned)((total + threads - 1) / threads), threads, 0, s>>>(
        spi, n, count, max_n, reinterpret_cast<const unsigned long long *>(gates), flags, out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        tdp::gError = std::string("tdp_insertion_extensions_device: ") + cudaGetErrorString(e);
        return TDP_ERR_CUDA;
    }
    return 0;
}
