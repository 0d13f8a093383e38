// Batched canonical form of configurations: Configuration.getCanonical / hashCode
// (Configuration.java:56-104, 147-195, 241-245, 290-303), one warp per configuration.
//
// A configuration is spi over symbols 0..n-1 (n <= 63), every symbol in a cycle of length
// >= 2, with pi = (0 1 ... n-1) (CANONICAL_PI).  Its 2n equivalent signatures are, for every
// start symbol r of pi, the signature under pi started at r (variant 2r) and the signature
// of the mirrored configuration (variant 2r+1: spi conjugated by the involution that swaps
// the symbols at pi positions i and n-1-i, then inverted).  The canonical signature is the
// one with the least hash (CRC32 of the big-endian float bytes, as a signed int), ties
// broken lexicographically, scanning the variants in the reference's order; the
// configuration's hash code is that hash.
//
// Per warp and row: the spi cycle tables (leader = smallest symbol, t = forward steps from
// the leader, L) go to shared memory once.  Per variant, each lane takes pi positions
// p = lane and lane + 32:
//  * its symbol's cycle in the variant (the mirror runs spi's cycles backwards through the
//    involution), the cycle's first position along pi (shared-memory atomicMin per cycle),
//    label = rank of that first position among the cycles' first positions, orientation =
//    more than one leap of pi^-1 positions around the cycle (atomicAdd per cycle), index of
//    an oriented symbol along the cycle from the symbol at the cycle's first position.
// Variants are built 32 at a time into a shared-memory block of rows; then the lanes switch to
// variants and each computes its row's CRC32 from a byte table.  The least hash, ties broken
// by the lexicographically least row, does not depend on the order the variants are
// scanned in, so the groups give the reference's answer.  The best row so far stays in
// shared memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>

#include "canonical.h"

namespace tdp {
namespace {

constexpr int kWarps = 4;   // warps (configurations) per block
constexpr int kMaxN = 63;   // two pi positions per lane
constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr uint32_t kPoly = 0xEDB88320u;  // reflected CRC-32 polynomial (java.util.zip.CRC32)

struct CanonArgs {
    const uint8_t *spi;  // rows of 64 bytes: successor array
    const uint8_t *n;    // per-row symbol count
    int count;
    float *sig;          // rows of 64 floats: canonical signature
    int32_t *hash;
    int32_t *variant;
};

constexpr int kRowPitch = 65;  // floats per row: an odd pitch keeps variant-major reads off one bank

struct WarpSmem {
    float rows[32][kRowPitch];  // the current group of up to 32 variant rows
    float best[64];
    uint8_t spi[64], inv[64], leader[64], t[64], len[64];
    int firstPos[64], leaps[64], anchorT[64], count[64];
};

__device__ __forceinline__ int mod_n(int x, int n) { return x >= n ? x - n : (x < 0 ? x + n : x); }

__global__ void __launch_bounds__(kWarps * 32) canonical_kernel(const CanonArgs A) {
    __shared__ uint32_t crcTable[256];
    __shared__ WarpSmem smem[kWarps];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        uint32_t c = (uint32_t)i;
        for (int k = 0; k < 8; ++k) c = (c >> 1) ^ (kPoly & (0u - (c & 1u)));
        crcTable[i] = c;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    WarpSmem &S = smem[threadIdx.x >> 5];
    for (int row = blockIdx.x * kWarps + (threadIdx.x >> 5); row < A.count; row += gridDim.x * kWarps) {
        const int n = A.n[row];
        const uint8_t *src = A.spi + (size_t)row * 64;
        // validity: 2 <= n <= 63, spi a permutation of 0..n-1 without fixed points; a bad row
        // gets variant -1, hash 0 and a zero signature
        S.count[lane] = 0;
        S.count[lane + 32] = 0;
        __syncwarp();
        bool bad = n < 2 || n > kMaxN;
        if (!bad) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int x = lane + 32 * h;
                if (x < n) {
                    const int s = src[x];
                    if (s >= n || s == x) {
                        bad = true;
                    } else {
                        atomicAdd(&S.count[s], 1);
                        S.spi[x] = (uint8_t)s;
                        S.inv[s] = (uint8_t)x;
                    }
                }
            }
        }
        __syncwarp();
        if (!bad) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int x = lane + 32 * h;
                if (x < n && S.count[x] != 1) bad = true;
            }
        }
        float *dst = A.sig + (size_t)row * 64;
        if (__any_sync(kFull, bad)) {
            dst[lane] = 0.f;
            dst[lane + 32] = 0.f;
            if (lane == 0) {
                A.hash[row] = 0;
                A.variant[row] = -1;
            }
            __syncwarp();
            continue;
        }
        // spi cycle tables: each lane walks the cycles of its symbols (length <= n)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int x = lane + 32 * h;
            if (x < n) {
                int m = x, steps = 0, L = 1;
                for (int y = S.spi[x]; y != x && L <= kMaxN; y = S.spi[y]) {
                    m = min(m, y);
                    ++L;
                }
                for (int y = x; y != m && steps <= kMaxN; y = S.spi[y]) ++steps;
                S.leader[x] = (uint8_t)m;
                S.t[x] = (uint8_t)(steps == 0 ? 0 : L - steps);
                S.len[x] = (uint8_t)L;
            }
        }
        __syncwarp();
        int32_t bestHash = INT32_MAX;
        int bestV = -1;
        for (int group = 0; group < 2 * n; group += 32) {
            const int nv = min(32, 2 * n - group);
            for (int k = 0; k < nv; ++k) {
                const int v = group + k;
                const int r = v >> 1;
                const bool mirror = v & 1;
                S.firstPos[lane] = 127;
                S.firstPos[lane + 32] = 127;
                S.leaps[lane] = 0;
                S.leaps[lane + 32] = 0;
                __syncwarp();
                int cid[2], tS[2], L[2];
                bool act[2];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int p = lane + 32 * h;
                    act[h] = p < n;
                    cid[h] = 0, tS[h] = 0, L[h] = 1;
                    if (act[h]) {
                        const int s = mod_n(r + p, n);
                        int succ;
                        if (!mirror) {
                            succ = S.spi[s];
                            cid[h] = S.leader[s];
                            tS[h] = S.t[s];
                            L[h] = S.len[s];
                        } else {
                            // c(x) = symbol at pi position n-1-pos(x); m(x) = c(spi^-1(c(x)))
                            const int cs = mod_n(r + (n - 1 - p), n);
                            const int pp = mod_n((int)S.inv[cs] - r, n);
                            succ = mod_n(r + (n - 1 - pp), n);
                            cid[h] = S.leader[cs];
                            L[h] = S.len[cs];
                            tS[h] = S.t[cs] == 0 ? 0 : L[h] - S.t[cs];  // m runs spi's cycle backwards
                        }
                        atomicMin(&S.firstPos[cid[h]], p);
                        // leap of pi^-1 positions: n-1-pos(s) > n-1-pos(succ) <=> pos(s) < pos(succ)
                        if (p < mod_n(succ - r, n)) atomicAdd(&S.leaps[cid[h]], 1);
                    }
                }
                __syncwarp();
                bool isFirst[2];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    isFirst[h] = act[h] && S.firstPos[cid[h]] == lane + 32 * h;
                    if (isFirst[h]) S.anchorT[cid[h]] = tS[h];
                }
                const uint64_t firsts = (uint64_t)__ballot_sync(kFull, isFirst[0]) |
                                        ((uint64_t)__ballot_sync(kFull, isFirst[1]) << 32);
                __syncwarp();
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    if (act[h]) {
                        const int fp = S.firstPos[cid[h]];
                        const uint64_t upTo = (fp >= 63) ? ~0ull : ((2ull << fp) - 1ull);
                        const int label = __popcll(firsts & upTo);
                        const bool oriented = S.leaps[cid[h]] > 1;
                        int idx = tS[h] - S.anchorT[cid[h]];
                        if (idx < 0) idx += L[h];
                        const float fl = __int2float_rn(label);
                        S.rows[k][lane + 32 * h] =
                            oriented ? __fadd_rn(fl, __fdiv_rn(__int2float_rn(idx + 1), 100.0f)) : fl;
                    }
                }
                __syncwarp();
            }
            // lanes = variants of the group: CRC32 of the row's big-endian float bytes
            int32_t h = INT32_MAX;
            if (lane < nv) {
                uint32_t crc = 0xFFFFFFFFu;
                for (int i = 0; i < n; ++i) {
                    const uint32_t bits = __float_as_uint(S.rows[lane][i]);
#pragma unroll
                    for (int b = 3; b >= 0; --b) crc = crcTable[(crc ^ (bits >> (8 * b))) & 0xFFu] ^ (crc >> 8);
                }
                h = (int32_t)(crc ^ 0xFFFFFFFFu);
            }
            const int32_t m = __reduce_min_sync(kFull, h);
            const unsigned cand = __ballot_sync(kFull, lane < nv && h == m);
            // Configuration.getCanonical: the least hash, ties by Arrays.compare
            if (lane == 0 && m <= bestHash) {
                unsigned c = cand;
                while (c) {
                    const int w = __ffs(c) - 1;
                    c &= c - 1u;
                    bool take = bestV < 0 || m < bestHash;
                    if (!take) {
                        for (int i = 0; i < n; ++i) {
                            const float a = S.rows[w][i], b = S.best[i];
                            if (a != b) {
                                take = a < b;
                                break;
                            }
                        }
                    }
                    if (take) {
                        bestHash = m;
                        bestV = group + w;
                        for (int i = 0; i < n; ++i) S.best[i] = S.rows[w][i];
                    }
                }
            }
            bestHash = __shfl_sync(kFull, bestHash, 0);
            bestV = __shfl_sync(kFull, bestV, 0);
            __syncwarp();
        }
        dst[lane] = lane < n ? S.best[lane] : 0.f;
        dst[lane + 32] = lane + 32 < n ? S.best[lane + 32] : 0.f;
        if (lane == 0) {
            A.hash[row] = bestHash;
            A.variant[row] = bestV;
        }
        __syncwarp();
    }
}

bool ok(cudaError_t e, std::string &err, const char *what) {
    if (e == cudaSuccess) return true;
    err = std::string(what) + ": CUDA error " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return false;
}

}  // namespace

int canonical_validate(const uint8_t *spi, const uint8_t *n, int count, std::string &err) {
    for (int r = 0; r < count; ++r) {
        const int m = n[r];
        if (m < 2 || m > kMaxN) {
            err = "tdp_canonical: row " + std::to_string(r) + ": n must be in 2..63";
            return -1;
        }
        uint64_t seen = 0;
        const uint8_t *s = spi + (size_t)r * 64;
        for (int x = 0; x < m; ++x) {
            if (s[x] >= m || ((seen >> s[x]) & 1ull) || s[x] == x) {
                err = "tdp_canonical: row " + std::to_string(r) +
                      ": spi must be a permutation of 0..n-1 without fixed points";
                return -1;
            }
            seen |= 1ull << s[x];
        }
    }
    return 0;
}

int canonical_device(const uint8_t *spiDev, const uint8_t *nDev, int count, float *sigDev, int32_t *hashDev,
                     int32_t *variantDev, cudaStream_t stream, std::string &err) {
    if (count < 0) {
        err = "tdp_canonical: count must be >= 0";
        return -1;
    }
    if (count == 0) return 0;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = (int)std::min<long long>(((long long)count + kWarps - 1) / kWarps, (long long)sms * 16);
    CanonArgs A{spiDev, nDev, count, sigDev, hashDev, variantDev};
    canonical_kernel<<<blocks, kWarps * 32, 0, stream>>>(A);
    if (!ok(cudaGetLastError(), err, "canonical launch")) return -3;
    return 0;
}

}  // namespace tdp
