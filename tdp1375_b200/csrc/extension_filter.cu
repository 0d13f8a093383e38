// Batched extension filter: the permutation-filter predicates of the reference
// (pi_filter.cu:55-115, CommonOperations.java:406-445) applied to every extension of many
// base configurations that adds one 3-cycle.  No reference counterpart as a batch: the
// reference filters the (n-1)! pi of a single cycle.
//
// Candidates of a base (spi, pi) over n symbols, in this order:
//   A. for every a<b<c (lexicographic) and orientation o: spi' = spi o rho with rho = (a b c)
//      (o = 0) or (a c b) (o = 1), pi' = pi; the added cycle is rho;
//   B. for every 0 <= g1 <= g2 <= g3 <= n (lexicographic) and orientation o: new symbols
//      x=n, y=n+1, z=n+2 inserted into pi before original positions g1, g2, g3 (x first on
//      ties), spi' = spi plus (x y z) (o = 0) or (x z y) (o = 1).
// Kept: the added cycle, as written, is in cyclic order in pi'; some cycle of spi' is
// oriented; no oriented cycle of spi' admits a 2-move.  One thread per candidate: it builds
// spi'/pi' positions in registers-backed local arrays (n' <= 63), walks the cycles once and
// tests each oriented cycle for a 2-move.  ALU-bound; the only traffic is one keep byte per
// candidate.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "extension_filter.h"

namespace tdp {
namespace {

constexpr int kThreads = 256;

struct ExtArgs {
    const uint8_t *spi;  // bases, rows of 64 bytes
    const uint8_t *pi;
    int n;
    int count;
    int perBase;
    int partA;
    uint8_t *keep;
};

__device__ __forceinline__ void decode_triple(int t, int n, int &i, int &j, int &k) {
    i = 0;
    while (i < n - 3 && t >= (n - 1 - i) * (n - 2 - i) / 2) t -= (n - 1 - i) * (n - 2 - i) / 2, ++i;
    j = i + 1;
    while (j < n - 2 && t >= n - 1 - j) t -= n - 1 - j, ++j;
    k = j + 1 + t;
}

__device__ __forceinline__ bool cyclic3(const uint8_t *index, int a, int b, int c) {
    const int ia = index[a], ib = index[b], ic = index[c];
    return ((ia > ib) + (ib > ic) + (ic > ia)) <= 1;
}

__device__ __forceinline__ bool cyclic_seq(const uint8_t *index, const uint8_t *sym, int count) {
    int leaps = 0;
    for (int i = 0; i < count; ++i) {
        const int nx = (i + 1 == count) ? 0 : i + 1;
        if (index[sym[i]] > index[sym[nx]] && ++leaps > 1) return false;
    }
    return true;
}

__device__ bool cycle_has_2_move(const uint8_t *index, const uint8_t *cyc, const uint8_t *cidx, int len) {
    const int before = len & 1;
    for (int i = 0; i < len - 2; ++i)
        for (int j = i + 1; j < len - 1; ++j)
            for (int k = j + 1; k < len; ++k) {
                const int a = cyc[i], b = cyc[j], c = cyc[k];
                if (!cyclic3(index, a, b, c)) continue;
                const int ai = cidx[a], bi = cidx[b], ci = cidx[c];
                const int kab = bi >= ai ? bi - ai : len - ai + bi;
                const int kbc = ci >= bi ? ci - bi : len - bi + ci;
                const int kca = ai >= ci ? ai - ci : len - ci + ai;
                if ((kab & 1) + (kbc & 1) + (kca & 1) - before == 2) return true;
            }
    return false;
}

__global__ void __launch_bounds__(kThreads) extension_filter_kernel(const ExtArgs A) {
    const long long gid = (long long)blockIdx.x * kThreads + threadIdx.x;
    if (gid >= (long long)A.count * A.perBase) return;
    const int base = (int)(gid / A.perBase);
    const int e = (int)(gid - (long long)base * A.perBase);
    const uint8_t *spi = A.spi + (size_t)base * 64;
    const uint8_t *pi = A.pi + (size_t)base * 64;
    const int n = A.n;
    uint8_t s2[64], p2[64], index[64], rindex[64], added[3];
    int m;
    if (e < A.partA) {
        const int t = e >> 1, o = e & 1;
        int a, b, c;
        decode_triple(t, n, a, b, c);
        const int r1 = o == 0 ? b : c, r2 = o == 0 ? c : b;
        for (int x = 0; x < n; ++x) {
            const int y = (x == a) ? r1 : (x == r1) ? r2 : (x == r2) ? a : x;
            s2[x] = spi[y];
            p2[x] = pi[x];
        }
        added[0] = (uint8_t)a, added[1] = (uint8_t)r1, added[2] = (uint8_t)r2;
        m = n;
    } else {
        const int t = (e - A.partA) >> 1, o = (e - A.partA) & 1;
        int i, j, k;
        decode_triple(t, n + 3, i, j, k);
        const int g0 = i, g1 = j - 1, g2 = k - 2;
        int q = 0;
        for (int pos = 0; pos <= n; ++pos) {
            if (g0 == pos) p2[q++] = (uint8_t)n;
            if (g1 == pos) p2[q++] = (uint8_t)(n + 1);
            if (g2 == pos) p2[q++] = (uint8_t)(n + 2);
            if (pos < n) p2[q++] = pi[pos];
        }
        for (int x = 0; x < n; ++x) s2[x] = spi[x];
        const int x = n, y = n + 1, z = n + 2;
        if (o == 0) {
            s2[x] = (uint8_t)y, s2[y] = (uint8_t)z, s2[z] = (uint8_t)x;
            added[0] = (uint8_t)x, added[1] = (uint8_t)y, added[2] = (uint8_t)z;
        } else {
            s2[x] = (uint8_t)z, s2[z] = (uint8_t)y, s2[y] = (uint8_t)x;
            added[0] = (uint8_t)x, added[1] = (uint8_t)z, added[2] = (uint8_t)y;
        }
        m = n + 3;
    }
    for (int q = 0; q < m; ++q) index[p2[q]] = (uint8_t)q;
    bool keep = cyclic3(index, added[0], added[1], added[2]);
    if (keep) {
        for (int s = 0; s < m; ++s) rindex[s] = (uint8_t)((m - 1) - index[s]);
        uint64_t seen = 0;
        bool anyOriented = false;
        for (int s = 0; s < m && keep; ++s) {
            if ((seen >> s) & 1ull) continue;
            uint8_t cyc[64], cidx[64];
            int len = 0, cur = s;
            do {
                seen |= 1ull << cur;
                cidx[cur] = (uint8_t)len;
                cyc[len++] = (uint8_t)cur;
                cur = s2[cur];
            } while (cur != s && len < 64);
            if (cyclic_seq(rindex, cyc, len)) continue;
            anyOriented = true;
            if (cycle_has_2_move(index, cyc, cidx, len)) keep = false;
        }
        keep = keep && anyOriented;
    }
    A.keep[gid] = keep ? 1 : 0;
}

bool ok(cudaError_t e, std::string &err, const char *what) {
    if (e == cudaSuccess) return true;
    err = std::string(what) + ": CUDA error " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return false;
}

int host_comb3(int n) { return n < 3 ? 0 : n * (n - 1) * (n - 2) / 6; }

}  // namespace

int extension_count(int n) { return 2 * host_comb3(n) + 2 * host_comb3(n + 3); }

int extension_filter_device(const uint8_t *spiDev, const uint8_t *piDev, int n, int count, uint8_t *keepDev,
                            cudaStream_t stream, std::string &err) {
    if (n < 3 || n + 3 > 63 || count < 0) {
        err = "tdp_extension_filter: n must be in 3..60";
        return -1;
    }
    if (count == 0) return 0;
    ExtArgs A{spiDev, piDev, n, count, extension_count(n), 2 * host_comb3(n), keepDev};
    const long long total = (long long)count * A.perBase;
    const int blocks = (int)((total + kThreads - 1) / kThreads);
    extension_filter_kernel<<<blocks, kThreads, 0, stream>>>(A);
    if (!ok(cudaGetLastError(), err, "extension filter launch")) return -3;
    return 0;
}

}  // namespace tdp
