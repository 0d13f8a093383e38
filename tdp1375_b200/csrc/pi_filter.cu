// Permutation filter (replaces pi_filter_kernel / performGpuPiFilter, pi_filter.cu:38-260).
//
// Every pi with pi[0] = 0 over n symbols is visited in lexicographic order of
// pi[1..n-1] (the factoradic rank order of pi_filter.cu:38-53) and kept when
//   (1) the oriented triple is in cyclic order in pi           (pi_filter.cu:132-133),
//   (2) the cycle is NOT in cyclic order in pi reversed        (pi_filter.cu:135-142,
//       CommonOperations.isOriented, CommonOperations.java:443-445),
//   (3) unless skipped, the cycle admits no 2-move             (pi_filter.cu:86-115,
//       CommonOperations.java:406-431).
// B200 layout: each thread walks kRanksPerThread consecutive ranks (one factoradic unrank,
// then next-permutation steps), so the O(n^2) divisions of the reference happen once per
// 16 candidates.  Hits are written in rank order: a counting pass stores per-thread hit
// counts and a block-exclusive prefix, one block scans the block totals, and a writing
// pass re-evaluates and stores rows at their final offsets.  The reference appends with
// one atomicAdd per hit in arbitrary order.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "pi_filter.h"

namespace tdp {

thread_local double gLastFilterKernelMs = 0.0;

namespace {

constexpr int kThreads = 256;
constexpr int kRanksPerThread = 16;
constexpr int kRanksPerBlock = kThreads * kRanksPerThread;
constexpr uint64_t kLaunchRanks = 1ull << 30;

struct FilterArgs {
    uint8_t cycle[64];
    uint8_t triple[64];
    uint8_t cycleIndex[64];
    unsigned long long fact[21];
    int cycleLen;
    int tripleLen;
    int n;
    int skip2Move;
    unsigned long long base;   // first rank of this launch
    unsigned long long total;  // (n-1)!
};

__device__ __forceinline__ bool cyclic_order(const uint8_t *index, const uint8_t *symbols, int count) {
    int leaps = 0;
    for (int i = 0; i < count; ++i) {
        const int next = (i + 1 == count) ? 0 : i + 1;
        if (index[symbols[i]] > index[symbols[next]]) {
            if (++leaps > 1) return false;
        }
    }
    return true;
}

__device__ __forceinline__ bool cyclic_order3(const uint8_t *index, int a, int b, int c) {
    const int ia = index[a], ib = index[b], ic = index[c];
    return ((ia > ib) + (ib > ic) + (ic > ia)) <= 1;
}

__device__ __forceinline__ int cycle_distance(const uint8_t *cycleIndex, int len, int a, int b) {
    const int ai = cycleIndex[a], bi = cycleIndex[b];
    return (bi >= ai) ? bi - ai : (len - ai) + bi;
}

__device__ bool has_2_move(const FilterArgs &A, const uint8_t *index) {
    const int len = A.cycleLen;
    const int before = len & 1;
    for (int i = 0; i < len - 2; ++i)
        for (int j = i + 1; j < len - 1; ++j)
            for (int k = j + 1; k < len; ++k) {
                const int a = A.cycle[i], b = A.cycle[j], c = A.cycle[k];
                if (!cyclic_order3(index, a, b, c)) continue;
                const int after = (cycle_distance(A.cycleIndex, len, a, b) & 1) +
                                  (cycle_distance(A.cycleIndex, len, b, c) & 1) +
                                  (cycle_distance(A.cycleIndex, len, c, a) & 1);
                if (after - before == 2) return true;
            }
    return false;
}

__device__ __forceinline__ void unrank(unsigned long long r, int n, const unsigned long long *fact, uint8_t *p) {
    uint8_t avail[64];
    for (int i = 0; i < n - 1; ++i) avail[i] = (uint8_t)(i + 1);
    p[0] = 0;
    for (int pos = 0; pos < n - 1; ++pos) {
        const unsigned long long f = fact[n - 2 - pos];
        const int choice = (int)(r / f);
        r -= (unsigned long long)choice * f;
        p[pos + 1] = avail[choice];
        for (int q = choice; q < n - 2 - pos; ++q) avail[q] = avail[q + 1];
    }
}

__device__ __forceinline__ void next_perm(uint8_t *p, int n) {
    int i = n - 2;
    while (i >= 1 && p[i] > p[i + 1]) --i;
    if (i < 1) return;
    int j = n - 1;
    while (p[j] < p[i]) --j;
    const uint8_t t = p[i];
    p[i] = p[j];
    p[j] = t;
    for (int l = i + 1, r = n - 1; l < r; ++l, --r) {
        const uint8_t u = p[l];
        p[l] = p[r];
        p[r] = u;
    }
}

__device__ __forceinline__ bool keep(const FilterArgs &A, const uint8_t *p, uint8_t *index, uint8_t *rindex) {
    const int n = A.n;
    for (int i = 0; i < n; ++i) index[p[i]] = (uint8_t)i;
    if (!cyclic_order(index, A.triple, A.tripleLen)) return false;
    for (int s = 0; s < n; ++s) rindex[s] = (uint8_t)((n - 1) - index[s]);
    if (cyclic_order(rindex, A.cycle, A.cycleLen)) return false;
    if (!A.skip2Move && has_2_move(A, index)) return false;
    return true;
}

// Block-wide exclusive scan of one value per thread; returns the prefix, total in *total.
__device__ __forceinline__ unsigned block_exclusive_scan(unsigned v, unsigned *total) {
    __shared__ unsigned warpSums[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warpSums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        unsigned s = (lane < kThreads / 32) ? warpSums[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xFFFFFFFFu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < kThreads / 32) warpSums[lane] = s;
    }
    __syncthreads();
    const unsigned before = (warp > 0 ? warpSums[warp - 1] : 0u) + x - v;
    *total = warpSums[kThreads / 32 - 1];
    __syncthreads();
    return before;
}

__global__ void __launch_bounds__(kThreads) pi_filter_count_kernel(const FilterArgs A, unsigned *threadPrefix,
                                                                    unsigned *blockTotal) {
    uint8_t p[64], index[64], rindex[64];
    const unsigned long long first =
        A.base + ((unsigned long long)blockIdx.x * kThreads + threadIdx.x) * kRanksPerThread;
    unsigned hits = 0;
    if (first < A.total) {
        unrank(first, A.n, A.fact, p);
        const unsigned long long last = min(first + kRanksPerThread, A.total);
        for (unsigned long long r = first; r < last; ++r) {
            hits += keep(A, p, index, rindex) ? 1u : 0u;
            next_perm(p, A.n);
        }
    }
    unsigned total;
    const unsigned prefix = block_exclusive_scan(hits, &total);
    threadPrefix[(size_t)blockIdx.x * kThreads + threadIdx.x] = prefix;
    if (threadIdx.x == 0) blockTotal[blockIdx.x] = total;
}

// One block: exclusive scan of the block totals (64-bit running offset).
__global__ void __launch_bounds__(kThreads) pi_filter_scan_kernel(const unsigned *blockTotal,
                                                                   unsigned long long *blockOffset, int blocks,
                                                                   unsigned long long *grandTotal) {
    __shared__ unsigned long long running;
    if (threadIdx.x == 0) running = *grandTotal;
    __syncthreads();
    for (int base = 0; base < blocks; base += kThreads) {
        const int i = base + (int)threadIdx.x;
        const unsigned v = (i < blocks) ? blockTotal[i] : 0u;
        unsigned tileTotal;
        const unsigned prefix = block_exclusive_scan(v, &tileTotal);
        if (i < blocks) blockOffset[i] = running + prefix;
        __syncthreads();
        if (threadIdx.x == 0) running += tileTotal;
        __syncthreads();
    }
    if (threadIdx.x == 0) *grandTotal = running;
}

__global__ void __launch_bounds__(kThreads) pi_filter_write_kernel(const FilterArgs A, const unsigned *threadPrefix,
                                                                    const unsigned long long *blockOffset,
                                                                    uint8_t *out, unsigned long long maxRows) {
    uint8_t p[64], index[64], rindex[64];
    const unsigned long long first =
        A.base + ((unsigned long long)blockIdx.x * kThreads + threadIdx.x) * kRanksPerThread;
    if (first >= A.total) return;
    unsigned long long row = blockOffset[blockIdx.x] + threadPrefix[(size_t)blockIdx.x * kThreads + threadIdx.x];
    if (row >= maxRows) return;
    unrank(first, A.n, A.fact, p);
    const unsigned long long last = min(first + kRanksPerThread, A.total);
    for (unsigned long long r = first; r < last && row < maxRows; ++r) {
        if (keep(A, p, index, rindex)) {
            uint8_t *dst = out + row * (unsigned long long)A.n;
            for (int i = 0; i < A.n; ++i) dst[i] = p[i];
            ++row;
        }
        next_perm(p, A.n);
    }
}

// ---------------------------------------------------------------- packed path (n <= 16)
// With n <= 16 a whole pi fits in one 64-bit register as 4-bit symbols (nibble p = pi[p]),
// and so does its inverse (nibble s = position of symbol s).  A thread walks kPackedRanks
// consecutive ranks with next-permutation steps on those two registers (a step rewrites
// only the suffix it permutes), so no per-thread arrays exist and nothing goes to local
// memory.  The predicates read positions straight from the inverse:
//   (1) triple in cyclic order in pi: at most one descent around the triple's positions;
//   (2) cycle oriented: the cycle is in cyclic order in reversed pi iff its positions have
//       at most one ascent around the cycle (reversal turns ascents into descents), so the
//       cycle is kept when it has two or more;
//   (3) 2-move: the cycle triples (i<j<k in cycle order) whose cycle-distance parities give
//       after - before == 2 do not depend on pi; the host lists them once (at most
//       C(16,3) = 560) and a pi has a 2-move iff one listed triple is in cyclic order.
constexpr int kPackedMaxN = 16;
constexpr int kPackedRanks = 32;
constexpr int kPackedRanksPerBlock = kThreads * kPackedRanks;
constexpr int kMaxTwoMoveTriples = 560;

struct PackedArgs {
    unsigned long long fact[17];
    unsigned long long base, total;
    uint8_t cycle[16];
    uint8_t triple[16];
    uint16_t twoMove[kMaxTwoMoveTriples];  // a | b << 4 | c << 8
    int cycleLen, tripleLen, n, skip2Move, twoMoveCount;
};

__device__ __forceinline__ uint32_t nib(unsigned long long w, uint32_t i) { return (uint32_t)(w >> (4u * i)) & 15u; }
__device__ __forceinline__ unsigned long long set_nib(unsigned long long w, uint32_t i, uint32_t v) {
    return (w & ~(15ull << (4u * i))) | ((unsigned long long)v << (4u * i));
}

__device__ __forceinline__ void packed_unrank(const PackedArgs &A, unsigned long long r, unsigned long long &pi,
                                              unsigned long long &inv) {
    // available symbols 1..n-1 as nibbles, removed one by one (Lehmer digits, highest first)
    const int n = A.n;
    unsigned long long avail = 0;
    for (int i = 0; i < n - 1; ++i) avail |= (unsigned long long)(i + 1) << (4 * i);
    pi = 0;
    inv = 0;
    for (int pos = 1; pos < n; ++pos) {
        const unsigned long long f = A.fact[n - 1 - pos];
        const uint32_t choice = (uint32_t)(r / f);
        r -= (unsigned long long)choice * f;
        const uint32_t sym = nib(avail, choice);
        const unsigned long long low = avail & ((1ull << (4 * choice)) - 1ull);
        const unsigned long long high = (choice + 1 < 16) ? (avail >> (4 * (choice + 1))) << (4 * choice) : 0ull;
        avail = low | high;
        pi = set_nib(pi, (uint32_t)pos, sym);
        inv = set_nib(inv, sym, (uint32_t)pos);
    }
}

// Lexicographic successor of pi[1..n-1] (pi[0] = 0 stays), updating the inverse.
__device__ __forceinline__ void packed_next(int n, unsigned long long &pi, unsigned long long &inv) {
    int i = n - 2;
    while (i >= 1 && nib(pi, i) > nib(pi, i + 1)) --i;
    if (i < 1) return;
    int j = n - 1;
    const uint32_t pv = nib(pi, i);
    while (nib(pi, j) < pv) --j;
    const uint32_t qv = nib(pi, j);
    pi = set_nib(set_nib(pi, i, qv), j, pv);
    for (int l = i + 1, r = n - 1; l < r; ++l, --r) {
        const uint32_t a = nib(pi, l), b = nib(pi, r);
        pi = set_nib(set_nib(pi, l, b), r, a);
    }
    for (int p = i; p < n; ++p) inv = set_nib(inv, nib(pi, p), (uint32_t)p);
}

__device__ __forceinline__ bool packed_keep(const PackedArgs &A, unsigned long long inv) {
    int leaps = 0;
    for (int t = 0; t < A.tripleLen; ++t) {
        const uint32_t a = nib(inv, A.triple[t]);
        const uint32_t b = nib(inv, A.triple[t + 1 == A.tripleLen ? 0 : t + 1]);
        leaps += a > b ? 1 : 0;
    }
    if (leaps > 1) return false;
    int ascents = 0;
    for (int t = 0; t < A.cycleLen; ++t) {
        const uint32_t a = nib(inv, A.cycle[t]);
        const uint32_t b = nib(inv, A.cycle[t + 1 == A.cycleLen ? 0 : t + 1]);
        ascents += a < b ? 1 : 0;
    }
    if (ascents <= 1) return false;
    if (A.skip2Move) return true;
    for (int t = 0; t < A.twoMoveCount; ++t) {
        const uint32_t w = A.twoMove[t];
        const uint32_t pa = nib(inv, w & 15u), pb = nib(inv, (w >> 4) & 15u), pc = nib(inv, (w >> 8) & 15u);
        if ((pa > pb) + (pb > pc) + (pc > pa) <= 1) return false;
    }
    return true;
}

__global__ void __launch_bounds__(kThreads) packed_count_kernel(const PackedArgs A, unsigned *threadPrefix,
                                                                 unsigned *blockTotal) {
    const unsigned long long first =
        A.base + ((unsigned long long)blockIdx.x * kThreads + threadIdx.x) * kPackedRanks;
    unsigned hits = 0;
    if (first < A.total) {
        unsigned long long pi, inv;
        packed_unrank(A, first, pi, inv);
        const unsigned long long last = min(first + kPackedRanks, A.total);
        for (unsigned long long r = first; r < last; ++r) {
            hits += packed_keep(A, inv) ? 1u : 0u;
            packed_next(A.n, pi, inv);
        }
    }
    unsigned total;
    const unsigned prefix = block_exclusive_scan(hits, &total);
    threadPrefix[(size_t)blockIdx.x * kThreads + threadIdx.x] = prefix;
    if (threadIdx.x == 0) blockTotal[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kThreads) packed_write_kernel(const PackedArgs A, const unsigned *threadPrefix,
                                                                 const unsigned long long *blockOffset, uint8_t *out,
                                                                 unsigned long long maxRows) {
    const unsigned long long first =
        A.base + ((unsigned long long)blockIdx.x * kThreads + threadIdx.x) * kPackedRanks;
    if (first >= A.total) return;
    const unsigned next = (threadIdx.x + 1 < kThreads)
                              ? threadPrefix[(size_t)blockIdx.x * kThreads + threadIdx.x + 1]
                              : 0xFFFFFFFFu;
    const unsigned mine = threadPrefix[(size_t)blockIdx.x * kThreads + threadIdx.x];
    if (next == mine) return;  // no hit among this thread's ranks
    unsigned long long row = blockOffset[blockIdx.x] + mine;
    if (row >= maxRows) return;
    unsigned long long pi, inv;
    packed_unrank(A, first, pi, inv);
    const unsigned long long last = min(first + kPackedRanks, A.total);
    for (unsigned long long r = first; r < last && row < maxRows; ++r) {
        if (packed_keep(A, inv)) {
            uint8_t *dst = out + row * (unsigned long long)A.n;
            for (int i = 0; i < A.n; ++i) dst[i] = (uint8_t)nib(pi, i);
            ++row;
        }
        packed_next(A.n, pi, inv);
    }
}

// The host half of the packed path: the pi-independent 2-move triple list
// (pi_filter.cu:86-115 restated: cycle positions i<j<k, cycle distances a->b, b->c, c->a).
int two_move_triples(const uint8_t *cycle, int len, uint16_t *out) {
    uint8_t index[64] = {};
    for (int i = 0; i < len; ++i) index[cycle[i]] = (uint8_t)i;
    auto dist = [&](int a, int b) {
        const int ai = index[a], bi = index[b];
        return (bi >= ai) ? bi - ai : (len - ai) + bi;
    };
    const int before = len & 1;
    int count = 0;
    for (int i = 0; i < len - 2; ++i)
        for (int j = i + 1; j < len - 1; ++j)
            for (int k = j + 1; k < len; ++k) {
                const int a = cycle[i], b = cycle[j], c = cycle[k];
                const int after = (dist(a, b) & 1) + (dist(b, c) & 1) + (dist(c, a) & 1);
                if (after - before == 2) out[count++] = (uint16_t)(a | (b << 4) | (c << 8));
            }
    return count;
}

// ---------------------------------------------------------------- allocation-free variant
// Scratch of tdp_pi_filter_noalloc, for callers that cannot allocate device memory: slot 0
// holds the hit total, slots [1, 1+B) the block offsets and [1+B, 1+2B) the block totals,
// B = number of 4096-rank blocks of 11! candidates (n <= 12).  Every GPU that loads the
// library keeps these 156 KB until the process exits.  In host code the symbol is only a
// stand-in: the device address comes from cudaGetSymbolAddress (noalloc_scratch below).
constexpr int kNoAllocMaxN = 12;
constexpr unsigned long long kNoAllocMaxRanks = 39916800ull;  // 11!
constexpr int kNoAllocMaxBlocks = (int)((kNoAllocMaxRanks + kRanksPerBlock - 1) / kRanksPerBlock);
static __device__ __align__(256) unsigned long long gNoAllocScratch[1 + 2 * kNoAllocMaxBlocks];

// Count pass without per-thread scratch: block totals only.
__global__ void __launch_bounds__(kThreads) noalloc_count_kernel(const FilterArgs A, unsigned long long *scratch,
                                                                  int blocks) {
    uint8_t p[64], index[64], rindex[64];
    const unsigned long long first = ((unsigned long long)blockIdx.x * kThreads + threadIdx.x) * kRanksPerThread;
    unsigned hits = 0;
    if (first < A.total) {
        unrank(first, A.n, A.fact, p);
        const unsigned long long last = min(first + kRanksPerThread, A.total);
        for (unsigned long long r = first; r < last; ++r) {
            hits += keep(A, p, index, rindex) ? 1u : 0u;
            next_perm(p, A.n);
        }
    }
    unsigned total;
    block_exclusive_scan(hits, &total);
    if (threadIdx.x == 0) scratch[1 + blocks + blockIdx.x] = total;
}

// One block: block offsets from the block totals; the hit total goes to scratch[0].
__global__ void __launch_bounds__(kThreads) noalloc_scan_kernel(unsigned long long *scratch, int blocks) {
    __shared__ unsigned long long running;
    if (threadIdx.x == 0) running = 0ull;
    __syncthreads();
    for (int base = 0; base < blocks; base += kThreads) {
        const int i = base + (int)threadIdx.x;
        const unsigned v = (i < blocks) ? (unsigned)scratch[1 + blocks + i] : 0u;
        unsigned tileTotal;
        const unsigned prefix = block_exclusive_scan(v, &tileTotal);
        if (i < blocks) scratch[1 + i] = running + prefix;
        __syncthreads();
        if (threadIdx.x == 0) running += tileTotal;
        __syncthreads();
    }
    if (threadIdx.x == 0) scratch[0] = running;
}

// Write pass: each thread recounts its ranks to find its offset inside the block, then
// re-walks them and stores the kept rows.
__global__ void __launch_bounds__(kThreads) noalloc_write_kernel(const FilterArgs A, const unsigned long long *scratch,
                                                                  uint8_t *out, unsigned long long maxRows) {
    uint8_t p[64], index[64], rindex[64];
    const unsigned long long first = ((unsigned long long)blockIdx.x * kThreads + threadIdx.x) * kRanksPerThread;
    const unsigned long long last = min(first + kRanksPerThread, A.total);
    unsigned hits = 0;
    if (first < A.total) {
        unrank(first, A.n, A.fact, p);
        for (unsigned long long r = first; r < last; ++r) {
            hits += keep(A, p, index, rindex) ? 1u : 0u;
            next_perm(p, A.n);
        }
    }
    unsigned total;
    const unsigned prefix = block_exclusive_scan(hits, &total);
    if (first >= A.total || hits == 0) return;
    unsigned long long row = scratch[1 + blockIdx.x] + prefix;
    if (row >= maxRows) return;
    unrank(first, A.n, A.fact, p);
    for (unsigned long long r = first; r < last && row < maxRows; ++r) {
        if (keep(A, p, index, rindex)) {
            uint8_t *dst = out + row * (unsigned long long)A.n;
            for (int i = 0; i < A.n; ++i) dst[i] = p[i];
            ++row;
        }
        next_perm(p, A.n);
    }
}

// Device address of gNoAllocScratch for the current device.  It is looked up
// (cudaGetSymbolAddress, with that device current) on the first call on a device and cached
// together with the device's current context, and looked up again when that context has
// changed (after cudaDeviceReset the old address is stale).
unsigned long long *noalloc_scratch(std::string &err) {
    using CtxGetCurrent = int (*)(void **);
    static std::mutex mu;
    static CtxGetCurrent ctxGetCurrent = nullptr;
    static void *ctxOf[64] = {};
    static unsigned long long *addr[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        err = "tdp_pi_filter_noalloc: no current CUDA device";
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (!ctxGetCurrent) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn) {
            err = "tdp_pi_filter_noalloc: cuCtxGetCurrent is not available";
            return nullptr;
        }
        ctxGetCurrent = reinterpret_cast<CtxGetCurrent>(fn);
    }
    void *ctx = nullptr;
    if (!addr[dev] || ctxGetCurrent(&ctx) != 0 || ctx != ctxOf[dev]) {
        void *ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, gNoAllocScratch);
        if (e != cudaSuccess || !ptr) {
            err = std::string("tdp_pi_filter_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e);
            return nullptr;
        }
        // the runtime has made the device's primary context current by now
        ctx = nullptr;
        if (ctxGetCurrent(&ctx) != 0) ctx = nullptr;
        ctxOf[dev] = ctx;
        addr[dev] = static_cast<unsigned long long *>(ptr);
    }
    return addr[dev];
}

struct DeviceBuffer {
    void *ptr = nullptr;
    ~DeviceBuffer() {
        if (ptr) cudaFree(ptr);
    }
};

bool ok(cudaError_t e, std::string &err, const char *what) {
    if (e == cudaSuccess) return true;
    err = std::string(what) + ": CUDA error " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return false;
}

}  // namespace

int64_t pi_filter_run(const uint8_t *cycle, int cycleLen, const uint8_t *triple, int tripleLen, int n,
                      int skip2Move, uint8_t *out, int64_t maxRows, double timeLimitS, std::string &err) {
    if (n > 63) {
        err = "n exceeds PI_FILTER_MAX_N";
        return -1;
    }
    if (n < 1) {
        err = "n must be at least 1";
        return -1;
    }
    if (n > 21) {
        err = "pi filter: (n-1)! does not fit in 64 bits for n > 21";
        return -1;
    }
    if (cycleLen < 0 || cycleLen > 63 || tripleLen < 0 || tripleLen > 63 || maxRows < 0) {
        err = "pi filter: invalid cycle/triple length or row limit";
        return -1;
    }
    for (int i = 0; i < cycleLen; ++i)
        if (cycle[i] >= n) {
            err = "pi filter: cycle symbol out of range";
            return -1;
        }
    for (int i = 0; i < tripleLen; ++i)
        if (triple[i] >= n) {
            err = "pi filter: triple symbol out of range";
            return -1;
        }
    FilterArgs A;
    std::memset(&A, 0, sizeof(A));
    std::memcpy(A.cycle, cycle, cycleLen);
    std::memcpy(A.triple, triple, tripleLen);
    for (int i = 0; i < cycleLen; ++i) A.cycleIndex[cycle[i]] = (uint8_t)i;
    A.fact[0] = 1;
    for (int i = 1; i < 21; ++i) A.fact[i] = A.fact[i - 1] * (unsigned long long)i;
    A.cycleLen = cycleLen;
    A.tripleLen = tripleLen;
    A.n = n;
    A.skip2Move = skip2Move ? 1 : 0;
    A.total = A.fact[n - 1 > 0 ? n - 1 : 0];

    // n <= 16 (with cycle and triple of at most 16 symbols) takes the packed-register kernels
    const bool packed = n <= kPackedMaxN && cycleLen <= 16 && tripleLen <= 16;
    PackedArgs P;
    std::memset(&P, 0, sizeof(P));
    if (packed) {
        for (int i = 0; i <= 16; ++i) P.fact[i] = A.fact[i];
        P.total = A.total;
        std::memcpy(P.cycle, cycle, cycleLen);
        std::memcpy(P.triple, triple, tripleLen);
        P.cycleLen = cycleLen;
        P.tripleLen = tripleLen;
        P.n = n;
        P.skip2Move = A.skip2Move;
        P.twoMoveCount = two_move_triples(cycle, cycleLen, P.twoMove);
    }
    const int ranksPerBlock = packed ? kPackedRanksPerBlock : kRanksPerBlock;
    const uint64_t launchRanks = std::min<uint64_t>(kLaunchRanks, A.total);
    const int maxBlocks = (int)((launchRanks + ranksPerBlock - 1) / ranksPerBlock);
    DeviceBuffer prefix, totals, offsets, grand, rows;
    if (!ok(cudaMalloc(&prefix.ptr, (size_t)maxBlocks * kThreads * sizeof(unsigned)), err, "cudaMalloc") ||
        !ok(cudaMalloc(&totals.ptr, (size_t)maxBlocks * sizeof(unsigned)), err, "cudaMalloc") ||
        !ok(cudaMalloc(&offsets.ptr, (size_t)maxBlocks * sizeof(unsigned long long)), err, "cudaMalloc") ||
        !ok(cudaMalloc(&grand.ptr, sizeof(unsigned long long)), err, "cudaMalloc") ||
        !ok(cudaMemset(grand.ptr, 0, sizeof(unsigned long long)), err, "cudaMemset"))
        return -3;
    const size_t outBytes = (size_t)std::max<int64_t>(maxRows, 1) * (size_t)n;
    if (maxRows > 0 && !ok(cudaMalloc(&rows.ptr, outBytes), err, "cudaMalloc(rows)")) return -4;

    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (!ok(cudaEventCreate(&e0), err, "cudaEventCreate") || !ok(cudaEventCreate(&e1), err, "cudaEventCreate")) {
        if (e0) cudaEventDestroy(e0);
        return -3;
    }
    float kernelMs = 0.f;
    const auto start = std::chrono::steady_clock::now();
    int64_t rc = 0;
    for (uint64_t base = 0; base < A.total && rc == 0; base += kLaunchRanks) {
        A.base = base;
        P.base = base;
        const uint64_t ranks = std::min<uint64_t>(kLaunchRanks, A.total - base);
        const int blocks = (int)((ranks + ranksPerBlock - 1) / ranksPerBlock);
        cudaEventRecord(e0);
        if (packed) {
            packed_count_kernel<<<blocks, kThreads>>>(P, (unsigned *)prefix.ptr, (unsigned *)totals.ptr);
        } else {
            pi_filter_count_kernel<<<blocks, kThreads>>>(A, (unsigned *)prefix.ptr, (unsigned *)totals.ptr);
        }
        pi_filter_scan_kernel<<<1, kThreads>>>((const unsigned *)totals.ptr, (unsigned long long *)offsets.ptr,
                                               blocks, (unsigned long long *)grand.ptr);
        if (maxRows > 0) {
            if (packed) {
                packed_write_kernel<<<blocks, kThreads>>>(P, (const unsigned *)prefix.ptr,
                                                          (const unsigned long long *)offsets.ptr,
                                                          (uint8_t *)rows.ptr, (unsigned long long)maxRows);
            } else {
                pi_filter_write_kernel<<<blocks, kThreads>>>(A, (const unsigned *)prefix.ptr,
                                                             (const unsigned long long *)offsets.ptr,
                                                             (uint8_t *)rows.ptr, (unsigned long long)maxRows);
            }
        }
        cudaEventRecord(e1);
        if (!ok(cudaGetLastError(), err, "pi filter launch") || !ok(cudaDeviceSynchronize(), err, "pi filter")) {
            rc = -3;
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        kernelMs += ms;
        const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
        if (base + kLaunchRanks < A.total && elapsed > timeLimitS) {
            err = "pi filter: time limit exceeded";
            rc = -5;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != 0) return rc;
    gLastFilterKernelMs = kernelMs;
    unsigned long long hits = 0;
    if (!ok(cudaMemcpy(&hits, grand.ptr, sizeof(hits), cudaMemcpyDeviceToHost), err, "read count")) return -3;
    const int64_t kept = std::min<int64_t>((int64_t)hits, maxRows);
    if (kept > 0 && out &&
        !ok(cudaMemcpy(out, rows.ptr, (size_t)kept * (size_t)n, cudaMemcpyDeviceToHost), err, "read rows"))
        return -3;
    return (int64_t)hits;
}

int64_t pi_filter_noalloc_run(const uint8_t *cycle, int cycleLen, const uint8_t *triple, int tripleLen, int n,
                              int skip2Move, uint8_t *outDevice, int64_t maxRows, cudaStream_t stream,
                              std::string &err) {
    if (n < 1 || n > kNoAllocMaxN) {
        err = "tdp_pi_filter_noalloc: n must be in 1..12 (its static scratch covers (n-1)! <= 11! candidates); "
              "use tdp_pi_filter for larger n";
        return -1;
    }
    if (cycleLen < 0 || cycleLen > 63 || tripleLen < 0 || tripleLen > 63 || maxRows < 0 ||
        (maxRows > 0 && !outDevice) || (cycleLen > 0 && !cycle) || (tripleLen > 0 && !triple)) {
        err = "tdp_pi_filter_noalloc: invalid cycle/triple length, row limit or output buffer";
        return -1;
    }
    for (int i = 0; i < cycleLen; ++i)
        if (cycle[i] >= n) {
            err = "tdp_pi_filter_noalloc: cycle symbol out of range";
            return -1;
        }
    for (int i = 0; i < tripleLen; ++i)
        if (triple[i] >= n) {
            err = "tdp_pi_filter_noalloc: triple symbol out of range";
            return -1;
        }
    unsigned long long *scratch = noalloc_scratch(err);
    if (!scratch) return -3;
    FilterArgs A;
    std::memset(&A, 0, sizeof(A));
    std::memcpy(A.cycle, cycle, cycleLen);
    std::memcpy(A.triple, triple, tripleLen);
    for (int i = 0; i < cycleLen; ++i) A.cycleIndex[cycle[i]] = (uint8_t)i;
    A.fact[0] = 1;
    for (int i = 1; i < 21; ++i) A.fact[i] = A.fact[i - 1] * (unsigned long long)i;
    A.cycleLen = cycleLen;
    A.tripleLen = tripleLen;
    A.n = n;
    A.skip2Move = skip2Move ? 1 : 0;
    A.total = A.fact[n - 1 > 0 ? n - 1 : 0];
    A.base = 0;
    const int blocks = (int)((A.total + kRanksPerBlock - 1) / kRanksPerBlock);
    // The scratch keeps the previous call's contents; nothing needs clearing: the count pass
    // writes every block total the scan reads, and the scan writes every offset the write
    // pass reads and the hit total.
    noalloc_count_kernel<<<blocks, kThreads, 0, stream>>>(A, scratch, blocks);
    noalloc_scan_kernel<<<1, kThreads, 0, stream>>>(scratch, blocks);
    if (maxRows > 0)
        noalloc_write_kernel<<<blocks, kThreads, 0, stream>>>(A, scratch, outDevice, (unsigned long long)maxRows);
    if (!ok(cudaGetLastError(), err, "tdp_pi_filter_noalloc launch")) return -3;
    unsigned long long hits = 0;
    if (!ok(cudaMemcpyAsync(&hits, scratch, sizeof(hits), cudaMemcpyDeviceToHost, stream), err,
            "tdp_pi_filter_noalloc read") ||
        !ok(cudaStreamSynchronize(stream), err, "tdp_pi_filter_noalloc"))
        return -3;
    return (int64_t)hits;
}

}  // namespace tdp
