// Persistent warp-parallel DFS over search instances (device code).
//
// Replaces sorting_search_persistent_kernel / initialize_queues_kernel of the reference
// (sorting_search.cu:377-615) with the same verdict semantics:
//   * the root (depth 0) is always expanded;
//   * every child is first tested for success (satisfies_rate, sorting_search.cu:559);
//   * a child that is not a success is explored only if depth < maxDepth, it passes
//     can_still_reach and the transposition table admits it (sorting_search.cu:562-563);
//   * the transposition table prunes a state only when the same state of the same
//     instance was admitted at a depth <= the current one (sorting_search.cu:261-298);
//     a full probe window admits without inserting (table_replacement 0), or recycles
//     one of its live entries (policies 1-3), which only changes the work.
// Layout differences (B200-first, not a translation):
//   * one warp runs a lazy DFS: a node's children are evaluated 32 at a time (one triple
//     per lane: lexicographic, or only the same-cycle pairs/triples that can help),
//     admitted children are kept as a 32-bit pending mask and descended into one by one;
//     the frame stack (<= 16 frames) lives in shared memory (per-lane symbol words and one
//     record per frame), so no node is ever copied through global memory except when work
//     is donated;
//   * the warp probes the table together: eight lanes read one child's eight-entry window,
//     header and key words at once (dedup_admit_warp);
//   * each lane owns one symbol/position word (spi, pi, cycle leader, steps to leader,
//     cycle length) so a child's odd-cycle count is an O(1) delta (tdp_math.cuh) instead
//     of an O(n) recount, and a descent rebuilds the cycle tables with pointer jumping
//     over warp shuffles;
//   * once every instance is admitted, an idle warp registers its id in a lock-free ring and
//     polls only its own mailbox line; a busy warp that sees waiting warps dequeues one and
//     writes a Task straight into its mailbox: half the unexplored range of its shallowest
//     frame, or an admitted child it has not descended into yet (work donation);
//   * an instance ends when its last task finishes (outstanding counter), so there is
//     no global termination scan and no queue to overflow;
//   * the pruning rule is looked up in host-built bit tables (exact float32 semantics);
//   * table entries carry a (generation, instance) tag so nothing is cleared between
//     searches; entries of finished instances are reclaimed in place.
// Every spin has an iteration limit and every loop checks a device deadline, so a bug
// ends the launch with an error flag instead of hanging the GPU.
#pragma once

#include "engine.cuh"

namespace tdp {
namespace dev {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kWarpsPerBlock = 8;
constexpr int kSpinLimit = 1 << 20;

template <int NW>
struct KeyTraits;
template <>
struct KeyTraits<1> {
    static constexpr int KW = 3, BITS = 5, PER = 12;
};
template <>
struct KeyTraits<2> {
    static constexpr int KW = 7, BITS = 6, PER = 10;
};

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_relaxed_s32(const int *p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(uint32_t *p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long global_time_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

template <int NW>
__device__ __forceinline__ uint32_t gather(const uint32_t (&v)[NW], uint32_t idx) {
    if constexpr (NW == 1) {
        return __shfl_sync(kFull, v[0], (int)idx);
    } else {
        const uint32_t lo = __shfl_sync(kFull, v[0], (int)(idx & 31u));
        const uint32_t hi = __shfl_sync(kFull, v[1], (int)(idx & 31u));
        return idx < 32u ? lo : hi;
    }
}

__device__ __forceinline__ uint64_t shfl64(uint64_t v, int src) {
    const uint32_t lo = __shfl_sync(kFull, (uint32_t)v, src);
    const uint32_t hi = __shfl_sync(kFull, (uint32_t)(v >> 32), src);
    return ((uint64_t)hi << 32) | lo;
}

// Rebuilds leader / steps-to-leader / length fields of every word from its spi field.
template <int NW>
__device__ __forceinline__ void build_tables(uint32_t (&w)[NW], int n, int lane) {
    constexpr int R = (NW == 1) ? 5 : 6;
    uint32_t sv[NW], m[NW], j[NW];
#pragma unroll
    for (int h = 0; h < NW; ++h) {
        const uint32_t x = (uint32_t)(lane + 32 * h);
        const bool valid = x < (uint32_t)n;
        sv[h] = w_spi(w[h]);
        m[h] = x;
        j[h] = valid ? sv[h] : x;
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        uint32_t nm[NW], nj[NW];
#pragma unroll
        for (int h = 0; h < NW; ++h) {
            nm[h] = min(m[h], gather<NW>(m, j[h]));
            nj[h] = gather<NW>(j, j[h]);
        }
#pragma unroll
        for (int h = 0; h < NW; ++h) {
            m[h] = nm[h];
            j[h] = nj[h];
        }
    }
    uint32_t d[NW], p[NW];
#pragma unroll
    for (int h = 0; h < NW; ++h) {
        const uint32_t x = (uint32_t)(lane + 32 * h);
        const bool sink = (x >= (uint32_t)n) || (x == m[h]);
        d[h] = sink ? 0u : 1u;
        p[h] = sink ? x : sv[h];
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        uint32_t nd[NW], np[NW];
#pragma unroll
        for (int h = 0; h < NW; ++h) {
            nd[h] = d[h] + gather<NW>(d, p[h]);
            np[h] = gather<NW>(p, p[h]);
        }
#pragma unroll
        for (int h = 0; h < NW; ++h) {
            d[h] = nd[h];
            p[h] = np[h];
        }
    }
#pragma unroll
    for (int h = 0; h < NW; ++h) {
        const uint32_t afterLeader = gather<NW>(sv, m[h]);
        const uint32_t len = gather<NW>(d, afterLeader) + 1u;
        const uint32_t x = (uint32_t)(lane + 32 * h);
        w[h] = (x < (uint32_t)n) ? w_make(sv[h], w_pi(w[h]), m[h], d[h], len) : 0u;
    }
}

template <int NW>
__device__ __forceinline__ void compute_key(const uint32_t (&w)[NW], int n, int lane,
                                            uint64_t (&key)[KeyTraits<NW>::KW]) {
    using K = KeyTraits<NW>;
#pragma unroll
    for (int q = 0; q < K::KW; ++q) {
        uint64_t c = 0;
#pragma unroll
        for (int h = 0; h < NW; ++h) {
            const int x = lane + 32 * h;
            if (x < n && x / K::PER == q) c |= (uint64_t)w_spi(w[h]) << (K::BITS * (x % K::PER));
        }
        const uint32_t lo = __reduce_or_sync(kFull, (uint32_t)c);
        const uint32_t hi = __reduce_or_sync(kFull, (uint32_t)(c >> 32));
        key[q] = ((uint64_t)hi << 32) | lo;
    }
}

template <int NW>
__device__ __forceinline__ void set_field(uint64_t (&key)[KeyTraits<NW>::KW], uint32_t x, uint32_t v) {
    using K = KeyTraits<NW>;
    const uint32_t q = x / K::PER;
    const uint32_t s = K::BITS * (x - q * K::PER);
    const uint64_t mask = ((1ull << K::BITS) - 1ull) << s;
    const uint64_t val = (uint64_t)v << s;
#pragma unroll
    for (int qq = 0; qq < K::KW; ++qq)
        if (qq == (int)q) key[qq] = (key[qq] & ~mask) | val;
}

template <int KW>
__device__ __forceinline__ uint64_t key_hash(const uint64_t (&k)[KW], uint32_t tag) {
    uint64_t h = 0x9E3779B97F4A7C15ull ^ ((uint64_t)tag << 17);
#pragma unroll
    for (int q = 0; q < KW; ++q) {
        h ^= k[q];
        h *= 0xBF58476D1CE4E5B9ull;
        h ^= h >> 29;
    }
    h *= 0x94D049BB133111EBull;
    h ^= h >> 32;
    return h;
}

// Outcome bits of dedup_admit_warp: admitted, inserted into an empty, reclaimed or replaced
// entry, admitted without an entry because the window was full, inserted over a live entry
// of a full window, and "issued an atomic" (a claim or a depth update, for the statistics).
constexpr uint32_t kAdmitted = 1u, kInserted = 2u, kWindowFull = 4u, kReplaced = 8u, kAtomic = 16u;

__device__ __forceinline__ uint64_t ld_relaxed_u64(const void *p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ void st_relaxed_u64(void *p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint64_t cas_acq_rel_u64(void *p, uint64_t cmp, uint64_t val) {
    uint64_t old;
    asm volatile("atom.acq_rel.gpu.global.cas.b64 %0, [%1], %2, %3;"
                 : "=l"(old)
                 : "l"(p), "l"(cmp), "l"(val)
                 : "memory");
    return old;
}
// A CAS whose outcome nobody reads (the epoch refresh of an entry that pruned): the warp
// does not wait for it.
__device__ __forceinline__ void cas_relaxed_u64_nowait(void *p, uint64_t cmp, uint64_t val) {
    uint64_t old;
    asm volatile("atom.relaxed.gpu.global.cas.b64 %0, [%1], %2, %3;" : "=l"(old) : "l"(p), "l"(cmp), "l"(val));
    (void)old;
}

// Transposition-table admission (sorting_search.cu:261-298 semantics, per instance): a
// state of the same instance admitted at a depth <= `depth` prunes it; otherwise it is
// admitted and recorded.
//
// The warp probes together: every round takes up to four of the chunk's children, and the
// eight lanes of group g read the eight entries of child g's window, each lane one whole
// entry (header and key words in 16-byte loads), so a window costs one round trip and a
// prune needs no other.  The group decides from its ballots; one lane of the group then
// issues the group's only atomic, and the outcome goes back to the child's lane.
//
// Entries are written under a claim: a 64-bit CAS of the header (tag, meta) from the value
// read to (kTagWriting, version + 1 | epoch | depth) with acquire-release order, then the
// key words, each tagged with (version + 1) & 15 in its top 4 bits, then a release store of
// the tag.  With P.replace = 0 only empty entries and entries of older generations or
// finished instances are claimed; with P.replace > 0 a full window claims one of its live
// entries instead (policy 1: the deepest, if at least as deep as the newcomer; 2: the
// oldest; 3: the deepest, the oldest among those), so a key read may race with a rewrite.
// An entry matches when it carries the instance's tag and every key word equals the
// child's key and carries the version of the header read: such words were all written by
// that version's writer, which published that tag, unless the entry was rewritten a
// multiple of 16 times between the loads of one round, each rewrite needing a header read
// and a CAS on the entry after the previous one's release.  A key word of another version
// (a rewrite in flight, or a store not yet visible) makes the entry unknown: the child is
// admitted without an entry, which only costs work.  A depth improvement is a CAS of the
// header read, which fails after a rewrite.  With the recency policies (2, 3) a prune also
// moves the entry's epoch to now, so entries that keep pruning outlive entries nobody meets.
// Two children of one round that share a window may pick the same entry; the losing CAS
// admits its child without an entry.
template <int KW>
__device__ __forceinline__ void load_entry(const DedupEntry<KW> *e, uint64_t &hdr, uint64_t (&kw)[KW]) {
    const uint64_t *p = reinterpret_cast<const uint64_t *>(e);
    uint64_t v[KW + 1];
#pragma unroll
    for (int t = 0; t < (KW + 1) / 2; ++t)
        asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];"
                     : "=l"(v[2 * t]), "=l"(v[2 * t + 1])
                     : "l"(p + 2 * t));
    hdr = v[0];
#pragma unroll
    for (int kq = 0; kq < KW; ++kq) kw[kq] = v[kq + 1];
}

// All lanes call it with the ballot `todo` of the lanes that probe; returns the outcome bits
// of the calling lane's own child (0 for a lane not in todo).
template <int KW>
__device__ __forceinline__ uint32_t dedup_admit_warp(const EngineParams &P, uint32_t generation, uint32_t tag,
                                                     unsigned todo, const uint64_t (&key)[KW], uint64_t h,
                                                     uint32_t depth, int lane) {
    auto *table = reinterpret_cast<DedupEntry<KW> *>(P.table);
    const uint32_t myBase = (uint32_t)(h >> 24) & P.tableMask & ~7u;
    const uint32_t epoch = (uint32_t)(global_time_ns() >> 20) & 255u;
    const int grp = lane >> 3, q = lane & 7, sh = grp * 8;
    uint32_t mine = 0u;
    while (todo) {
        // this round: the first four children of todo, the g-th for group g
        unsigned rest = todo;
        int src = -1;
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            const int b = rest ? __ffs(rest) - 1 : -1;
            if (g == grp) src = b;
            rest &= rest - 1u;
        }
        const unsigned round = todo & ~rest;
        todo = rest;
        const bool active = src >= 0;
        const int s = active ? src : lane;
        const uint32_t base = __shfl_sync(kFull, myBase, s);
        uint64_t k[KW];
#pragma unroll
        for (int kq = 0; kq < KW; ++kq) k[kq] = shfl64(key[kq], s);
        DedupEntry<KW> *e = &table[base + q];
        uint64_t hd = 0ull, kw[KW];
#pragma unroll
        for (int kq = 0; kq < KW; ++kq) kw[kq] = 0ull;
        if (active) load_entry<KW>(e, hd, kw);
        const uint32_t t = (uint32_t)hd, mm = (uint32_t)(hd >> 32);
        const uint64_t check = (uint64_t)((mm >> kVersionShift) & 15u) << kKeyCheckShift;
        bool eq = true, other = false;
#pragma unroll
        for (int kq = 0; kq < KW; ++kq) {
            eq &= (kw[kq] & kKeyBits) == k[kq];
            other |= (kw[kq] & ~kKeyBits) != check;
        }
        const bool isTag = active && t == tag;
        const bool isFree = active && (t == 0u || (t != kTagWriting && (t >> kInstanceBits) != generation));
        const bool isLive = active && !isTag && !isFree && t != kTagWriting;
        const unsigned e8 = (__ballot_sync(kFull, isTag && eq && !other) >> sh) & 0xFFu;
        const unsigned u8 = (__ballot_sync(kFull, isTag && other) >> sh) & 0xFFu;
        unsigned f8 = (__ballot_sync(kFull, isFree) >> sh) & 0xFFu;
        const unsigned l8 = (__ballot_sync(kFull, isLive || (isTag && !eq && !other)) >> sh) & 0xFFu;
        const bool insertPath = active && e8 == 0u && u8 == 0u;
        if (!P.replace && __any_sync(kFull, insertPath && f8 == 0u)) {
            // no empty or old-generation entry: entries of finished instances are free too
            bool done = false;
            if (insertPath && f8 == 0u && ((l8 >> q) & 1u)) {
                const uint32_t idx = t & ((1u << kInstanceBits) - 1u);
                done = (ld_relaxed_u32(P.doneBits + (idx >> 5)) >> (idx & 31u)) & 1u;
            }
            f8 |= (__ballot_sync(kFull, done) >> sh) & 0xFFu;
        }
        // the victim of a full window (P.replace > 0): the highest score, ties to the later
        // slot; score 0 = not a candidate
        uint32_t pick = 0u;
        if (P.replace && __any_sync(kFull, insertPath && f8 == 0u)) {
            const uint32_t d = mm & kDepthMask;
            const uint32_t age = (epoch - ((mm & kEpochMask) >> kEpochShift)) & 255u;
            const uint32_t score = !((l8 >> q) & 1u) ? 0u
                                   : P.replace == 1 ? (d >= depth ? d + 1u : 0u)
                                   : P.replace == 2 ? age + 1u
                                                    : ((d << 8) | age) + 1u;
            pick = (score << 3) | (uint32_t)q;
#pragma unroll
            for (int o = 1; o < 8; o <<= 1) pick = max(pick, __shfl_xor_sync(kFull, pick, o));
        }
        // the group's decision, taken by one lane of the group
        uint32_t res = 0u;
        bool claim = false, improve = false;
        uint64_t casNew = 0ull;
        if (active) {
            if (e8) {
                if (q == __ffs(e8) - 1) {
                    if ((mm & kDepthMask) <= depth) {
                        if (P.replace >= 2 && ((mm & kEpochMask) >> kEpochShift) != epoch)
                            cas_relaxed_u64_nowait(e, hd,
                                                   ((uint64_t)((mm & ~kEpochMask) | (epoch << kEpochShift)) << 32) | tag);
                    } else if (P.replace) {
                        improve = true;
                        casNew = ((uint64_t)((mm & ~(kDepthMask | kEpochMask)) | (epoch << kEpochShift) | depth) << 32) |
                                 tag;
                        res = kAdmitted | kAtomic;
                    } else {
                        // best depths only decrease while the instance runs (no rewrite of its
                        // live entries without replacement)
                        const uint32_t prev = atomicMin(&e->meta, (mm & ~kDepthMask) | depth);
                        res = (prev & kDepthMask) <= depth ? kAtomic : (kAdmitted | kAtomic);
                    }
                }
            } else if (u8) {
                if (q == 0) res = kAdmitted;
            } else {
                const int slot = f8 ? __ffs(f8) - 1 : ((pick >> 3) ? (int)(pick & 7u) : -1);
                if (slot < 0) {
                    if (q == 0) res = kAdmitted | kWindowFull;
                } else if (q == slot) {
                    claim = true;
                    const uint32_t version = (mm >> kVersionShift) + 1u;
                    casNew = ((uint64_t)((version << kVersionShift) | (epoch << kEpochShift) | depth) << 32) | kTagWriting;
                    res = kAdmitted | kInserted | (f8 ? 0u : kReplaced) | kAtomic;
                }
            }
        }
        if (claim || improve) {
            const uint64_t got = cas_acq_rel_u64(e, hd, casNew);
            if (claim) {
                if (got == hd) {
                    const uint64_t nib = (uint64_t)((((mm >> kVersionShift) + 1u) & 15u)) << kKeyCheckShift;
#pragma unroll
                    for (int kq = 0; kq < KW; ++kq) st_relaxed_u64(&e->key[kq], k[kq] | nib);
                    st_release_u32(&e->tag, tag);  // the release orders the key stores before it
                } else {
                    res = kAdmitted | kAtomic;
                }
            }
        }
        // the group's outcome to every lane of the group, then to the child's lane
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) res |= __shfl_xor_sync(kFull, res, o);
        const int rank = __popc(round & ((1u << lane) - 1u));
        const uint32_t got = __shfl_sync(kFull, res, (rank & 3) * 8);
        if ((round >> lane) & 1u) mine = got;
    }
    return mine;
}

// Partial-order reduction of commuting moves (verdict-preserving; no counterpart in the
// reference).  The node of frame f was reached by the move (x y z) at positions I<J<K of its
// parent P; its child (a b c) at positions i<j<k is skipped when {a,b,c} and {x,y,z} are
// disjoint, (a b c) is also a move at P (a, b, c in cyclic order there: the inverse block
// swap of (I,J,K) gives their positions in P), (x y z) is a move once (a b c) has been
// applied at P, and min(a,b,c) < min(x,y,z).  Disjoint 3-cycles commute, so P.(a b c).(x y z)
// reaches the same state at the same depth through the kept order.  Every admission
// condition of the rule tables is monotone along a move sequence (a move changes the
// odd-cycle count by at most 2), so the kept order passes them wherever the skipped one
// does.  With the transposition table a state is expanded only at its admissions; a child
// skipped at one is reached through the parent's commuted sibling, whose admission may skip
// the (larger) incoming move in turn, and so on: the least symbol of the last move grows
// strictly along that chain, so by induction on depth every reachable state is admitted at
// a depth no larger than its own.
__device__ __forceinline__ bool por_skip(uint32_t inc, uint32_t x, uint32_t y, uint32_t z, uint32_t i, uint32_t j,
                                         uint32_t k, uint32_t a, uint32_t b, uint32_t c) {
    if (a == x || a == y || a == z || b == x || b == y || b == z || c == x || c == y || c == z) return false;
    const int I = (int)tri_i(inc), J = (int)tri_j(inc), K = (int)tri_k(inc);
    const int pa = block_swap_src((int)i, I, J, K), pb = block_swap_src((int)j, I, J, K),
              pc = block_swap_src((int)k, I, J, K);
    if ((pa > pb) + (pb > pc) + (pc > pa) > 1) return false;
    const int q0 = min(pa, min(pb, pc)), q2 = max(pa, max(pb, pc)), q1 = pa + pb + pc - q0 - q2;
    const int lenA = q1 - q0, lenB = q2 - q1;
    const int fI = (I >= q0 && I < q1) ? I + lenB : (I >= q1 && I < q2) ? I - lenA : I;
    const int fJ = (J >= q0 && J < q1) ? J + lenB : (J >= q1 && J < q2) ? J - lenA : J;
    const int fK = (K >= q0 && K < q1) ? K + lenB : (K >= q1 && K < q2) ? K - lenA : K;
    if ((fI > fJ) + (fJ > fK) + (fK > fI) > 1) return false;
    return min(a, min(b, c)) < min(x, min(y, z));
}

// Idle-warp ring: a bounded lock-free multi-producer/multi-consumer queue of warp ids.  Slot
// s carries a lap word d = seq - s (zero-initialised): d == lap means free for the enqueue
// of that lap, d == lap + 1 means it holds an id.  The ring has at least as many slots as
// the grid has warps and a warp registers at most once at a time, so an enqueue never
// finds its slot held by an earlier lap for longer than a dequeue in progress.
__device__ __forceinline__ bool ring_enqueue(const EngineParams &P, uint32_t wid) {
    const uint32_t pos = atomicAdd(&P.ctl->ringTail, 1u);
    const uint32_t slot = pos & P.ringMask, lap = pos & ~P.ringMask;
    for (int it = 0; it < kSpinLimit; ++it) {
        if (ld_acquire_u32(P.ringSeq + slot) == lap) {
            P.ringWid[slot] = wid;
            st_release_u32(P.ringSeq + slot, lap + 1u);
            return true;
        }
        __nanosleep(32);
    }
    atomicExch(&P.ctl->error, kErrSpinLimit);
    atomicExch(&P.ctl->stop, 1);
    return false;
}

// Returns a registered idle warp id, or -1 when the ring is empty (or the race was lost).
__device__ __forceinline__ int ring_dequeue(const EngineParams &P) {
    for (int attempt = 0; attempt < 8; ++attempt) {
        const uint32_t h = ld_relaxed_u32(&P.ctl->ringHead);
        const uint32_t slot = h & P.ringMask, lap = h & ~P.ringMask;
        const uint32_t d = ld_acquire_u32(P.ringSeq + slot);
        if (d == lap + 1u) {
            if (atomicCAS(&P.ctl->ringHead, h, h + 1u) == h) {
                const uint32_t w = ld_relaxed_u32(P.ringWid + slot);
                st_release_u32(P.ringSeq + slot, lap + P.ringMask + 1u);
                return (int)w;
            }
        } else if ((int)(d - (lap + 1u)) < 0) {
            return -1;  // not filled yet: nobody is waiting at this position
        }
    }
    return -1;
}

// Children words (spi/pi fields only; tables are rebuilt by the caller) of the move that
// takes positions (i, j, k), i.e. symbols a, b, c with cycle words wa, wb, wc.
template <int NW>
__device__ __forceinline__ void apply_move(const uint32_t (&w)[NW], uint32_t (&out)[NW], int lane, uint32_t i,
                                           uint32_t j, uint32_t k, uint32_t a, uint32_t b, uint32_t c, uint32_t wa,
                                           uint32_t wb, uint32_t wc) {
#pragma unroll
    for (int h = 0; h < NW; ++h) {
        const uint32_t x = (uint32_t)(lane + 32 * h);
        uint32_t s = w_spi(w[h]);
        if (x == a) s = w_spi(wc);
        if (x == b) s = w_spi(wa);
        if (x == c) s = w_spi(wb);
        const uint32_t src = (uint32_t)block_swap_src((int)x, (int)i, (int)j, (int)k);
        out[h] = s | (w_pi(gather<NW>(w, src)) << 6);
    }
}

// Restricted child enumerations (n <= 32, one position per lane).  Both rest on the cycle
// structure of spi: a child's odd-cycle count changes by +2 only if its three symbols lie
// in one cycle, or two lie in one even-length cycle and the third in another even-length
// cycle; a triple over three distinct cycles changes the count by -2, or by 0 only when two
// of those cycles have even length.
//
// * Pairs (mode 1).  When no child with a -2 change is useful, and either 0-changes are
//   useless too or the node has at most one even-length cycle, every useful child has two
//   of its three symbols in one cycle.  The frame enumerates position pairs p < q whose
//   symbols share a cycle, one pair per chunk, with the lane as the third position r; a
//   triple lying in one cycle is taken only from its two smallest positions.
// * Triples (mode 2).  When only +2 children are useful and the node has at most one
//   even-length cycle, every useful child takes its three symbols from one cycle.  The
//   frame enumerates the position triples p < q < r inside each cycle, 32 per chunk, from
//   a list the warp writes to shared memory at frame set-up (at most kMaxTriples entries;
//   a larger frame uses pairs).  In searches at the ratio limit this is nearly every frame,
//   and a frame then needs one or two chunks instead of one per same-cycle pair.
constexpr int kMaxTriples = 256;

struct SparseFrame {
    uint32_t same;       // positions > lane whose symbol shares the cycle of pi[lane]
    uint32_t incl;       // inclusive prefix over lanes of popc(same) (pairs) or C(popc(same), 2) (triples)
    uint32_t leaderPos;  // cycle leader of pi[lane]
    int np;              // number of pairs or triples
    int mode;            // 0 dense, 1 pairs, 2 triples
};

struct PairSel {
    int p, q;
    uint32_t leader;
};

// allow: 0 dense only, 1 pairs, 2 pairs and triples.  triList (or null) receives the
// triple list of a triple-mode frame; pass null to classify a frame without touching the
// list of the frame being enumerated.
template <int NW>
__device__ __forceinline__ SparseFrame sparse_setup(const uint32_t (&w)[NW], int n, int lane, int even,
                                                    uint64_t satMask, uint64_t expMask, int allow,
                                                    uint32_t *triList) {
    SparseFrame sf;
    sf.same = 0u;
    sf.incl = 0u;
    sf.leaderPos = 0u;
    sf.np = 0;
    sf.mode = 0;
    if constexpr (NW != 1) {
        return sf;
    } else {
        if (allow <= 0) return sf;
        const uint64_t useful = satMask | expMask;
        const bool neg = even >= 2 && ((useful >> (even - 2)) & 1ull);
        if (neg) return sf;
        const bool zero = (useful >> even) & 1ull;
        const bool isLeader = lane < n && w_leader(w[0]) == (uint32_t)lane;
        const int evenLen = __popc(__ballot_sync(kFull, isLeader && (w_len(w[0]) & 1u) == 0u));
        if (zero && evenLen >= 2) return sf;
        const uint32_t leaderPos = w_leader(gather<1>(w, w_pi(w[0])));
        const uint32_t key = (lane < n) ? leaderPos : 64u + (uint32_t)lane;
        const uint32_t same = __match_any_sync(kFull, key) & ~((2u << lane) - 1u);
        sf.same = same;
        sf.leaderPos = leaderPos;
        const uint32_t k = (uint32_t)__popc(same);
        if (allow >= 2 && !zero && evenLen <= 1) {
            const uint32_t c2 = k * (k - 1u) / 2u;
            uint32_t incl = c2;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(kFull, incl, o);
                if (lane >= o) incl += y;
            }
            const int total = (int)__shfl_sync(kFull, incl, 31);
            if (total <= kMaxTriples) {
                if (triList) {
                    __syncwarp();  // every lane is done reading the previous frame's list
                    uint32_t at = incl - c2;
                    uint32_t m1 = same;
                    while (m1) {
                        const uint32_t q = (uint32_t)(__ffs(m1) - 1);
                        m1 &= m1 - 1u;
                        uint32_t m2 = m1;
                        while (m2) {
                            const uint32_t r = (uint32_t)(__ffs(m2) - 1);
                            m2 &= m2 - 1u;
                            triList[at++] = pack_triple((uint32_t)lane, q, r);
                        }
                    }
                    __syncwarp();
                }
                sf.incl = incl;
                sf.np = total;
                sf.mode = 2;
                return sf;
            }
        }
        uint32_t incl = k;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += y;
        }
        sf.incl = incl;
        sf.np = (int)__shfl_sync(kFull, incl, 31);
        sf.mode = 1;
        return sf;
    }
}

// Decodes pair index u (uniform) into positions p < q.
__device__ __forceinline__ PairSel sparse_pair(const SparseFrame &sf, int u) {
    const unsigned owner = __ballot_sync(kFull, sf.incl > (uint32_t)u);
    const int p = __ffs(owner) - 1;
    const uint32_t sameP = __shfl_sync(kFull, sf.same, p);
    const uint32_t exclP = __shfl_sync(kFull, sf.incl, p) - (uint32_t)__popc(sameP);
    uint32_t m = sameP;
    for (uint32_t t = (uint32_t)u - exclP; t > 0u; --t) m &= m - 1u;
    PairSel ps;
    ps.p = p;
    ps.q = __ffs(m) - 1;
    ps.leader = __shfl_sync(kFull, sf.leaderPos, p);
    return ps;
}

// Triple index u (uniform) of a triple-mode frame, decoded without its list, in list order:
// owner position p, then the v-th pair q < r of the positions in same(p) (lexicographic).
__device__ __forceinline__ uint32_t triple_at(const SparseFrame &sf, int u) {
    const unsigned owner = __ballot_sync(kFull, sf.incl > (uint32_t)u);
    const int p = __ffs(owner) - 1;
    const uint32_t sameP = __shfl_sync(kFull, sf.same, p);
    const uint32_t k = (uint32_t)__popc(sameP);
    uint32_t v = (uint32_t)u - (__shfl_sync(kFull, sf.incl, p) - k * (k - 1u) / 2u);
    uint32_t m1 = sameP, q = 0u, r = 0u;
    for (uint32_t it = 0; it < 32u && m1; ++it) {
        q = (uint32_t)(__ffs(m1) - 1);
        m1 &= m1 - 1u;
        const uint32_t cnt = (uint32_t)__popc(m1);
        if (v < cnt) {
            uint32_t m2 = m1;
            for (uint32_t t = v; t > 0u; --t) m2 &= m2 - 1u;
            r = (uint32_t)(__ffs(m2) - 1);
            break;
        }
        v -= cnt;
    }
    return pack_triple((uint32_t)p, q, r);
}

// Saved state of a DFS frame, written when the warp descends from it (one writer lane).
template <int KW>
struct FrameRec {
    int cursor, end, chunk, even, step;  // next chunk, range end, chunk of `pending`, odd-cycle count, chunk step
    uint32_t pending;                    // admitted children of chunk `chunk` not yet descended into
    uint32_t move;                       // move that left this frame (the path)
    uint32_t pad;
    uint64_t key[KW];                    // transposition-table key of the frame's node
};

template <int NW>
struct WarpShared {
    uint32_t words[kMaxDepth + 1][NW * 32];
    FrameRec<KeyTraits<NW>::KW> frames[kMaxDepth + 1];
    uint32_t tri[NW == 1 ? kMaxTriples : 1];  // triple list of the frame being enumerated
    uint64_t rules[32];                       // success (0..15) and expansion (16..31) tables of the instance
    unsigned long long taskNodes, taskChildren;  // counters of the task in hand
    int rank1;                                   // root-order rank of the current first-level node (-1: none)
    uint32_t staging[52];
    unsigned long long stats[kStatCount];  // per-warp counters, flushed once at exit
};

template <int NW>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, NW == 1 ? 4 : 2) search_engine_kernel(const EngineParams P) {
    using K = KeyTraits<NW>;
    constexpr int KW = K::KW;
    __shared__ WarpShared<NW> smem[kWarpsPerBlock];
    const int lane = (int)(threadIdx.x & 31u);
    WarpShared<NW> &S = smem[threadIdx.x >> 5];
    EngineCtl *ctl = P.ctl;
    const unsigned long long deadline = global_time_ns() + P.timeLimitNs;
    const uint32_t generation = __ldcg(P.generation);

    if (lane < kStatCount) S.stats[lane] = 0ull;
    __syncwarp();
    const uint32_t gw = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    bool registered = false;
    int backoff = 64;
    // Busy and lifetime cycles accumulate in the warp's shared counters (start times are
    // subtracted, end times added; unsigned arithmetic wraps back), so no register stays live.
    if (lane == 0) S.stats[kStatWarpCycles] -= (unsigned long long)clock64();
    int idleRound = 0;
    bool stopAll = false;

    while (!stopAll) {
        // ---------------------------------------------------------------- get work
        // Before the last instance is admitted an idle warp admits the next instance; after
        // that it registers once in the idle ring and polls only its own mailbox line.
        int kind = 0, idx = 0;
        if (lane == 0) {
            if (registered && ld_acquire_u32(&P.mail[gw].flag) != 0u) kind = 1;
            if (kind == 0) {
                const bool full = registered ? ((++idleRound & 7) == 0) : true;
                if (full) {
                    const int stopFlag = ld_relaxed_s32(&ctl->stop);
                    const int cancelFlag = ld_relaxed_s32(P.cancel);
                    const bool late = global_time_ns() > deadline;
                    if (late && !(stopFlag | cancelFlag)) {
                        atomicExch(&ctl->error, kErrDeadline);
                        atomicExch(&ctl->stop, 1);
                    }
                    if ((stopFlag | cancelFlag) || late) kind = -1;
                }
                if (kind == 0 && !registered) {
                    // With a cap, a warp admits only while fewer than maxInFlight admitted
                    // instances are unfinished (a racy check: the cap may be exceeded by the
                    // few warps that pass it together); otherwise it registers as a helper.
                    // The warp that finishes an instance is unregistered, so it admits the
                    // next one: the cap cannot leave instances unadmitted.
                    const int next = ld_relaxed_s32(&ctl->nextInstance);
                    const bool room =
                        P.maxInFlight <= 0 || next - ld_relaxed_s32(&ctl->doneCount) < P.maxInFlight;
                    if (next < P.count && room) {
                        const int i = atomicAdd(&ctl->nextInstance, 1);
                        if (i < P.count) {
                            kind = 2;
                            idx = i;
                        }
                    }
                    if (kind == 0) {
                        if (ring_enqueue(P, gw)) {
                            registered = true;
                        } else {
                            kind = -1;
                        }
                    }
                }
                if (kind == 0 && full && ld_relaxed_s32(&ctl->doneCount) >= P.count) kind = -1;
            }
        }
        kind = __shfl_sync(kFull, kind, 0);
        idx = __shfl_sync(kFull, idx, 0);
        if (kind < 0) break;
        if (kind == 0) {
            __nanosleep(backoff);
            backoff = min(backoff * 2, 256);  // a donated task is picked up within ~0.3 us
            continue;
        }
        backoff = 64;
        idleRound = 0;
        if (lane == 0) S.stats[kStatBusyCycles] -= (unsigned long long)clock64();

        // ---------------------------------------------------------------- set up
        uint32_t inst;
        int baseDepth, even, lo, hi;
        uint32_t w[NW];
        if (kind == 1) {
            __threadfence();  // every lane reads the task only after lane 0 observed the flag
            const uint32_t *src = reinterpret_cast<const uint32_t *>(&P.mail[gw].task);
            for (int q = lane; q < 52; q += 32) S.staging[q] = __ldcg(src + q);
            __syncwarp();
            if (lane == 0) {
                // the mailbox is free again before this warp can re-register
                *reinterpret_cast<volatile uint32_t *>(&P.mail[gw].flag) = 0u;
                __threadfence();
                ++S.stats[kStatTaskPops];
            }
            registered = false;
            inst = S.staging[0];
            baseDepth = (int)(S.staging[1] & 0xFFu);
            even = (int)((S.staging[1] >> 8) & 0xFFu);
            lo = (int)(S.staging[2] & 0xFFFFu);
            hi = (int)(S.staging[2] >> 16);
            if (lane == 0) {
                S.taskNodes = S.staging[3] & 1u;
                S.rank1 = baseDepth == 1 ? (int)((S.staging[3] >> 8) & 0xFFu) - 1 : -1;
            }
            if (lane < baseDepth) S.frames[lane].move = S.staging[4 + lane];
            const uint8_t *bytes = reinterpret_cast<const uint8_t *>(S.staging);
            const int n = P.in[inst].n;
#pragma unroll
            for (int h = 0; h < NW; ++h) {
                const int x = lane + 32 * h;
                w[h] = (x < n) ? ((uint32_t)bytes[80 + x] | ((uint32_t)bytes[144 + x] << 6)) : 0u;
            }
            __syncwarp();
        } else {
            inst = (uint32_t)idx;
            const InstanceIn *I = P.in + inst;
            if (lane == 0) {
                atomicExch(&P.out[inst].outstanding, 1);
                atomicExch(&P.out[inst].state, kStateRunning);
            }
            baseDepth = 0;
            even = I->even0;
            lo = 0;
            hi = 0xFFFF;
            const int n = I->n;
#pragma unroll
            for (int h = 0; h < NW; ++h) {
                const int x = lane + 32 * h;
                w[h] = (x < n) ? ((uint32_t)I->spi[x] | ((uint32_t)I->pi[x] << 6)) : 0u;
            }
            if (lane == 0) {
                S.taskNodes = 1;
                S.rank1 = -1;
            }
        }
        if (lane == 0) S.taskChildren = 0;
        const int n = P.in[inst].n;
        const int T = combinations3(n);
        const uint32_t *trip = P.triples + combinations4(n);
        const uint32_t tag = (generation << kInstanceBits) | inst;
        const RuleTable *rt = P.rules + P.in[inst].rule;
        S.rules[lane] = (lane < 16) ? rt->sat[lane] : rt->expand[lane - 16];
        __syncwarp();

        build_tables<NW>(w, n, lane);
        uint64_t key[KW];
        compute_key<NW>(w, n, lane, key);

        int f = baseDepth;
        int cursor = lo, end = hi, chunk = 0;
        uint32_t pending = 0;
#pragma unroll
        for (int h = 0; h < NW; ++h) S.words[f][h * 32 + lane] = w[h];
        uint64_t satMask = S.rules[f + 1];
        uint64_t expMask = S.rules[16 + f + 1];
        // The root of an instance with a learned order enumerates its children in that order
        // (dense mode, index space = positions in the order).  With first-level lists, the
        // node after root child rank r < order2Ranks enumerates its list first and then every
        // child in plain order (dense, index space = list slots then triples), so it stays
        // exhaustive; a child in both parts meets the table the second time.
        const uint16_t *rootOrder = (P.order && NW == 1) ? P.order + (size_t)inst * (size_t)P.orderStride : nullptr;
        auto listOf = [&](int g) -> const uint16_t * {
            if (!P.order2 || !rootOrder || g != 1) return nullptr;
            const int r = S.rank1;
            return (r >= 0 && r < P.order2Ranks) ? P.order2 + ((size_t)inst * P.order2Ranks + r) * P.order2List
                                                 : nullptr;
        };
        auto ordered = [&](int g) -> bool { return (rootOrder && g == 0) || listOf(g) != nullptr; };
        // dense index t of frame g -> packed triple; 0xFFFFFFFF marks an empty list slot
        auto decode = [&](int g, int t) -> uint32_t {
            if (rootOrder && g == 0) return __ldg(trip + (int)__ldg(rootOrder + t));
            const uint16_t *L = listOf(g);
            if (L) {
                if (t < P.order2List) {
                    const uint16_t e = __ldg(L + t);
                    return e == 0xFFFFu ? 0xFFFFFFFFu : __ldg(trip + (int)e);
                }
                t -= P.order2List;
            }
            return __ldg(trip + t);
        };
        auto denseEnd = [&](int g) -> int { return T + (listOf(g) ? P.order2List : 0); };
        SparseFrame sf = sparse_setup<NW>(w, n, lane, even, satMask, expMask, ordered(f) ? 0 : P.sparse, S.tri);
        // A donated range is in the units of its frame's mode (the receiver derives the same
        // mode from the same node); hi = 0xFFFF covers every child.
        if (hi == 0xFFFF) end = sf.mode ? sf.np : denseEnd(f);

        // outcome: 0 subtree exhausted, 1 instance found (here or elsewhere), 2 launch stop
        int outcome = 0;
        if (kind == 1) {
            int st = 0;
            if (lane == 0) st = ld_relaxed_s32(&P.out[inst].state);
            if (__shfl_sync(kFull, st, 0) == kStateFound) outcome = 1;
        }
        int poll = 0;
        while (outcome == 0) {
            if (pending == 0u) {
                if (cursor >= end) {
                    if (f == baseDepth) break;
                    --f;
                    const FrameRec<KW> &fr = S.frames[f];
                    cursor = fr.cursor;
                    end = fr.end;
                    pending = fr.pending;
                    // An exhausted parent is left at once: its words, key and enumeration
                    // state are not needed.
                    if (pending == 0u && cursor >= end) continue;
                    chunk = fr.chunk;
                    even = fr.even;
#pragma unroll
                    for (int q = 0; q < KW; ++q) key[q] = fr.key[q];
#pragma unroll
                    for (int h = 0; h < NW; ++h) w[h] = S.words[f][h * 32 + lane];
                    satMask = S.rules[f + 1];
                    expMask = S.rules[16 + f + 1];
                    sf = sparse_setup<NW>(w, n, lane, even, satMask, expMask, ordered(f) ? 0 : P.sparse, S.tri);
                    continue;
                }
                if (++poll >= P.pollInterval) {
                    poll = 0;
                    int act = 0;
                    if (lane == 0) {
                        // Independent loads, issued together: one L2 round trip per poll.
                        const int stopFlag = ld_relaxed_s32(&ctl->stop);
                        const int cancelFlag = ld_relaxed_s32(P.cancel);
                        const int state = ld_relaxed_s32(&P.out[inst].state);
                        const uint32_t rt = ld_relaxed_u32(&ctl->ringTail);
                        const uint32_t rh = ld_relaxed_u32(&ctl->ringHead);
                        const bool late = global_time_ns() > deadline;
                        if (stopFlag | cancelFlag) {
                            act = 2;
                        } else if (late) {
                            atomicExch(&ctl->error, kErrDeadline);
                            atomicExch(&ctl->stop, 1);
                            act = 2;
                        } else if (state == kStateFound) {
                            act = 1;
                        } else if (rt != rh) {
                            act = 3;
                        }
                    }
                    act = __shfl_sync(kFull, act, 0);
                    if (act == 1 || act == 2) {
                        outcome = act;
                        break;
                    }
                    if (act == 3) {
                        // ------------------------------------------------ donate
                        // Candidates: the shallowest frame with >= 2 unevaluated chunks
                        // (split its range), or a shallower frame holding admitted children
                        // not yet descended into (hand over one of them as a fresh node).
                        const int step = sf.mode == 1 ? 1 : 32;
                        int remChunks = 0;
                        uint32_t pend = 0u;
                        if (lane >= baseDepth && lane < f) {
                            const FrameRec<KW> &fr = S.frames[lane];
                            remChunks = (fr.end - fr.cursor + fr.step - 1) / fr.step;
                            pend = fr.pending;
                        }
                        if (lane == f) {
                            remChunks = (end - cursor + step - 1) / step;
                            pend = pending;
                        }
                        const unsigned big = __ballot_sync(kFull, remChunks >= 2);
                        const unsigned held = __ballot_sync(kFull, pend != 0u);
                        const unsigned some = __ballot_sync(kFull, remChunks > 0 && lane < f);
                        const int g1 = big ? (__ffs(big) - 1) : 99;
                        const int gp = held ? (__ffs(held) - 1) : 99;
                        const int g0 = some ? (__ffs(some) - 1) : 99;
                        int mode = 0, g = -1;  // 1 range split, 2 pending child, 3 whole range
                        if (gp < g1 && gp < 99) {
                            mode = 2;
                            g = gp;
                        } else if (g1 < 99) {
                            mode = 1;
                            g = g1;
                        } else if (g0 < 99) {
                            mode = 3;
                            g = g0;
                        }
                        int target = -1;
                        if (mode != 0 && lane == 0) target = ring_dequeue(P);
                        target = __shfl_sync(kFull, target, 0);
                        if (target >= 0) {
                            Task *tk = &P.mail[target].task;
                            const int gEven = (g == f) ? even : S.frames[g].even;
                            uint32_t hdr1, hdr2, hdr3;
                            if (mode == 2) {
                                const int gChunk = (g == f) ? chunk : S.frames[g].chunk;
                                const uint32_t gPend = __shfl_sync(kFull, pend, g);
                                const int l = __ffs(gPend) - 1;
                                uint32_t wg[NW];
#pragma unroll
                                for (int h = 0; h < NW; ++h) wg[h] = S.words[g][h * 32 + lane];
                                const uint64_t gSat = S.rules[g + 1];
                                const uint64_t gExp = S.rules[16 + g + 1];
                                const SparseFrame gsf =
                                    sparse_setup<NW>(wg, n, lane, gEven, gSat, gExp, ordered(g) ? 0 : P.sparse, nullptr);
                                uint32_t ctr;
                                if (gsf.mode == 1) {
                                    const PairSel ps = sparse_pair(gsf, gChunk);
                                    ctr = (l < ps.p) ? pack_triple(l, ps.p, ps.q)
                                                     : (l < ps.q) ? pack_triple(ps.p, l, ps.q)
                                                                  : pack_triple(ps.p, ps.q, l);
                                } else if (gsf.mode == 2) {
                                    ctr = triple_at(gsf, gChunk + l);
                                } else {
                                    const int t = gChunk + l;
                                    ctr = decode(g, t);
                                }
                                const uint32_t ci = tri_i(ctr), cj = tri_j(ctr), ck = tri_k(ctr);
                                const uint32_t ca = w_pi(gather<NW>(wg, ci));
                                const uint32_t cb = w_pi(gather<NW>(wg, cj));
                                const uint32_t cc = w_pi(gather<NW>(wg, ck));
                                const uint32_t cwa = gather<NW>(wg, ca);
                                const uint32_t cwb = gather<NW>(wg, cb);
                                const uint32_t cwc = gather<NW>(wg, cc);
                                const int cEven = gEven + move_delta(cwa, cwb, cwc);
                                uint32_t cw[NW];
                                apply_move<NW>(wg, cw, lane, ci, cj, ck, ca, cb, cc, cwa, cwb, cwc);
#pragma unroll
                                for (int h = 0; h < NW; ++h) {
                                    const int x = lane + 32 * h;
                                    if (x < n) {
                                        tk->spi[x] = (uint8_t)w_spi(cw[h]);
                                        tk->pi[x] = (uint8_t)w_pi(cw[h]);
                                    }
                                }
                                if (lane < g) tk->path[lane] = S.frames[lane].move;
                                if (lane == g) tk->path[g] = ctr;
                                hdr1 = (uint32_t)(g + 1) | ((uint32_t)cEven << 8);
                                hdr2 = 0xFFFFu << 16;
                                hdr3 = 1u;
                                // a root child handed over keeps its learned rank (first-level list)
                                if (g == 0 && rootOrder && gChunk + l < P.order2Ranks)
                                    hdr3 |= (uint32_t)(gChunk + l + 1) << 8;
                                const uint32_t bit = 1u << l;
                                if (g == f) {
                                    pending &= ~bit;
                                } else if (lane == 0) {
                                    S.frames[g].pending &= ~bit;
                                }
                            } else {
                                const int gc = (g == f) ? cursor : S.frames[g].cursor;
                                const int ge = (g == f) ? end : S.frames[g].end;
                                const int gStep = (g == f) ? step : S.frames[g].step;
                                const int remg = (ge - gc + gStep - 1) / gStep;
                                const int keepChunks = (mode == 1) ? (remg + 1) / 2 : 0;
                                const int newEnd = min(ge, gc + keepChunks * gStep);
#pragma unroll
                                for (int h = 0; h < NW; ++h) {
                                    const int x = lane + 32 * h;
                                    if (x < n) {
                                        const uint32_t wg = S.words[g][h * 32 + lane];
                                        tk->spi[x] = (uint8_t)w_spi(wg);
                                        tk->pi[x] = (uint8_t)w_pi(wg);
                                    }
                                }
                                if (lane < g) tk->path[lane] = S.frames[lane].move;
                                hdr1 = (uint32_t)g | ((uint32_t)gEven << 8);
                                hdr2 = (uint32_t)newEnd | ((uint32_t)ge << 16);
                                hdr3 = 0u;
                                // a first-level range is in its list's index space: pass the rank
                                if (g == 1 && S.rank1 >= 0 && S.rank1 < P.order2Ranks)
                                    hdr3 |= (uint32_t)(S.rank1 + 1) << 8;
                                if (g == f) {
                                    end = newEnd;
                                } else if (lane == 0) {
                                    S.frames[g].end = newEnd;
                                }
                            }
                            if (lane == 0) {
                                uint32_t *hdr = reinterpret_cast<uint32_t *>(tk);
                                hdr[0] = inst;
                                hdr[1] = hdr1;
                                hdr[2] = hdr2;
                                hdr[3] = hdr3;
                                atomicAdd(&P.out[inst].outstanding, 1);
                            }
                            __threadfence();
                            __syncwarp();
                            if (lane == 0) {
                                st_release_u32(&P.mail[target].flag, 1u);
                                ++S.stats[kStatDonations];
                            }
                        }
                        // A range split keeps at least one chunk of the donor's frame and a
                        // hand-off never touches the current frame's range (its pending mask
                        // is empty here), so the donor carries on with its next chunk.
                    }
                }
                // ---------------------------------------------------- evaluate a chunk
                uint32_t tr, a, b, c;
                bool valid;
                int nValid;
                chunk = cursor;
                if (sf.mode == 1) {
                    // one same-cycle position pair (p, q) per chunk, lane = third position r
                    cursor += 1;
                    const PairSel ps = sparse_pair(sf, chunk);
                    const uint32_t r = (uint32_t)lane;
                    valid = (int)r < n && (int)r != ps.p && (int)r != ps.q &&
                            (sf.leaderPos != ps.leader || (int)r > ps.q);
                    const uint32_t symP = w_pi(__shfl_sync(kFull, w[0], ps.p));
                    const uint32_t symQ = w_pi(__shfl_sync(kFull, w[0], ps.q));
                    const uint32_t symR = w_pi(w[0]);
                    if ((int)r < ps.p) {
                        tr = pack_triple(r, ps.p, ps.q);
                        a = symR, b = symP, c = symQ;
                    } else if ((int)r < ps.q) {
                        tr = pack_triple(ps.p, r, ps.q);
                        a = symP, b = symR, c = symQ;
                    } else {
                        tr = pack_triple(ps.p, ps.q, r);
                        a = symP, b = symQ, c = symR;
                    }
                    if (!valid) tr = a = b = c = 0u;
                    nValid = __popc(__ballot_sync(kFull, valid));
                } else {
                    // 32 consecutive triples: from the frame's same-cycle list (mode 2) or the
                    // lexicographic table (mode 0, in learned order at a root that has one)
                    const int t = cursor + lane;
                    cursor += 32;
                    valid = t < end;
                    if (sf.mode == 2) {
                        tr = valid ? S.tri[t] : 0u;
                    } else {
                        tr = valid ? decode(f, t) : 0u;
                        if (tr == 0xFFFFFFFFu) {
                            valid = false;
                            tr = 0u;
                        }
                    }
                    a = w_pi(gather<NW>(w, tri_i(tr)));
                    b = w_pi(gather<NW>(w, tri_j(tr)));
                    c = w_pi(gather<NW>(w, tri_k(tr)));
                    nValid = min(32, end - chunk);
                }
                const uint32_t wa = gather<NW>(w, a);
                const uint32_t wb = gather<NW>(w, b);
                const uint32_t wc = gather<NW>(w, c);
                const int e = even + move_delta(wa, wb, wc);
                const bool sat = valid && ((satMask >> e) & 1ull);
                if (lane == 0) S.taskChildren += (unsigned long long)nValid;
                const unsigned satBallot = __ballot_sync(kFull, sat);
                if (satBallot) {
                    const int winner = __ffs(satBallot) - 1;
                    const uint32_t wtr = __shfl_sync(kFull, tr, winner);
                    int won = 0;
                    if (lane == 0) won = atomicCAS(&P.out[inst].state, kStateRunning, kStateFound) == kStateRunning;
                    won = __shfl_sync(kFull, won, 0);
                    if (won) {
                        if (lane < f) P.out[inst].moves[lane] = S.frames[lane].move;
                        if (lane == f) {
                            P.out[inst].moves[f] = wtr;
                            P.out[inst].depth = f + 1;
                        }
                        __threadfence();
                    }
                    outcome = 1;
                    break;
                }
                bool probe = valid && ((expMask >> e) & 1ull);
                if (P.commute && f > 0) {
                    // the move that reached this frame and its symbols (y now at I, x at I+K-J, z at K)
                    const uint32_t inc = S.frames[f - 1].move;
                    const uint32_t I = tri_i(inc), J = tri_j(inc), K = tri_k(inc);
                    const uint32_t y = w_pi(gather<NW>(w, I)), x = w_pi(gather<NW>(w, I + K - J)),
                                   z = w_pi(gather<NW>(w, K));
                    const bool skip = probe && por_skip(inc, x, y, z, tri_i(tr), tri_j(tr), tri_k(tr), a, b, c);
                    const unsigned skipped = __ballot_sync(kFull, skip);
                    if (lane == 0) S.stats[kStatCommuteSkips] += (unsigned)__popc(skipped);
                    probe = probe && !skip;
                }
                // A child whose own children can only be tested for success (no node two levels
                // down is admitted for expansion) is cheaper to expand again than to look up:
                // unless probe_leaves is set it is admitted without touching the table.
                bool leafAdmit = false;
                if (!P.probeLeaves && (f + 2 > kMaxDepth || S.rules[16 + f + 2] == 0ull)) {
                    leafAdmit = probe;
                    probe = false;
                }
                const unsigned probing = __ballot_sync(kFull, probe);
                uint32_t outc = leafAdmit ? kAdmitted : 0u;
                if (probing) {
                    uint64_t ck[KW];
#pragma unroll
                    for (int q = 0; q < KW; ++q) ck[q] = key[q];
                    set_field<NW>(ck, a, w_spi(wc));
                    set_field<NW>(ck, b, w_spi(wa));
                    set_field<NW>(ck, c, w_spi(wb));
                    const uint32_t r =
                        dedup_admit_warp<KW>(P, generation, tag, probing, ck, key_hash<KW>(ck, tag), (uint32_t)(f + 1), lane);
                    if (probe) outc = r;
                }
                pending = __ballot_sync(kFull, outc & kAdmitted);
                const unsigned atomics = __ballot_sync(kFull, outc & kAtomic);
                if (probing) {
                    const unsigned ins = __ballot_sync(kFull, outc & kInserted);
                    const unsigned full = __ballot_sync(kFull, outc & kWindowFull);
                    const unsigned repl = __ballot_sync(kFull, outc & kReplaced);
                    if (lane == 0) {
                        S.stats[kStatDedupProbes] += (unsigned)__popc(probing);
                        S.stats[kStatDedupPruned] += (unsigned)__popc(probing & ~pending);
                        S.stats[kStatDedupInserts] += (unsigned)__popc(ins);
                        S.stats[kStatDedupFull] += (unsigned)__popc(full);
                        S.stats[kStatDedupReplaced] += (unsigned)__popc(repl);
                        S.stats[kStatTableAtomics] += (unsigned)__popc(atomics);
                    }
                }
                continue;
            }
            // -------------------------------------------------------- descend
            const int l = __ffs(pending) - 1;
            pending &= pending - 1u;
            uint32_t tr;
            if (sf.mode == 1) {
                const PairSel ps = sparse_pair(sf, chunk);
                const int r = l;
                tr = (r < ps.p) ? pack_triple(r, ps.p, ps.q)
                                : (r < ps.q) ? pack_triple(ps.p, r, ps.q) : pack_triple(ps.p, ps.q, r);
            } else if (sf.mode == 2) {
                tr = S.tri[chunk + l];
            } else {
                const int t = chunk + l;
                tr = decode(f, t);
            }
            if (lane == 0) {
                FrameRec<KW> &fr = S.frames[f];
                fr.cursor = cursor;
                fr.end = end;
                fr.pending = pending;
                fr.chunk = chunk;
                fr.even = even;
                fr.step = sf.mode == 1 ? 1 : 32;
                fr.move = tr;
#pragma unroll
                for (int q = 0; q < KW; ++q) fr.key[q] = key[q];
                // leaving the root: the child's rank in the root's learned order
                if (f == 0) S.rank1 = rootOrder ? chunk + l : -1;
            }
            __syncwarp();
            const uint32_t i = tri_i(tr), j = tri_j(tr), k = tri_k(tr);
            const uint32_t a = w_pi(gather<NW>(w, i));
            const uint32_t b = w_pi(gather<NW>(w, j));
            const uint32_t c = w_pi(gather<NW>(w, k));
            const uint32_t wa = gather<NW>(w, a);
            const uint32_t wb = gather<NW>(w, b);
            const uint32_t wc = gather<NW>(w, c);
            const int delta = move_delta(wa, wb, wc);
            even += delta;
            set_field<NW>(key, a, w_spi(wc));
            set_field<NW>(key, b, w_spi(wa));
            set_field<NW>(key, c, w_spi(wb));
            uint32_t nw[NW];
            apply_move<NW>(w, nw, lane, i, j, k, a, b, c, wa, wb, wc);
            // A +2 move with a, b, c in one cycle splits it into three arcs: the cycle fields
            // follow per lane from a, b and c (no shuffles); other moves rebuild them.
            const bool split = delta == 2 && w_leader(wa) == w_leader(wb) && w_leader(wb) == w_leader(wc);
#pragma unroll
            for (int h = 0; h < NW; ++h) {
                const int x = lane + 32 * h;
                if (split && x < n) nw[h] |= split_cycle_fields(w[h], a, b, c, wa, wb, wc) & ~0xFFFu;
                w[h] = nw[h];
            }
            if (!split) build_tables<NW>(w, n, lane);
            ++f;
#pragma unroll
            for (int h = 0; h < NW; ++h) S.words[f][h * 32 + lane] = w[h];
            satMask = S.rules[f + 1];
            expMask = S.rules[16 + f + 1];
            sf = sparse_setup<NW>(w, n, lane, even, satMask, expMask, ordered(f) ? 0 : P.sparse, S.tri);
            cursor = 0;
            end = sf.mode ? sf.np : denseEnd(f);
            pending = 0u;
            if (lane == 0) ++S.taskNodes;
        }
        if (lane == 0) {
            S.stats[kStatNodes] += S.taskNodes;
            S.stats[kStatChildren] += S.taskChildren;
        }
        if (outcome == 2) {
            if (lane == 0) S.stats[kStatBusyCycles] += (unsigned long long)clock64();
            stopAll = true;
            break;
        }
        // ---------------------------------------------------------------- finish task
        if (lane == 0) {
            S.stats[kStatBusyCycles] += (unsigned long long)clock64();
            atomicAdd(&P.out[inst].nodes, S.taskNodes);
            atomicAdd(&P.out[inst].children, S.taskChildren);
            const int prev = atomicSub(&P.out[inst].outstanding, 1);
            if (prev == 1) {
                atomicCAS(&P.out[inst].state, kStateRunning, kStateNotFound);
                atomicOr(P.doneBits + (inst >> 5), 1u << (inst & 31u));
                __threadfence();
                atomicAdd(&ctl->doneCount, 1);
            }
        }
        __syncwarp();
    }

    // ---------------------------------------------------------------- statistics
    if (lane == 0) {
        atomicAdd(&ctl->stats[kStatNodes], S.stats[kStatNodes]);
        atomicAdd(&ctl->stats[kStatChildren], S.stats[kStatChildren]);
        atomicAdd(&ctl->stats[kStatDedupProbes], S.stats[kStatDedupProbes]);
        atomicAdd(&ctl->stats[kStatDedupPruned], S.stats[kStatDedupPruned]);
        atomicAdd(&ctl->stats[kStatDedupInserts], S.stats[kStatDedupInserts]);
        atomicAdd(&ctl->stats[kStatDedupFull], S.stats[kStatDedupFull]);
        atomicAdd(&ctl->stats[kStatDonations], S.stats[kStatDonations]);
        atomicAdd(&ctl->stats[kStatTaskPops], S.stats[kStatTaskPops]);
        atomicAdd(&ctl->stats[kStatDedupReplaced], S.stats[kStatDedupReplaced]);
        atomicAdd(&ctl->stats[kStatTableAtomics], S.stats[kStatTableAtomics]);
        atomicAdd(&ctl->stats[kStatCommuteSkips], S.stats[kStatCommuteSkips]);
        S.stats[kStatWarpCycles] += (unsigned long long)clock64();
        atomicAdd(&ctl->stats[kStatBusyCycles], S.stats[kStatBusyCycles]);
        atomicAdd(&ctl->stats[kStatWarpCycles], S.stats[kStatWarpCycles]);
    }
}

}  // namespace dev
}  // namespace tdp
