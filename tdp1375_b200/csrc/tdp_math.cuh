// Shared arithmetic of the transposition search: usable from device code and from
// host code (the host runtime builds the rule tables with the same functions, and a
// host-only unit test checks the O(1) move delta against a full recount).
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define TDP_HD __host__ __device__ __forceinline__
#else
#define TDP_HD inline
#endif

#ifndef __CUDACC__
#include <math.h>
#endif

namespace tdp {

constexpr int kMaxN = 63;      // MAX_N of the reference (core/common.cuh:33-35)
constexpr int kMaxDepth = 15;  // MAX_DEPTH of the reference (core/common.cuh:29-31)

// ---------------------------------------------------------------------------
// Per-symbol word.  Every lane of a warp owns symbol/position x = lane + 32*h and
// keeps one 32-bit word for it:
//   bits  0..5   spi[x]          image of symbol x under spi
//   bits  6..11  pi[x]           symbol written at position x of the pi array
//   bits 12..17  leader(x)       anchor of x's spi-cycle: its smallest symbol after a full
//                                rebuild, the cycle's last moved symbol after a split
//                                (split_cycle_fields); any one symbol per cycle works
//   bits 18..23  s2l(x)          steps from x to its leader following spi
//   bits 24..30  len(x)          length of x's spi-cycle
// ---------------------------------------------------------------------------
TDP_HD uint32_t w_spi(uint32_t w) { return w & 63u; }
TDP_HD uint32_t w_pi(uint32_t w) { return (w >> 6) & 63u; }
TDP_HD uint32_t w_leader(uint32_t w) { return (w >> 12) & 63u; }
TDP_HD uint32_t w_s2l(uint32_t w) { return (w >> 18) & 63u; }
TDP_HD uint32_t w_len(uint32_t w) { return (w >> 24) & 127u; }
TDP_HD uint32_t w_make(uint32_t spi, uint32_t pi, uint32_t leader, uint32_t s2l, uint32_t len) {
    return spi | (pi << 6) | (leader << 12) | (s2l << 18) | (len << 24);
}

// Change in the number of odd-length spi-cycles ("even cycles" in the reference,
// SortingSearch.java:120-122) when spi becomes spi o (a b c)^-1, from the cycle words
// of a, b and c.  The reference recounts every child in O(n)
// (sorting_search.cu:302-317, 557); the cycle-split/merge rules below give the same
// number in O(1):
//   three distinct cycles -> one cycle of length La+Lb+Lc;
//   a,b in one cycle, c in another -> lengths Lc+d(b,a) and d(a,b);
//   b,c together, a alone         -> lengths La+d(c,b) and d(b,c);
//   a,c together, b alone         -> lengths Lb+d(a,c) and d(c,a);
//   all three in one cycle, spi-order a->b->c -> lengths d(a,b), d(b,c), d(c,a);
//   all three in one cycle, spi-order a->c->b -> one cycle of the same length.
// d(x,y) is the number of spi steps from x to y.
TDP_HD int move_delta(uint32_t wa, uint32_t wb, uint32_t wc) {
    const int ca = (int)w_leader(wa), cb = (int)w_leader(wb), cc = (int)w_leader(wc);
    const int sa = (int)w_s2l(wa), sb = (int)w_s2l(wb), sc = (int)w_s2l(wc);
    const int La = (int)w_len(wa), Lb = (int)w_len(wb), Lc = (int)w_len(wc);
    if (ca == cb) {
        int dab = sa - sb;
        if (dab < 0) dab += La;
        if (cb == cc) {
            int dac = sa - sc;
            if (dac < 0) dac += La;
            if (dab > dac) return 0;
            return (dab & 1) + ((dac - dab) & 1) + ((La - dac) & 1) - (La & 1);
        }
        return ((Lc + La - dab) & 1) + (dab & 1) - (La & 1) - (Lc & 1);
    }
    if (cb == cc) {
        int dbc = sb - sc;
        if (dbc < 0) dbc += Lb;
        return ((La + Lb - dbc) & 1) + (dbc & 1) - (Lb & 1) - (La & 1);
    }
    if (ca == cc) {
        int dac = sa - sc;
        if (dac < 0) dac += La;
        return ((Lb + dac) & 1) + ((La - dac) & 1) - (La & 1) - (Lb & 1);
    }
    return ((La + Lb + Lc) & 1) - (La & 1) - (Lb & 1) - (Lc & 1);
}

// Cycle fields of symbol x after the move (a b c) when a, b and c lie in one cycle in the
// spi-order a -> b -> c (the split case of move_delta, a +2 change): the cycle breaks into
// the arcs (a, b], (b, c] and (c, a], each anchored at its last element (b, c and a), with
// steps counted forward to the anchor.  wx is x's word before the move; its spi/pi fields
// are kept and words of other cycles are returned unchanged.  This replaces a full
// pointer-jumping rebuild of the cycle fields after such a move.
TDP_HD uint32_t split_cycle_fields(uint32_t wx, uint32_t a, uint32_t b, uint32_t c, uint32_t wa, uint32_t wb,
                                   uint32_t wc) {
    if (w_leader(wx) != w_leader(wa)) return wx;
    const int L = (int)w_len(wa);
    const int sa = (int)w_s2l(wa);
    int dB = sa - (int)w_s2l(wb);  // forward distance a -> b
    if (dB < 0) dB += L;
    int dC = sa - (int)w_s2l(wc);  // a -> c
    if (dC < 0) dC += L;
    int dx = sa - (int)w_s2l(wx);  // a -> x
    if (dx < 0) dx += L;
    uint32_t anchor, steps, len;
    if (dx >= 1 && dx <= dB) {
        anchor = b, len = (uint32_t)dB, steps = (uint32_t)(dB - dx);
    } else if (dx > dB && dx <= dC) {
        anchor = c, len = (uint32_t)(dC - dB), steps = (uint32_t)(dC - dx);
    } else {
        anchor = a, len = (uint32_t)(L - dC), steps = dx == 0 ? 0u : (uint32_t)(L - dx);
    }
    return (wx & 0xFFFu) | (anchor << 12) | (steps << 18) | (len << 24);
}

// Block swap of [i,j) and [j,k) as a gather index (transposition.cuh:5-11).
TDP_HD int block_swap_src(int p, int i, int j, int k) {
    const int lenA = j - i, lenB = k - j;
    const int inLow = (p >= i) & (p < i + lenB);
    const int inHigh = (p >= i + lenB) & (p < k);
    return p + inLow * lenA - inHigh * lenB;
}

// Packed triple of positions (i<j<k), 6 bits each, like PackedMove (core/common.cuh:37-63).
TDP_HD uint32_t pack_triple(uint32_t i, uint32_t j, uint32_t k) { return i | (j << 6) | (k << 12); }
TDP_HD uint32_t tri_i(uint32_t t) { return t & 63u; }
TDP_HD uint32_t tri_j(uint32_t t) { return (t >> 6) & 63u; }
TDP_HD uint32_t tri_k(uint32_t t) { return (t >> 12) & 63u; }

TDP_HD int combinations3(int n) { return n < 3 ? 0 : n * (n - 1) * (n - 2) / 6; }
TDP_HD int combinations4(int n) { return n < 4 ? 0 : n * (n - 1) * (n - 2) * (n - 3) / 24; }

// ---------------------------------------------------------------------------
// The verdict-defining float32 rule of sorting_search.cu:321-362, evaluated once per
// (odd-cycle count, depth) on the host into bit tables.  Host float arithmetic is
// IEEE binary32 with round-to-nearest, as is CUDA's default (no fast-math), so the
// tables hold exactly the bits the reference kernel would compute.
// ---------------------------------------------------------------------------
struct RuleParams {
    int n;
    int initialEven;
    int maxDepth;
    float minRate;
    int fullSorting;
};

// satisfies_rate (sorting_search.cu:321-331)
inline bool rule_satisfies(const RuleParams &r, int even, int depth) {
    if (depth <= 0) return false;
    if (r.fullSorting && even != r.n) return false;
    const int gained = even - r.initialEven;
    const float achieved = (float)gained / (float)depth;
    return gained > 0 && achieved >= r.minRate;
}

// can_still_reach (sorting_search.cu:333-362)
inline bool rule_can_still_reach(const RuleParams &r, int even, int depth) {
    const int gained = even - r.initialEven;
    const int movesLeft = r.maxDepth - depth;
    if (movesLeft < 0) return false;
    const int maxPossible = r.n - even;
    if (r.fullSorting) {
        const int lowerBound = (maxPossible + 1) / 2;
        if (depth + lowerBound > r.maxDepth) return false;
        const int optimistic = gained + 2 * movesLeft;
        const float inner = (float)depth + ceilf((float)maxPossible / 2.0f);
        if ((float)optimistic < ceilf(r.minRate * inner)) return false;
    } else {
        const int optimistic = gained + 2 * movesLeft;
        const int requiredAtMax = (int)floorf(r.minRate * (float)r.maxDepth);
        if (optimistic < requiredAtMax) return false;
        const int lowerBound = (maxPossible + 1) / 2;
        const int bestDepth = depth + lowerBound;
        if (bestDepth > 0) {
            const float ratio = (float)(gained + maxPossible) / (float)bestDepth;
            if (ratio < r.minRate) return false;
        }
    }
    return true;
}

// Verdict-preserving strengthening used by this engine only.  A node (depth, even)
// can lead to a success only if some final depth L in (depth, maxDepth] passes
// rule_satisfies with the largest odd-cycle count still reachable,
// min(even + 2(L - depth), n): a move changes the count by -2, 0 or +2, and
// rule_satisfies is monotone in the count for a fixed depth (in full-sorting mode only
// count == n succeeds).  Pruning with it never removes a success path, so verdicts are
// those of the reference rule; it only shrinks the explored tree.
inline bool rule_success_reachable(const RuleParams &r, int even, int depth) {
    for (int L = depth + 1; L <= r.maxDepth; ++L) {
        int best = even + 2 * (L - depth);
        if (best > r.n) best = r.n;
        if (r.fullSorting && best != r.n) continue;
        if (rule_satisfies(r, best, L)) return true;
    }
    return false;
}

// Bit tables: bit e of sat[d] = a node at depth d with e odd cycles is a success;
// bit e of expand[d] = such a node is admitted for expansion (d < maxDepth and
// can_still_reach, and, when tight, rule_success_reachable).
struct RuleTable {
    uint64_t sat[kMaxDepth + 1];
    uint64_t expand[kMaxDepth + 1];
};

inline RuleTable build_rule_table(const RuleParams &r, bool tight) {
    RuleTable t;
    for (int d = 0; d <= kMaxDepth; ++d) {
        uint64_t s = 0, x = 0;
        for (int e = 0; e <= r.n && e < 64; ++e) {
            if (d <= r.maxDepth && rule_satisfies(r, e, d)) s |= (1ull << e);
            if (d < r.maxDepth && rule_can_still_reach(r, e, d) && (!tight || rule_success_reachable(r, e, d)))
                x |= (1ull << e);
        }
        t.sat[d] = s;
        t.expand[d] = x;
    }
    return t;
}

}  // namespace tdp
