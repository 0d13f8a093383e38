// CPU ORACLE — TEST INFRASTRUCTURE ONLY.
//
// This file restates, on the host and in plain C++17, the arithmetic of the
// reference's transposition-sequence search and permutation filter so that the
// CUDA product can be checked against it.  Only the test-suite, the smoke test
// and the CPU-baseline leg of the benchmark may load it.  Nothing in the
// product links or calls it.
//
// Parity pins for this file (all checked by tests/test_oracle_golden.py):
//   * src/main/resources/cases/cases-comb.txt (673 known positives),
//     cases-3,2.txt (16) and cases-oriented-7cycle.txt (1): every listed
//     sequence replays as a valid sorting within the ratio, and the GPU-rule
//     search below answers "found" for every listed configuration;
//   * CommonOperationsTest.java:21-24 and PermutationGroupsTest.java:10-12:
//     block-swap / left-product algebra of a move.
// There is no reference fixture for negative verdicts or for the pi filter;
// those are cross-checked between independent formulations (brute force,
// with and without the transposition table) in the tests.
//
// Functions and the reference lines they restate:
//   oracle_count_even_cycles      sorting_search.cu:302-317 (odd-length cycles,
//                                 fixed points included: SortingSearch.java:120-122)
//   gpu_satisfies / gpu_reach     sorting_search.cu:321-362 (float32 rule, both modes)
//   oracle_search_gpu_rule        sorting_search.cu:377-615 semantics as a sequential
//                                 DFS (root always expanded, children checked for
//                                 success first, then depth/prune/dedup), lexicographic
//                                 (i,j,k) order on the current pi array, block swap
//                                 transposition.cuh:5-19
//   oracle_search_cpu_rule        SortingSearch.java:35-118 (double-precision prune,
//                                 full sorting only, symbols returned)
//   oracle_replay_positions       GPUSortingSearch.java:65-87 (positions -> symbols by
//                                 replaying block swaps) + the ratio check of
//                                 SortingSearch.java:46-53 / sorting_search.cu:321-331
//   oracle_pi_filter              pi_filter.cu:38-154 (factoradic rank order, the
//                                 three predicates), CommonOperations.java:167-182,
//                                 406-445
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

namespace {

constexpr int kMaxN = 63;
constexpr int kMaxDepth = 15;

int count_even(const uint8_t *spi, int n) {
    uint64_t visited = 0;
    int count = 0;
    for (int s = 0; s < n; ++s) {
        if (visited & (1ULL << s)) continue;
        int size = 0, cur = s;
        do {
            visited |= (1ULL << cur);
            ++size;
            cur = spi[cur];
        } while (cur != s);
        if (size & 1) ++count;
    }
    return count;
}

// Block swap of [i,j) and [j,k): transposition.cuh:5-11 restated.
int src_index(int p, int i, int j, int k) {
    const int lenA = j - i, lenB = k - j;
    if (p >= i && p < i + lenB) return p + lenA;
    if (p >= i + lenB && p < k) return p - lenB;
    return p;
}

void apply_block_swap(const uint8_t *pi, int n, int i, int j, int k, uint8_t *out) {
    for (int p = 0; p < n; ++p) out[p] = pi[src_index(p, i, j, k)];
}

// spi' = spi o (a b c)^-1 : sorting_search.cu:543-555.
void apply_spi(uint8_t *spi, int a, int b, int c) {
    const uint8_t av = spi[a], bv = spi[b], cv = spi[c];
    spi[a] = cv;
    spi[b] = av;
    spi[c] = bv;
}

struct Rule {
    int n;
    int initialEven;
    int maxDepth;
    float minRate;
    int fullSorting;
};

// sorting_search.cu:321-331, float32.
bool gpu_satisfies(const Rule &r, int even, int depth) {
    if (depth <= 0) return false;
    if (r.fullSorting && even != r.n) return false;
    const int gained = even - r.initialEven;
    const float achieved = static_cast<float>(gained) / static_cast<float>(depth);
    return gained > 0 && achieved >= r.minRate;
}

// sorting_search.cu:333-362, float32.
bool gpu_reach(const Rule &r, int even, int depth) {
    const int gained = even - r.initialEven;
    const int movesLeft = r.maxDepth - depth;
    if (movesLeft < 0) return false;
    const int maxPossible = r.n - even;
    if (r.fullSorting) {
        const int lowerBound = (maxPossible + 1) / 2;
        if (depth + lowerBound > r.maxDepth) return false;
        const int optimistic = gained + 2 * movesLeft;
        const float inner = static_cast<float>(depth) + ceilf(static_cast<float>(maxPossible) / 2.0f);
        if (static_cast<float>(optimistic) < ceilf(r.minRate * inner)) return false;
    } else {
        const int optimistic = gained + 2 * movesLeft;
        const int requiredAtMax = static_cast<int>(floorf(r.minRate * static_cast<float>(r.maxDepth)));
        if (optimistic < requiredAtMax) return false;
        const int lowerBound = (maxPossible + 1) / 2;
        const int bestDepth = depth + lowerBound;
        if (bestDepth > 0) {
            const float ratio = static_cast<float>(gained + maxPossible) / static_cast<float>(bestDepth);
            if (ratio < r.minRate) return false;
        }
    }
    return true;
}


// Verdict-preserving strengthening of gpu_reach (not in the reference): a node at
// (depth, even) can lead to a success only if some final depth L in (depth, maxDepth]
// admits a success with the largest gain still reachable, min(gained + 2(L-depth),
// n - initialEven) (each move changes the odd-cycle count by -2, 0 or +2), tested with
// gpu_satisfies itself.  In full-sorting mode the final state must have even == n.
bool tight_reach(const Rule &r, int even, int depth) {
    const int gained = even - r.initialEven;
    const int cap = r.n - r.initialEven;
    for (int L = depth + 1; L <= r.maxDepth; ++L) {
        int g = gained + 2 * (L - depth);
        if (g > cap) g = cap;
        if (r.fullSorting && g != cap) continue;
        if (gpu_satisfies(r, r.initialEven + g, L)) return true;
    }
    return false;
}

// Partial-order reduction (not in the reference; verdict-preserving, used by the engine's
// `commute` option).  At a node N reached by the move (x y z) at positions I<J<K of its
// parent P, the child (a b c) at positions i<j<k of N is skipped when {a,b,c} and {x,y,z}
// are disjoint, (a b c) is also a move at P (a, b, c in cyclic order there), (x y z) is a
// move after it, and the sorted triple (a,b,c) is smaller than the sorted (x,y,z): then
// P.(a b c).(x y z) reaches the same state (disjoint 3-cycles commute) through the kept
// order.  Positions in P follow from N's by the inverse block swap of (I,J,K).
bool cyclic3(int pa, int pb, int pc) { return ((pa > pb) + (pb > pc) + (pc > pa)) <= 1; }

bool por_skip(const uint8_t *pi, int I, int J, int K, int i, int j, int k) {
    const int a = pi[i], b = pi[j], c = pi[k];
    const int y = pi[I], x = pi[I + K - J], z = pi[K];
    if (a == x || a == y || a == z || b == x || b == y || b == z || c == x || c == y || c == z) return false;
    const int pa = src_index(i, I, J, K), pb = src_index(j, I, J, K), pc = src_index(k, I, J, K);
    if (!cyclic3(pa, pb, pc)) return false;
    int q[3] = {pa, pb, pc};
    std::sort(q, q + 3);
    auto fwd = [&](int p) {
        if (p >= q[0] && p < q[1]) return p + (q[2] - q[1]);
        if (p >= q[1] && p < q[2]) return p - (q[1] - q[0]);
        return p;
    };
    if (!cyclic3(fwd(I), fwd(J), fwd(K))) return false;
    int me[3] = {a, b, c}, in[3] = {x, y, z};
    std::sort(me, me + 3);
    std::sort(in, in + 3);
    return std::lexicographical_compare(me, me + 3, in, in + 3);
}

struct GpuRuleDfs {
    Rule rule;
    bool useDedup;
    bool tight = false;
    bool por = false;
    std::unordered_map<std::string, int> memo;
    uint64_t expanded = 0;
    uint64_t children = 0;
    uint64_t nodeLimit = 0;  // 0 = unlimited
    bool aborted = false;
    int path[kMaxDepth][3];
    int found = 0;
    int foundDepth = 0;

    bool admit(const uint8_t *spi, int depth) {
        if (!useDedup) return true;
        std::string key(reinterpret_cast<const char *>(spi), rule.n);
        auto it = memo.find(key);
        if (it == memo.end()) {
            memo.emplace(std::move(key), depth);
            return true;
        }
        if (it->second <= depth) return false;
        it->second = depth;
        return true;
    }

    // Expands the node (spi, pi) that sits at `depth`; returns true once found.
    bool expand(const uint8_t *spi, const uint8_t *pi, int depth) {
        if (nodeLimit && expanded >= nodeLimit) {
            aborted = true;
            return false;
        }
        ++expanded;
        const int n = rule.n;
        const int childDepth = depth + 1;
        uint8_t childSpi[kMaxN + 1];
        uint8_t childPi[kMaxN + 1];
        for (int i = 0; i < n - 2; ++i)
            for (int j = i + 1; j < n - 1; ++j)
                for (int k = j + 1; k < n; ++k) {
                    ++children;
                    std::memcpy(childSpi, spi, n);
                    apply_spi(childSpi, pi[i], pi[j], pi[k]);
                    const int even = count_even(childSpi, n);
                    path[depth][0] = i;
                    path[depth][1] = j;
                    path[depth][2] = k;
                    if (gpu_satisfies(rule, even, childDepth)) {
                        found = 1;
                        foundDepth = childDepth;
                        return true;
                    }
                    if (childDepth < rule.maxDepth && gpu_reach(rule, even, childDepth) &&
                        (!tight || tight_reach(rule, even, childDepth)) &&
                        !(por && depth > 0 &&
                          por_skip(pi, path[depth - 1][0], path[depth - 1][1], path[depth - 1][2], i, j, k)) &&
                        admit(childSpi, childDepth)) {
                        apply_block_swap(pi, n, i, j, k, childPi);
                        if (expand(childSpi, childPi, childDepth)) return true;
                        if (aborted) return false;
                    }
                }
        return false;
    }
};

struct CpuRuleDfs {
    int n;
    int initialEven;
    float minRate;
    int maxMoves;
    uint64_t expanded = 0;
    uint64_t nodeLimit = 0;
    bool aborted = false;
    int moves[kMaxDepth][3];

    // SortingSearch.java:35-104; spi and pi are updated in place and undone.
    int search(uint8_t *spi, uint8_t *pi, int depth) {
        const int even = count_even(spi, n);
        if (even == n) {
            const int gained = even - initialEven;
            const float achieved = static_cast<float>(gained) / static_cast<float>(depth);
            return (achieved >= minRate) ? depth : 0;
        }
        if (depth == maxMoves) return 0;
        const int gained = even - initialEven;
        const int movesLeft = maxMoves - depth;
        const int maxPossible = n - even;
        const double bound = std::ceil(static_cast<double>(minRate) *
                                       (static_cast<double>(depth) + std::ceil(maxPossible / 2.0)));
        if (static_cast<double>(gained + movesLeft * 2) < bound) return 0;
        const int lowerBound = static_cast<int>(std::ceil(maxPossible / 2.0));
        if (depth + lowerBound > maxMoves) return 0;
        if (nodeLimit && expanded >= nodeLimit) {
            aborted = true;
            return 0;
        }
        ++expanded;
        uint8_t saved[kMaxN + 1];
        for (int i = 0; i < n - 2; ++i)
            for (int j = i + 1; j < n - 1; ++j)
                for (int k = j + 1; k < n; ++k) {
                    const int a = pi[i], b = pi[j], c = pi[k];
                    const uint8_t av = spi[a], bv = spi[b], cv = spi[c];
                    apply_spi(spi, a, b, c);
                    moves[depth][0] = a;
                    moves[depth][1] = b;
                    moves[depth][2] = c;
                    std::memcpy(saved, pi, n);
                    apply_block_swap(saved, n, i, j, k, pi);
                    const int result = search(spi, pi, depth + 1);
                    if (result > 0) return result;
                    std::memcpy(pi, saved, n);
                    spi[a] = av;
                    spi[b] = bv;
                    spi[c] = cv;
                    if (aborted) return 0;
                }
        return 0;
    }
};

// ---- pi filter predicates: pi_filter.cu:55-115 -----------------------------

bool cyclic_order(const uint8_t *index, const uint8_t *symbols, int count) {
    int leaps = 0;
    for (int i = 0; i < count; ++i) {
        if (index[symbols[i]] > index[symbols[(i + 1) % count]]) {
            if (++leaps > 1) return false;
        }
    }
    return true;
}

bool cyclic_order3(const uint8_t *index, int a, int b, int c) {
    int leaps = 0;
    if (index[a] > index[b]) ++leaps;
    if (index[b] > index[c]) ++leaps;
    if (index[c] > index[a]) ++leaps;
    return leaps <= 1;
}

int cycle_distance(const uint8_t *cycleIndex, int len, int a, int b) {
    const int ai = cycleIndex[a], bi = cycleIndex[b];
    return (bi >= ai) ? bi - ai : (len - ai) + bi;
}

bool has_2_move(const uint8_t *piIndex, const uint8_t *cycle, const uint8_t *cycleIndex, int len) {
    const int before = (len % 2 == 1) ? 1 : 0;
    for (int i = 0; i < len - 2; ++i)
        for (int j = i + 1; j < len - 1; ++j)
            for (int k = j + 1; k < len; ++k) {
                const int a = cycle[i], b = cycle[j], c = cycle[k];
                if (!cyclic_order3(piIndex, a, b, c)) continue;
                const int after = (cycle_distance(cycleIndex, len, a, b) & 1) +
                                  (cycle_distance(cycleIndex, len, b, c) & 1) +
                                  (cycle_distance(cycleIndex, len, c, a) & 1);
                if (after - before == 2) return true;
            }
    return false;
}

}  // namespace

extern "C" {

int oracle_count_even_cycles(const uint8_t *spi, int n) { return count_even(spi, n); }

// Evaluates the float32 rule of sorting_search.cu:321-362 for one (even, depth).
// Returns bit0 = satisfies_rate, bit1 = can_still_reach.
int oracle_rule_eval(int n, int initialEven, float minRate, int maxDepth, int fullSorting, int even, int depth) {
    Rule r{n, initialEven, maxDepth, minRate, fullSorting};
    return (gpu_satisfies(r, even, depth) ? 1 : 0) | (gpu_reach(r, even, depth) ? 2 : 0);
}

// Sequential restatement of the GPU search semantics.
// Returns 1 found, 0 not found, -1 bad arguments, -2 node limit hit.
// outPositions receives depth*3 ints (positions on the current pi array, as the
// reference's JNI returns them); stats = {expanded nodes, children evaluated}.
int oracle_search_gpu_rule(const uint8_t *pi, const uint8_t *spi, int n, int initialEven, float minRate,
                           int maxDepth, int fullSorting, int useDedup, uint64_t nodeLimit,
                           int *outPositions, int *outDepth, uint64_t *stats) {
    *outDepth = 0;
    if (stats) stats[0] = stats[1] = 0;
    if (n > kMaxN || maxDepth <= 0 || maxDepth > kMaxDepth) return -1;
    if (n < 3) return 0;
    GpuRuleDfs dfs;
    dfs.rule = Rule{n, initialEven, maxDepth, minRate, fullSorting};
    dfs.useDedup = (useDedup & 1) != 0;
    dfs.tight = (useDedup & 2) != 0;
    dfs.por = (useDedup & 4) != 0;
    dfs.nodeLimit = nodeLimit;
    uint8_t s[kMaxN + 1], p[kMaxN + 1];
    std::memcpy(s, spi, n);
    std::memcpy(p, pi, n);
    dfs.expand(s, p, 0);
    if (stats) {
        stats[0] = dfs.expanded;
        stats[1] = dfs.children;
    }
    if (dfs.aborted) return -2;
    if (!dfs.found) return 0;
    *outDepth = dfs.foundDepth;
    for (int d = 0; d < dfs.foundDepth; ++d)
        for (int t = 0; t < 3; ++t) outPositions[d * 3 + t] = dfs.path[d][t];
    return 1;
}

// Restatement of SortingSearch.searchForSortingSeq (full sorting, double prune).
// Returns 1 found, 0 not found, -1 bad args, -2 node limit.  outSymbols gets
// depth*3 symbols (a,b,c) as the Java method returns them.
int oracle_search_cpu_rule(const uint8_t *pi, const uint8_t *spi, int n, int initialEven, float minRate,
                           int maxMoves, uint64_t nodeLimit, int *outSymbols, int *outDepth, uint64_t *stats) {
    *outDepth = 0;
    if (stats) stats[0] = 0;
    if (n > kMaxN || maxMoves <= 0 || maxMoves > kMaxDepth) return -1;
    CpuRuleDfs dfs;
    dfs.n = n;
    dfs.initialEven = initialEven;
    dfs.minRate = minRate;
    dfs.maxMoves = maxMoves;
    dfs.nodeLimit = nodeLimit;
    uint8_t s[kMaxN + 1], p[kMaxN + 1];
    std::memcpy(s, spi, n);
    std::memcpy(p, pi, n);
    const int depth = dfs.search(s, p, 0);
    if (stats) stats[0] = dfs.expanded;
    if (dfs.aborted) return -2;
    if (depth <= 0) return 0;
    *outDepth = depth;
    for (int d = 0; d < depth; ++d)
        for (int t = 0; t < 3; ++t) outSymbols[d * 3 + t] = dfs.moves[d][t];
    return 1;
}

// Replays positions like GPUSortingSearch.java:65-74 and validates the result.
// Returns 1 when every move is a valid i<j<k triple and the final state meets the
// rule's success test (sorting_search.cu:321-331); 0 otherwise.  outSymbols (may be
// null) receives the symbol triples.
int oracle_replay_positions(const uint8_t *pi, const uint8_t *spi, int n, const int *positions, int depth,
                            int initialEven, float minRate, int fullSorting, int *outSymbols) {
    if (depth <= 0 || depth > kMaxDepth || n > kMaxN) return 0;
    uint8_t p[kMaxN + 1], s[kMaxN + 1], t[kMaxN + 1];
    std::memcpy(p, pi, n);
    std::memcpy(s, spi, n);
    for (int d = 0; d < depth; ++d) {
        const int i = positions[d * 3], j = positions[d * 3 + 1], k = positions[d * 3 + 2];
        if (!(0 <= i && i < j && j < k && k < n)) return 0;
        const int a = p[i], b = p[j], c = p[k];
        if (outSymbols) {
            outSymbols[d * 3] = a;
            outSymbols[d * 3 + 1] = b;
            outSymbols[d * 3 + 2] = c;
        }
        apply_spi(s, a, b, c);
        apply_block_swap(p, n, i, j, k, t);
        std::memcpy(p, t, n);
    }
    Rule r{n, initialEven, kMaxDepth, minRate, fullSorting};
    return gpu_satisfies(r, count_even(s, n), depth) ? 1 : 0;
}

// Replays symbol 3-cycles (a b c) on (pi, spi): each move must have a,b,c in cyclic
// order in the current pi (AbstractSbtAlgorithm / Cycle semantics); returns the final
// even-cycle count, or -1 if a move is not a transposition of pi.
int oracle_replay_symbols(const uint8_t *pi, const uint8_t *spi, int n, const int *symbols, int depth,
                          uint8_t *outSpi) {
    uint8_t p[kMaxN + 1], s[kMaxN + 1], t[kMaxN + 1], idx[kMaxN + 1];
    std::memcpy(p, pi, n);
    std::memcpy(s, spi, n);
    for (int d = 0; d < depth; ++d) {
        const int a = symbols[d * 3], b = symbols[d * 3 + 1], c = symbols[d * 3 + 2];
        if (a < 0 || b < 0 || c < 0 || a >= n || b >= n || c >= n || a == b || b == c || a == c) return -1;
        for (int q = 0; q < n; ++q) idx[p[q]] = static_cast<uint8_t>(q);
        if (!cyclic_order3(idx, a, b, c)) return -1;
        int pos[3] = {idx[a], idx[b], idx[c]};
        // sort the three positions
        if (pos[0] > pos[1]) std::swap(pos[0], pos[1]);
        if (pos[1] > pos[2]) std::swap(pos[1], pos[2]);
        if (pos[0] > pos[1]) std::swap(pos[0], pos[1]);
        apply_spi(s, a, b, c);
        apply_block_swap(p, n, pos[0], pos[1], pos[2], t);
        std::memcpy(p, t, n);
    }
    if (outSpi) std::memcpy(outSpi, s, n);
    return count_even(s, n);
}

// pi_filter.cu:157-260 restated with a deterministic output order: every pi with
// pi[0]=0 over n symbols, visited in factoradic (lexicographic) rank order, kept when
// the three predicates hold.  Writes at most maxOut rows of n bytes, returns the
// total number of hits (which may exceed maxOut, like the reference's counter).
int64_t oracle_pi_filter(const uint8_t *cycle, int cycleLen, const uint8_t *triple, int tripleLen, int n,
                         int skip2MoveCheck, uint8_t *out, int64_t maxOut) {
    if (n < 1 || n > kMaxN) return -1;
    uint8_t cycleIndex[kMaxN + 1] = {0};
    for (int i = 0; i < cycleLen; ++i) cycleIndex[cycle[i]] = static_cast<uint8_t>(i);
    std::vector<uint8_t> perm(n);
    for (int i = 0; i < n; ++i) perm[i] = static_cast<uint8_t>(i);
    uint8_t index[kMaxN + 1], rindex[kMaxN + 1];
    int64_t hits = 0;
    while (true) {
        for (int i = 0; i < n; ++i) index[perm[i]] = static_cast<uint8_t>(i);
        bool keep = cyclic_order(index, triple, tripleLen);
        if (keep) {
            for (int i = 0; i < n; ++i) rindex[i] = static_cast<uint8_t>((n - 1) - index[i]);
            keep = !cyclic_order(rindex, cycle, cycleLen);
        }
        if (keep && !skip2MoveCheck) keep = !has_2_move(index, cycle, cycleIndex, cycleLen);
        if (keep) {
            if (hits < maxOut && out) std::memcpy(out + hits * n, perm.data(), n);
            ++hits;
        }
        // next permutation of perm[1..n-1] in lexicographic order
        int i = n - 2;
        while (i >= 1 && perm[i] > perm[i + 1]) --i;
        if (i < 1) break;
        int j = n - 1;
        while (perm[j] < perm[i]) --j;
        std::swap(perm[i], perm[j]);
        for (int l = i + 1, r = n - 1; l < r; ++l, --r) std::swap(perm[l], perm[r]);
    }
    return hits;
}

// Single-candidate predicate (used to check batched filter results).
int oracle_pi_filter_keep(const uint8_t *pi, int n, const uint8_t *cycle, int cycleLen, const uint8_t *triple,
                          int tripleLen, int skip2MoveCheck) {
    uint8_t cycleIndex[kMaxN + 1] = {0};
    for (int i = 0; i < cycleLen; ++i) cycleIndex[cycle[i]] = static_cast<uint8_t>(i);
    uint8_t index[kMaxN + 1], rindex[kMaxN + 1];
    for (int i = 0; i < n; ++i) index[pi[i]] = static_cast<uint8_t>(i);
    if (!cyclic_order(index, triple, tripleLen)) return 0;
    for (int i = 0; i < n; ++i) rindex[i] = static_cast<uint8_t>((n - 1) - index[i]);
    if (cyclic_order(rindex, cycle, cycleLen)) return 0;
    if (!skip2MoveCheck && has_2_move(index, cycle, cycleIndex, cycleLen)) return 0;
    return 1;
}

}  // extern "C"

// ---- extension filter (batched use of the pi_filter.cu:55-115 predicates) -----------------
// Candidates of a base configuration (spi, pi) over n symbols, in this order:
//   A. for every a<b<c (lexicographic) and orientation o in {0,1}: spi' = spi o rho with
//      rho = (a b c) (o = 0) or (a c b) (o = 1); pi' = pi; the added cycle is rho;
//   B. for every 0 <= g1 <= g2 <= g3 <= n (lexicographic) and orientation o: three new
//      symbols x=n, y=n+1, z=n+2 inserted into pi before original positions g1, g2, g3 (x
//      first on ties), spi' = spi plus the cycle (x y z) (o = 0) or (x z y) (o = 1).
// A candidate is kept when the added cycle, as written, is in cyclic order in pi'
// (pi_filter.cu:132-133), at least one cycle of spi' is oriented (pi_filter.cu:135-142,
// CommonOperations.java:443-445) and no oriented cycle of spi' admits a 2-move
// (pi_filter.cu:86-115, CommonOperations.java:406-431).
namespace {

int comb3(int n) { return n < 3 ? 0 : n * (n - 1) * (n - 2) / 6; }

void decode_triple(int t, int n, int &i, int &j, int &k) {
    i = 0;
    while (i < n - 3 && t >= (n - 1 - i) * (n - 2 - i) / 2) t -= (n - 1 - i) * (n - 2 - i) / 2, ++i;
    j = i + 1;
    while (j < n - 2 && t >= n - 1 - j) t -= n - 1 - j, ++j;
    k = j + 1 + t;
}

bool keep_candidate(const uint8_t *spi, const uint8_t *pi, int n, const uint8_t *added) {
    uint8_t index[kMaxN + 1], rindex[kMaxN + 1];
    for (int q = 0; q < n; ++q) index[pi[q]] = static_cast<uint8_t>(q);
    if (!cyclic_order3(index, added[0], added[1], added[2])) return false;
    for (int s = 0; s < n; ++s) rindex[s] = static_cast<uint8_t>((n - 1) - index[s]);
    uint64_t seen = 0;
    bool anyOriented = false;
    for (int s = 0; s < n; ++s) {
        if ((seen >> s) & 1ull) continue;
        uint8_t cyc[kMaxN + 1], cidx[kMaxN + 1] = {0};
        int len = 0, cur = s;
        do {
            seen |= 1ull << cur;
            cidx[cur] = static_cast<uint8_t>(len);
            cyc[len++] = static_cast<uint8_t>(cur);
            cur = spi[cur];
        } while (cur != s);
        if (cyclic_order(rindex, cyc, len)) continue;  // not oriented
        anyOriented = true;
        if (has_2_move(index, cyc, cidx, len)) return false;
    }
    return anyOriented;
}

}  // namespace

extern "C" int oracle_extension_count(int n) { return 2 * comb3(n) + 2 * comb3(n + 3); }

extern "C" int64_t oracle_extension_filter(const uint8_t *spi, const uint8_t *pi, int n, uint8_t *keep) {
    if (n < 3 || n + 3 > kMaxN) return -1;
    int64_t hits = 0;
    int e = 0;
    uint8_t s2[kMaxN + 1], p2[kMaxN + 1], added[3];
    for (int t = 0; t < comb3(n); ++t)
        for (int o = 0; o < 2; ++o, ++e) {
            int a, b, c;
            decode_triple(t, n, a, b, c);
            const int r1 = o == 0 ? b : c, r2 = o == 0 ? c : b;  // rho = (a r1 r2)
            int rho[kMaxN + 1];
            for (int x = 0; x < n; ++x) rho[x] = x;
            rho[a] = r1;
            rho[r1] = r2;
            rho[r2] = a;
            for (int x = 0; x < n; ++x) s2[x] = spi[rho[x]];
            added[0] = a, added[1] = r1, added[2] = r2;
            keep[e] = keep_candidate(s2, pi, n, added) ? 1 : 0;
            hits += keep[e];
        }
    const int m = n + 3;
    for (int t = 0; t < comb3(n + 3); ++t)
        for (int o = 0; o < 2; ++o, ++e) {
            int i, j, k;
            decode_triple(t, n + 3, i, j, k);
            const int g[3] = {i, j - 1, k - 2};
            int q = 0, w = 0;
            for (int pos = 0; pos <= n; ++pos) {
                while (w < 3 && g[w] == pos) p2[q++] = static_cast<uint8_t>(n + w), ++w;
                if (pos < n) p2[q++] = pi[pos];
            }
            for (int x = 0; x < n; ++x) s2[x] = spi[x];
            const int x = n, y = n + 1, z = n + 2;
            if (o == 0) s2[x] = y, s2[y] = z, s2[z] = x, added[0] = x, added[1] = y, added[2] = z;
            else s2[x] = z, s2[z] = y, s2[y] = x, added[0] = x, added[1] = z, added[2] = y;
            keep[e] = keep_candidate(s2, p2, m, added) ? 1 : 0;
            hits += keep[e];
        }
    return hits;
}

// ---- configuration signatures and canonical form: Configuration.java -----------------
//
// A configuration is spi over symbols 0..n-1 (every symbol in a cycle of length >= 2, as
// the reference requires: Configuration.signature dereferences each symbol's cycle) with pi
// the n-cycle (0 1 ... n-1) (CANONICAL_PI, CommonOperations.java:26-33).  spi is given as
// its successor array: spi[x] is the symbol after x in x's cycle.

namespace {

// Configuration.signature (Configuration.java:56-104) for spi (successor array) and the pi
// cycle written as the array pic[0..n-1].  Labels number the cycles by first appearance
// along pi; a cycle is oriented when its symbols are not in cyclic order in pi^-1
// (CommonOperations.java:167-182 on the reversed pi); an oriented cycle's symbols are
// numbered 1.. along the cycle from the one at the smallest pi position; the value is
// label + index / 100 in float arithmetic.
void signature_of(const int *spi, const int *pic, int n, float *out) {
    int pos[kMaxN + 2], label[kMaxN + 2], orient[kMaxN + 2], cyc[kMaxN + 2];
    for (int i = 0; i < n; ++i) pos[pic[i]] = i;
    // cycle id = smallest symbol of the cycle
    for (int x = 0; x < n; ++x) {
        int m = x;
        for (int y = spi[x]; y != x; y = spi[y]) m = std::min(m, y);
        cyc[x] = m;
    }
    for (int x = 0; x < n; ++x) label[x] = 0, orient[x] = -1;
    int next = 1;
    for (int i = 0; i < n; ++i) {
        const int s = pic[i], c = cyc[s];
        if (orient[c] < 0) {
            // cyclic order in pi^-1: index in the reversed pi array is n-1-pos
            int leaps = 0;
            int y = c;
            do {
                const int z = spi[y];
                if ((n - 1 - pos[y]) > (n - 1 - pos[z])) ++leaps;
                y = z;
            } while (y != c);
            orient[c] = leaps > 1 ? 1 : 0;
        }
        if (label[c] == 0) label[c] = next++;
        float v = (float)label[c];
        if (orient[c]) {
            // anchor: the cycle's symbol with the smallest pi position
            int anchor = c;
            int y = c;
            do {
                if (pos[y] < pos[anchor]) anchor = y;
                y = spi[y];
            } while (y != c);
            int idx = 1;
            for (int z = anchor; z != s; z = spi[z]) ++idx;
            v = (float)label[c] + (float)idx / 100.0f;
        }
        out[i] = v;
    }
}

// java.util.zip.CRC32 over the big-endian bytes of each float (Signature.hashCode,
// Configuration.java:290-303), as a signed int.
int32_t signature_hash(const float *sig, int n) {
    uint32_t crc = 0xFFFFFFFFu;
    for (int i = 0; i < n; ++i) {
        uint32_t bits;
        std::memcpy(&bits, &sig[i], 4);
        for (int b = 3; b >= 0; --b) {
            crc ^= (bits >> (8 * b)) & 0xFFu;
            for (int k = 0; k < 8; ++k) crc = (crc >> 1) ^ (0xEDB88320u & (0u - (crc & 1u)));
        }
    }
    return (int32_t)(crc ^ 0xFFFFFFFFu);
}

// Arrays.compare on float[] (Float.compare per element; equal lengths here).
int compare_signatures(const float *a, const float *b, int n) {
    for (int i = 0; i < n; ++i) {
        if (a[i] < b[i]) return -1;
        if (a[i] > b[i]) return 1;
    }
    return 0;
}

// Variant v of getEquivalentSignatures (Configuration.java:180-186): v = 2r is pi started
// at symbol r, v = 2r+1 its mirror (Configuration.java:188-195): spi conjugated by the
// involution swapping the symbols at pi positions i and n-1-i, then inverted.
void equivalent_signature(const int *spi, int n, int v, float *out) {
    const int r = v >> 1;
    int pic[kMaxN + 2];
    for (int i = 0; i < n; ++i) pic[i] = (r + i) % n;
    if ((v & 1) == 0) {
        signature_of(spi, pic, n, out);
        return;
    }
    int pos[kMaxN + 2], conj[kMaxN + 2], inv[kMaxN + 2], m[kMaxN + 2];
    for (int i = 0; i < n; ++i) pos[pic[i]] = i;
    for (int x = 0; x < n; ++x) conj[x] = pic[n - 1 - pos[x]];
    for (int x = 0; x < n; ++x) inv[spi[x]] = x;
    for (int x = 0; x < n; ++x) m[x] = conj[inv[conj[x]]];  // (c spi c)^-1
    signature_of(m, pic, n, out);
}

}  // namespace

extern "C" {

// Signature of spi (successor array) under CANONICAL_PI.  Returns 0, or -1 on bad input.
int oracle_signature(const uint8_t *spi, int n, float *out) {
    if (n < 2 || n > kMaxN) return -1;
    int s[kMaxN + 2], pic[kMaxN + 2];
    for (int i = 0; i < n; ++i) s[i] = spi[i], pic[i] = i;
    signature_of(s, pic, n, out);
    return 0;
}

// All 2n equivalent signatures, variant v at out + v*n.
int oracle_equivalent_signatures(const uint8_t *spi, int n, float *out) {
    if (n < 2 || n > kMaxN) return -1;
    int s[kMaxN + 2];
    for (int i = 0; i < n; ++i) s[i] = spi[i];
    for (int v = 0; v < 2 * n; ++v) equivalent_signature(s, n, v, out + (size_t)v * n);
    return 0;
}

int32_t oracle_signature_hash(const float *sig, int n) { return signature_hash(sig, n); }

// Configuration.getCanonical / hashCode (Configuration.java:147-174, 241-245): the
// equivalent signature with the least hash (signed), ties broken by Arrays.compare.
// Writes it to outSig, its hash to *outHash and its variant index to *outVariant.
int oracle_canonical(const uint8_t *spi, int n, float *outSig, int32_t *outHash, int32_t *outVariant) {
    if (n < 2 || n > kMaxN) return -1;
    int s[kMaxN + 2];
    for (int i = 0; i < n; ++i) s[i] = spi[i];
    float cur[kMaxN + 2];
    int32_t best = INT32_MAX;
    int bestV = -1;
    for (int v = 0; v < 2 * n; ++v) {
        equivalent_signature(s, n, v, cur);
        const int32_t h = signature_hash(cur, n);
        if (bestV < 0 || h < best || (h == best && compare_signatures(cur, outSig, n) < 0)) {
            best = h;
            bestV = v;
            std::memcpy(outSig, cur, sizeof(float) * (size_t)n);
        }
    }
    *outHash = best;
    *outVariant = bestV;
    return 0;
}

}  // extern "C"
