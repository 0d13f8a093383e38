// Host-only checks of tdp1375_b200/csrc/tdp_math.cuh (compiled with g++ by
// tests/test_host_math.py):
//  1. move_delta equals a full recount of odd-length cycles for random spi/pi/moves;
//  2. the rule tables agree bit for bit with an independent evaluation of the float32
//     rule (passed in as the oracle's answers on stdin);
//  3. the tight bound never removes a state from which a success is reachable
//     (brute force over small n by exhaustive search of gains);
//  4. the child restrictions behind the pair and triple enumerations ("restrict");
//  5. the triple list and its uniform decoder, emulated lane by lane ("triples");
//  6. the incremental cycle fields after a split move ("split").
#include <cstdio>
#include <cstdlib>
#include <random>
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../tdp1375_b200/csrc/tdp_math.cuh"

using namespace tdp;

static int count_even(const int *spi, int n) {
    unsigned long long v = 0;
    int c = 0;
    for (int s = 0; s < n; ++s) {
        if ((v >> s) & 1ull) continue;
        int sz = 0, cur = s;
        do {
            v |= 1ull << cur;
            ++sz;
            cur = spi[cur];
        } while (cur != s);
        c += sz & 1;
    }
    return c;
}

int main(int argc, char **argv) {
    const char *mode = argc > 1 ? argv[1] : "delta";
    if (std::string(mode) == "delta") {
        std::mt19937 rng(1375);
        long bad = 0, total = 0;
        for (int it = 0; it < 20000; ++it) {
            const int n = 3 + (int)(rng() % 61);
            int spi[64], pi[64];
            for (int i = 0; i < n; ++i) spi[i] = pi[i] = i;
            std::shuffle(spi, spi + n, rng);
            std::shuffle(pi + 1, pi + n, rng);
            uint32_t w[64];
            for (int x = 0; x < n; ++x) {
                int leader = x, cur = spi[x], len = 1;
                while (cur != x) {
                    leader = std::min(leader, cur);
                    cur = spi[cur];
                    ++len;
                }
                int steps = 0;
                cur = x;
                while (cur != leader) {
                    cur = spi[cur];
                    ++steps;
                }
                w[x] = w_make(spi[x], pi[x], leader, steps, len);
            }
            const int e0 = count_even(spi, n);
            for (int q = 0; q < 40; ++q) {
                const int i = rng() % n, j = rng() % n, k = rng() % n;
                if (i == j || j == k || i == k) continue;
                const int a = pi[i], b = pi[j], c = pi[k];
                int child[64];
                std::copy(spi, spi + n, child);
                child[a] = spi[c];
                child[b] = spi[a];
                child[c] = spi[b];
                ++total;
                if (count_even(child, n) - e0 != move_delta(w[a], w[b], w[c])) ++bad;
            }
        }
        printf("delta total=%ld bad=%ld\n", total, bad);
        return bad == 0 ? 0 : 1;
    }
    if (std::string(mode) == "restrict") {
        // Child restrictions behind the pair and triple enumerations of the search kernel, by
        // exhaustion over every spi of n <= 8 symbols and every ordered symbol triple, then
        // over random spi for n up to 32:
        //  (a) a child with change +2 whose node has at most one even-length cycle takes all
        //      three symbols from one cycle;
        //  (b) a child with change >= 0 whose three symbols lie in three distinct cycles
        //      needs two even-length cycles among them (so with -2 useless and, either 0
        //      useless or at most one even-length cycle, useful children have two symbols
        //      in one cycle).
        long checked = 0, bad = 0;
        auto check_spi = [&](const int *spi, int n) {
            int cyc[64], len[64], nc = 0, evenLen = 0;
            for (int x = 0; x < n; ++x) cyc[x] = -1;
            for (int x = 0; x < n; ++x) {
                if (cyc[x] >= 0) continue;
                int cur = x, L = 0;
                do {
                    cyc[cur] = nc;
                    cur = spi[cur];
                    ++L;
                } while (cur != x);
                len[nc++] = L;
                evenLen += (L % 2 == 0);
            }
            const int e0 = count_even(spi, n);
            int child[64];
            for (int a = 0; a < n; ++a)
                for (int b = 0; b < n; ++b)
                    for (int c = 0; c < n; ++c) {
                        if (a == b || b == c || a == c) continue;
                        std::copy(spi, spi + n, child);
                        child[a] = spi[c];
                        child[b] = spi[a];
                        child[c] = spi[b];
                        const int d = count_even(child, n) - e0;
                        ++checked;
                        const bool one = cyc[a] == cyc[b] && cyc[b] == cyc[c];
                        const bool three = cyc[a] != cyc[b] && cyc[b] != cyc[c] && cyc[a] != cyc[c];
                        if (d == 2 && evenLen <= 1 && !one) ++bad;
                        if (d >= 0 && three) {
                            const int ev = (len[cyc[a]] % 2 == 0) + (len[cyc[b]] % 2 == 0) + (len[cyc[c]] % 2 == 0);
                            if (ev < 2 || d == 2) ++bad;
                        }
                    }
        };
        for (int n = 3; n <= 8; ++n) {
            int spi[64];
            for (int i = 0; i < n; ++i) spi[i] = i;
            do {
                check_spi(spi, n);
            } while (std::next_permutation(spi, spi + n));
        }
        std::mt19937 rng(7);
        for (int it = 0; it < 300; ++it) {
            const int n = 9 + (int)(rng() % 24);
            int spi[64];
            for (int i = 0; i < n; ++i) spi[i] = i;
            std::shuffle(spi, spi + n, rng);
            check_spi(spi, n);
        }
        printf("restrict checked=%ld bad=%ld\n", checked, bad);
        return bad == 0 ? 0 : 1;
    }
    if (std::string(mode) == "split") {
        // split_cycle_fields against a recount: for random spi, chains of up to 6 split moves
        // (a, b, c in one cycle, spi-order a -> b -> c) are applied with the incremental
        // fields; after each, every symbol's anchor must lie in its child cycle, be reached
        // in s2l steps (anchor: 0 steps), len must be the child cycle's length, and
        // move_delta on the new words must equal a recount for random moves.
        std::mt19937 rng(23);
        long bad = 0, total = 0;
        for (int it = 0; it < 4000; ++it) {
            const int n = 3 + (int)(rng() % 30);
            int spi[64];
            uint32_t w[64];
            for (int i = 0; i < n; ++i) spi[i] = i;
            std::shuffle(spi, spi + n, rng);
            for (int x = 0; x < n; ++x) {
                int leader = x, cur = spi[x], len = 1;
                while (cur != x) {
                    leader = std::min(leader, cur);
                    cur = spi[cur];
                    ++len;
                }
                int steps = 0;
                for (cur = x; cur != leader; cur = spi[cur]) ++steps;
                w[x] = w_make(spi[x], 0, leader, steps, len);
            }
            for (int chain = 0; chain < 6; ++chain) {
                int a = -1, b = -1, c = -1;
                for (int tries = 0; tries < 200 && a < 0; ++tries) {
                    const int x = rng() % n, y = rng() % n, z = rng() % n;
                    if (x == y || y == z || x == z) continue;
                    if (w_leader(w[x]) != w_leader(w[y]) || w_leader(w[y]) != w_leader(w[z])) continue;
                    if (move_delta(w[x], w[y], w[z]) != 2) continue;
                    a = x, b = y, c = z;
                }
                if (a < 0) break;
                const uint32_t wa = w[a], wb = w[b], wc = w[c];
                int child[64];
                std::copy(spi, spi + n, child);
                child[a] = spi[c];
                child[b] = spi[a];
                child[c] = spi[b];
                uint32_t nw[64];
                for (int x = 0; x < n; ++x)
                    nw[x] = (split_cycle_fields(w[x], a, b, c, wa, wb, wc) & ~63u) | (uint32_t)child[x];
                for (int x = 0; x < n; ++x) {
                    ++total;
                    int L = 1;
                    for (int cur = child[x]; cur != x; cur = child[cur]) ++L;
                    int cur = x;
                    for (uint32_t s2 = 0; s2 < w_s2l(nw[x]); ++s2) cur = child[cur];
                    const int anchor = (int)w_leader(nw[x]);
                    if (cur != anchor || (int)w_len(nw[x]) != L || w_s2l(nw[anchor]) != 0 ||
                        (int)w_leader(nw[anchor]) != anchor)
                        ++bad;
                }
                std::copy(child, child + n, spi);
                std::copy(nw, nw + n, w);
                const int e0 = count_even(spi, n);
                for (int q = 0; q < 30; ++q) {
                    const int x = rng() % n, y = rng() % n, z = rng() % n;
                    if (x == y || y == z || x == z) continue;
                    int g[64];
                    std::copy(spi, spi + n, g);
                    g[x] = spi[z];
                    g[y] = spi[x];
                    g[z] = spi[y];
                    ++total;
                    if (count_even(g, n) - e0 != move_delta(w[x], w[y], w[z])) ++bad;
                }
            }
        }
        printf("split total=%ld bad=%ld\n", total, bad);
        return bad == 0 ? 0 : 1;
    }
    if (std::string(mode) == "triples") {
        // Emulates the triple enumeration of the search kernel lane by lane: same(x) = positions
        // > x whose symbol shares the cycle of pi[x]; lane x lists (x, q, r) for its pairs of
        // same(x) at the exclusive prefix of C(|same|, 2); the uniform decoder (owner = first
        // lane whose inclusive prefix exceeds u, then the v-th pair of same(owner)) must return
        // list[u], and the list must be exactly the same-cycle position triples.
        std::mt19937 rng(11);
        long bad = 0, total = 0;
        for (int it = 0; it < 3000; ++it) {
            const int n = 3 + (int)(rng() % 30);
            int spi[64], pi[64], cyc[64];
            for (int i = 0; i < n; ++i) spi[i] = pi[i] = i;
            if (it % 2) {
                std::shuffle(spi, spi + n, rng);
            } else {  // products of short cycles, like the search's states
                int perm[64];
                for (int i = 0; i < n; ++i) perm[i] = i;
                std::shuffle(perm, perm + n, rng);
                for (int i = 0; i + 2 < n; i += 3) {
                    spi[perm[i]] = perm[i + 1];
                    spi[perm[i + 1]] = perm[i + 2];
                    spi[perm[i + 2]] = perm[i];
                }
            }
            std::shuffle(pi, pi + n, rng);
            for (int x = 0; x < n; ++x) cyc[x] = -1;
            for (int x = 0, c = 0; x < n; ++x) {
                if (cyc[x] >= 0) continue;
                int cur = x;
                do {
                    cyc[cur] = c;
                    cur = spi[cur];
                } while (cur != x);
                ++c;
            }
            uint32_t same[32], incl[32];
            uint32_t run = 0;
            for (int x = 0; x < 32; ++x) {
                same[x] = 0;
                if (x < n)
                    for (int y = x + 1; y < n; ++y)
                        if (cyc[pi[y]] == cyc[pi[x]]) same[x] |= 1u << y;
                const uint32_t k = (uint32_t)__builtin_popcount(same[x]);
                run += k * (k - 1) / 2;
                incl[x] = run;
            }
            std::vector<uint32_t> list(run);
            for (int x = 0; x < 32; ++x) {
                const uint32_t k = (uint32_t)__builtin_popcount(same[x]);
                uint32_t at = incl[x] - k * (k - 1) / 2, m1 = same[x];
                while (m1) {
                    const uint32_t q = (uint32_t)__builtin_ctz(m1);
                    m1 &= m1 - 1;
                    for (uint32_t m2 = m1; m2; m2 &= m2 - 1) list[at++] = pack_triple(x, q, __builtin_ctz(m2));
                }
            }
            std::vector<uint32_t> want;
            for (int i = 0; i < n; ++i)
                for (int j = i + 1; j < n; ++j)
                    for (int k = j + 1; k < n; ++k)
                        if (cyc[pi[i]] == cyc[pi[j]] && cyc[pi[j]] == cyc[pi[k]]) want.push_back(pack_triple(i, j, k));
            ++total;
            if (want != list) ++bad;
            for (uint32_t u = 0; u < run; ++u) {
                int p = 0;
                while (incl[p] <= u) ++p;
                const uint32_t k = (uint32_t)__builtin_popcount(same[p]);
                uint32_t v = u - (incl[p] - k * (k - 1) / 2), m1 = same[p], q = 0, r = 0;
                while (m1) {
                    q = (uint32_t)__builtin_ctz(m1);
                    m1 &= m1 - 1;
                    const uint32_t cnt = (uint32_t)__builtin_popcount(m1);
                    if (v < cnt) {
                        uint32_t m2 = m1;
                        for (uint32_t t = v; t > 0; --t) m2 &= m2 - 1;
                        r = (uint32_t)__builtin_ctz(m2);
                        break;
                    }
                    v -= cnt;
                }
                ++total;
                if (pack_triple(p, q, r) != list[u]) ++bad;
            }
        }
        printf("triples total=%ld bad=%ld\n", total, bad);
        return bad == 0 ? 0 : 1;
    }
    if (std::string(mode) == "rules") {
        // stdin: lines "n init D full minRateBits" ; prints sat/expand words (reference rule only)
        int n, init, D, full;
        unsigned bits;
        while (scanf("%d %d %d %d %u", &n, &init, &D, &full, &bits) == 5) {
            float r;
            std::memcpy(&r, &bits, 4);
            RuleParams p{n, init, D, r, full};
            const RuleTable t = build_rule_table(p, false);
            for (int d = 0; d <= kMaxDepth; ++d) printf("%llu %llu ", (unsigned long long)t.sat[d], (unsigned long long)t.expand[d]);
            printf("\n");
        }
        return 0;
    }
    if (std::string(mode) == "tight") {
        // For every (n, init, D, mode, even, depth) with small n: if some sequence of per-move
        // changes in {-2,0,+2} (capped to [0,n]) reaches a success through nodes the reference
        // rule expands, the tight bound must keep the node.
        const float r = 2.0f / 1.375f;
        long checked = 0, bad = 0;
        for (int n = 3; n <= 24; ++n)
            for (int init = 0; init <= n; ++init)
                for (int D = 1; D <= 15; ++D)
                    for (int full = 0; full <= 1; ++full) {
                        RuleParams p{n, init, D, r, full};
                        // reach[d][e]: success reachable from (d,e) along reference-expandable nodes
                        bool reach[17][65] = {};
                        for (int d = D; d >= 0; --d)
                            for (int e = 0; e <= n; ++e) {
                                bool ok = false;
                                if (d < D)
                                    for (int de = -2; de <= 2; de += 2) {
                                        const int e2 = e + de;
                                        if (e2 < 0 || e2 > n) continue;
                                        if (rule_satisfies(p, e2, d + 1)) ok = true;
                                        else if (d + 1 < D && rule_can_still_reach(p, e2, d + 1) && reach[d + 1][e2]) ok = true;
                                    }
                                reach[d][e] = ok;
                            }
                        for (int d = 0; d < D; ++d)
                            for (int e = 0; e <= n; ++e) {
                                ++checked;
                                if (reach[d][e] && !rule_success_reachable(p, e, d)) ++bad;
                            }
                    }
        printf("tight checked=%ld bad=%ld\n", checked, bad);
        return bad == 0 ? 0 : 1;
    }
    return 2;
}
