// Host-only checks of tdp1375_b200/csrc/tdp_math.cuh (compiled with g++ by
// tests/test_host_math.py):
//  1. move_delta equals a full recount of odd-length cycles for random spi/pi/moves;
//  2. the rule tables agree bit for bit with an independent evaluation of the float32
//     rule (passed in as the oracle's answers on stdin);
//  3. the tight bound never removes a state from which a success is reachable
//     (brute force over small n by exhaustive search of gains).
#include <cstdio>
#include <cstdlib>
#include <random>
#include <algorithm>
#include <cstring>
#include <string>

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
