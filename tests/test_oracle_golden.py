"""Pins the CPU oracle to the reference's own fixtures and algebra tests."""
import numpy as np
import pytest

from conftest import load_golden

R1375 = float(np.float32(2) / np.float32(1.375))
R15 = float(np.float32(2) / np.float32(1.5))
FIXTURES = [("cases_comb.json", R1375), ("cases_3_2.json", R15), ("cases_7cycle.json", R15)]


def test_block_swap_algebra(oracle):
    """CommonOperationsTest.java:21-24: applying (0 4 1) to pi = (0 4 5 6 1 2 3) gives the
    identity cycle; PermutationGroupsTest.java:10-12: (0 4 1) o (0 4 5 6 1 2 3) = (0 1 ... 6)."""
    from tdp1375_b200.api import apply_transposition, positions_to_symbols
    pi = bytearray([0, 4, 5, 6, 1, 2, 3])
    apply_transposition(pi, 0, 1, 4)
    k = pi.index(0)
    assert list(pi[k:] + pi[:k]) == list(range(7))
    assert positions_to_symbols([0, 4, 5, 6, 1, 2, 3], [[0, 1, 4]]) == [[0, 4, 1]]
    # spi o (0 4 1)^-1 for spi = sigma o pi^-1 sorts the configuration
    sigma = [(x + 1) % 7 for x in range(7)]
    arr = [0, 4, 5, 6, 1, 2, 3]
    nxt = {arr[i]: arr[(i + 1) % 7] for i in range(7)}
    inv = {v: k for k, v in nxt.items()}
    spi = [sigma[inv[x]] for x in range(7)]
    even, final = oracle.replay_symbols(arr, spi, [[0, 4, 1]])
    assert final == list(range(7)) and even == 7


@pytest.mark.parametrize("name,rate", FIXTURES)
def test_fixture_sequences_replay(oracle, name, rate):
    """Every listed sequence is a valid transposition sequence reaching the ratio."""
    for rec in load_golden(name)["records"]:
        spi, pi, moves = rec["spi"], rec["pi"], rec["moves"]
        init = oracle.count_even(spi)
        even, _ = oracle.replay_symbols(pi, spi, moves)
        assert even >= 0
        assert even - init > 0 and np.float32(even - init) / np.float32(len(moves)) >= np.float32(rate)


@pytest.mark.parametrize("name,rate", FIXTURES)
def test_fixture_paths_pass_reference_prune(oracle, name, rate):
    """Every intermediate node of every listed sequence passes can_still_reach at the
    sequence's own length and at depth 11, so the reference's search must answer "found"
    for these configurations in partial mode (the known positives)."""
    for rec in load_golden(name)["records"]:
        spi, pi, moves = rec["spi"], rec["pi"], rec["moves"]
        n, init, L = len(spi), oracle.count_even(spi), len(moves)
        for D in sorted({L, max(L, 11)}):
            for d in range(1, L):
                even, _ = oracle.replay_symbols(pi, spi, moves[:d])
                assert oracle.rule_eval(n, init, rate, D, 0, even, d) & 2
            even, _ = oracle.replay_symbols(pi, spi, moves)
            assert oracle.rule_eval(n, init, rate, D, 0, even, L) & 1


@pytest.mark.parametrize("name,rate", [("cases_3_2.json", R15), ("cases_7cycle.json", R15)])
def test_oracle_search_finds_small_fixtures(oracle, name, rate):
    for rec in load_golden(name)["records"]:
        spi, pi = rec["spi"], rec["pi"]
        init = oracle.count_even(spi)
        st, pos, _ = oracle.search_gpu_rule(pi, spi, init, rate, len(rec["moves"]), False)
        assert st == 1
        ok, _ = oracle.replay_positions(pi, spi, pos, init, rate, False)
        assert ok


def test_oracle_search_finds_depth4_comb_fixtures(oracle):
    recs = [r for r in load_golden("cases_comb.json")["records"] if len(r["moves"]) == 4]
    assert len(recs) == 78
    for rec in recs[:30]:
        spi, pi = rec["spi"], rec["pi"]
        init = oracle.count_even(spi)
        st, pos, _ = oracle.search_gpu_rule(pi, spi, init, R1375, 4, False, tight=True, node_limit=200000)
        assert st == 1
        ok, _ = oracle.replay_positions(pi, spi, pos, init, R1375, False)
        assert ok


def _small_cases():
    from tdp1375_b200.cases import three_permutation
    rng = np.random.Generator(np.random.PCG64(99))
    out = []
    for m in (2, 3, 3, 4, 4):
        for _ in range(6):
            out.append(three_permutation(m, rng))
    return out


@pytest.mark.parametrize("full,depth", [(True, 5), (False, 4), (True, 6)])
def test_transposition_table_and_tight_bound_keep_verdicts(oracle, full, depth):
    """The oracle with the transposition table, and with the tight bound, answers like
    the plain exhaustive restatement (no table, no tight bound)."""
    for pi, spi, even in _small_cases():
        base = oracle.search_gpu_rule(list(pi), list(spi), even, R1375, depth, full, dedup=False)[0]
        dd = oracle.search_gpu_rule(list(pi), list(spi), even, R1375, depth, full, dedup=True)[0]
        tt = oracle.search_gpu_rule(list(pi), list(spi), even, R1375, depth, full, dedup=True, tight=True)[0]
        assert base in (0, 1) and base == dd == tt


def test_java_rule_and_cuda_rule_agree_on_small_full_sorting(oracle):
    """SortingSearch.java's double-precision rule and the CUDA float rule give the same
    verdicts away from the k = 11 hazard (here max depth 6)."""
    for pi, spi, even in _small_cases():
        g = oracle.search_gpu_rule(list(pi), list(spi), even, R1375, 6, True)[0]
        c, syms, _ = oracle.search_cpu_rule(list(pi), list(spi), even, R1375, 6, node_limit=2_000_000)
        assert c == g
        if c == 1:
            e, final = oracle.replay_symbols(list(pi), list(spi), syms)
            assert e == len(pi)


def test_pi_filter_oracle_matches_per_candidate_predicate(oracle):
    import itertools
    n = 7
    cycle, triple = [0, 3, 5, 1, 6, 2], [2, 4, 6]
    hits, rows = oracle.pi_filter(cycle, triple, n, False)
    brute = []
    for tail in itertools.permutations(range(1, n)):
        pi = [0] + list(tail)
        if oracle.pi_filter_keep(pi, cycle, triple, False):
            brute.append(bytes(pi))
    assert hits == len(brute) and rows == brute
