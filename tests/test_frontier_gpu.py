"""Batched frontier on the GPU: one canonicalisation launch and one search launch per
stage give the reference's staged verdicts (SortOrExtend.searchForSorting), once per
canonical configuration."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_frontier_staged_verdicts_match_oracle(native_lib, oracle):
    from tdp1375_b200 import GPUSortingSearch, frontier
    from tdp1375_b200.cases import three_permutation
    rng = np.random.Generator(np.random.PCG64(1375 + 9 * 10**6))
    base = []
    for _ in range(60):
        _, spi, _ = three_permutation(int(rng.integers(3, 7)), rng)
        base.append([int(x) for x in spi])
    # equivalent configurations (rotations and mirrors) must share one computation
    equivalent = [frontier.canonical_spi(s, int(rng.integers(0, 2 * len(s)))) for s in base[:20]]
    GPUSortingSearch(1, 1, 256 << 20, 1 << 22)
    try:
        f = frontier.Frontier(slot=0, max_ratio=1.375, max_depth=11)
        res = f.resolve(base + equivalent)
        for a, b in zip(res[:20], res[60:]):
            assert a is b
        rate = float(f.min_rate)
        for r in {id(x): x for x in res}.values():
            n, init = len(r.spi), frontier.odd_cycles(r.spi)
            want = False
            for depth in f._stages(frontier.upper_bound(r.spi, f.min_rate)):
                found, _, _ = oracle.search_gpu_rule(list(range(n)), r.spi, init, rate, depth, False,
                                                    dedup=True, tight=True)
                if found == 1:
                    want = True
                    break
            assert r.found == want, r.spi
            if r.found:
                even, _ = oracle.replay_symbols(list(range(n)), r.spi, [list(m) for m in r.moves])
                assert even - init > 0 and np.float32(even - init) / np.float32(len(r.moves)) >= f.min_rate
        # a second call finds everything decided
        again = f.resolve(base[:5])
        assert all(x is y for x, y in zip(again, res[:5]))
    finally:
        GPUSortingSearch.destroySlots()
