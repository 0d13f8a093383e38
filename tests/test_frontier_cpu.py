"""Host logic of the batched frontier: the canonical configuration rebuilt from a variant
has that variant's signature (Configuration.ofSignature), and the staged depths follow
SortOrExtend.searchForSorting."""
import random

import numpy as np

from tdp1375_b200 import frontier


def random_configuration(rng, n):
    q = list(range(n))
    rng.shuffle(q)
    p = list(range(n))
    i = 0
    while i < n:
        L = rng.randint(2, 7)
        if n - i - L == 1 or i + L > n:
            L = n - i
        cyc = q[i:i + L]
        for k, x in enumerate(cyc):
            p[x] = cyc[(k + 1) % len(cyc)]
        i += L
    return p


def test_canonical_spi_has_the_variant_signature(oracle):
    rng = random.Random(3)
    for _ in range(200):
        spi = random_configuration(rng, rng.randint(2, 40))
        eq = oracle.equivalent_signatures(spi)
        for v in range(len(eq)):
            c = frontier.canonical_spi(spi, v)
            assert sorted(c) == list(range(len(spi)))
            assert np.array_equal(np.float32(oracle.signature(c)), np.float32(eq[v]))


def test_canonical_form_round_trips_through_the_oracle(oracle):
    rng = random.Random(4)
    for _ in range(100):
        spi = random_configuration(rng, rng.randint(2, 40))
        sig, h, v = oracle.canonical(spi)
        c = frontier.canonical_spi(spi, v)
        assert np.array_equal(np.float32(oracle.signature(c)), np.float32(sig))
        assert oracle.canonical(c)[1] == h  # the canonical configuration is its own canonical form


def test_stages_and_upper_bound():
    f = frontier.Frontier(max_ratio=1.375, max_depth=11)
    # (0 1 2)(3 4 5)(6 7 8): three odd cycles of 9 symbols -> 3-norm 3 -> floor(3 * 1.375) = 4
    spi = [1, 2, 0, 4, 5, 3, 7, 8, 6]
    assert frontier.upper_bound(spi, f.min_rate) == 4
    assert f._stages(4) == [4]
    assert f._stages(6) == [4, 6]
    assert f._stages(8) == [4, 8]
    assert f._stages(9) == [4, 8, 9]
    assert f._stages(20) == [4, 8, 11]
