"""Seeded synthetic search instances.

Every instance is a configuration of the transposition-distance proof: a pair
(pi, spi) of byte arrays over n symbols together with the number of odd-length
cycles of spi (the reference calls those "even" cycles, SortingSearch.java:120-122).

* ``three_permutation(m, rng)``: spi is a product of m disjoint 3-cycles drawn
  uniformly over n = 3m symbols, pi is the identity array
  (MulticyclePermutation.java:15-28, CANONICAL_PI_BYTE), initial even cycles = m.
* ``random_permutation(n_prime, rng)``: pi = 0 followed by a shuffle of 1..n',
  spi = sigma o pi^-1 with sigma the canonical (n'+1)-cycle, as in
  GenerateLongerPermutations.java:23-36 and LongerPermutations.java:42-43.

Seeds are ``1375 + config * 10**6 + case`` with numpy's PCG64.
"""
from __future__ import annotations

import numpy as np

MIN_RATE = np.float32(2) / np.float32(1.375)  # SortOrExtend.java:43 (float arithmetic)
MAX_DEPTH = 11


def seed_for(config: int, case: int) -> int:
    return 1375 + config * 10**6 + case


def count_even_cycles(spi: np.ndarray) -> int:
    n = len(spi)
    seen = np.zeros(n, dtype=bool)
    count = 0
    for s in range(n):
        if seen[s]:
            continue
        size = 0
        cur = s
        while not seen[cur]:
            seen[cur] = True
            size += 1
            cur = int(spi[cur])
        count += size & 1
    return count


def three_permutation(m: int, rng: np.random.Generator):
    n = 3 * m
    q = rng.permutation(n)
    spi = np.arange(n, dtype=np.uint8)
    for t in range(m):
        a, b, c = int(q[3 * t]), int(q[3 * t + 1]), int(q[3 * t + 2])
        spi[a], spi[b], spi[c] = b, c, a
    pi = np.arange(n, dtype=np.uint8)
    return pi, spi, m


def random_permutation(n_prime: int, rng: np.random.Generator):
    n = n_prime + 1
    pi = np.concatenate([[0], rng.permutation(np.arange(1, n))]).astype(np.uint8)
    # sigma = (0 1 ... n-1); spi = sigma o pi^-1 where pi is the cycle written by the array.
    pi_next = np.empty(n, dtype=np.int64)
    pi_next[pi] = np.roll(pi, -1)  # pi(x): successor of x in the cycle
    pi_inv = np.empty(n, dtype=np.int64)
    pi_inv[pi_next] = np.arange(n)
    sigma = (np.arange(n) + 1) % n
    spi = sigma[pi_inv].astype(np.uint8)
    return pi, spi, count_even_cycles(spi)


def config_cases(config: int, count: int, start: int = 0):
    """Yields (pi, spi, initial_even, m) for the seeded benchmark configurations.

    config 1: m ~ U{4,5,6}; config 2: m ~ U{4..8}; config 4: m truncated geometric on
    3..10 (p=0.35) mixed with 10% random permutations of n'=20..30; config 5 (held-out
    evaluation set): m ~ U{8,9,10}.
    """
    geo = np.array([0.35 * 0.65**k for k in range(8)])
    geo /= geo.sum()
    for case in range(start, start + count):
        rng = np.random.Generator(np.random.PCG64(seed_for(config, case)))
        if config == 1:
            m = int(rng.integers(4, 7))
        elif config == 2:
            m = int(rng.integers(4, 9))
        elif config == 4:
            if rng.random() < 0.10:
                pi, spi, even = random_permutation(int(rng.integers(20, 31)), rng)
                yield pi, spi, even, 0
                continue
            m = 3 + int(rng.choice(8, p=geo))
        elif config == 5:
            m = int(rng.integers(8, 11))
        else:
            raise ValueError(f"no generator for config {config}")
        pi, spi, even = three_permutation(m, rng)
        yield pi, spi, even, m


def extension_bases(count: int, start: int = 0, m: int = 6):
    """Base configurations of the extension enumeration: (pi, spi) rows of 64 bytes.

    Each base is a product of m disjoint 3-cycles drawn uniformly over n = 3m symbols with pi
    the identity array (seed ``seed_for(3, case)``).  Returns two (count, 64) uint8 arrays
    and n.
    """
    n = 3 * m
    spi = np.zeros((count, 64), np.uint8)
    pi = np.zeros((count, 64), np.uint8)
    for r, case in enumerate(range(start, start + count)):
        rng = np.random.Generator(np.random.PCG64(seed_for(3, case)))
        p, s, _ = three_permutation(m, rng)
        spi[r, :n] = s
        pi[r, :n] = p
    return pi, spi, n
