"""The device generator of the extend step's insertions (tdp_insertion_extensions_device,
Extensions.java:95-141) against the host restatement on signatures
(tdp1375_b200.extensions: Type 1 for configurations with open gates, Type 2 otherwise), as
sets of extended configurations, and its open gates against getOpenGates' restatement."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def configurations():
    from oracle import oracle as O
    out = [O.parse_cycles(t) for t in ("(0 4 2)(1 5 3)", "(0 3 1 4 2)", "(0 10 2)(1 5 3)(4 8 6)(7 11 9)",
                                       "(0 2 1)", "(0 1 2)(3 5 4)", "(0,16,2)(1,5,3)(4,8,6)(7,11,9)(10,14,12)(13,17,15)")]
    rng = np.random.Generator(np.random.PCG64(8))
    for _ in range(24):
        m = int(rng.integers(2, 8))
        n = 3 * m
        q = rng.permutation(n)
        spi = list(range(n))
        for t in range(m):
            a, b, c = (int(v) for v in q[3 * t:3 * t + 3])
            spi[a], spi[b], spi[c] = b, c, a
        out.append(spi)
    return out


def test_insertions_match_the_host_extend_step(native_lib):
    from tdp1375_b200 import extend_gpu, extensions
    confs = configurations()
    got, gates = extend_gpu.insertion_extensions(confs)
    for spi, exts, mask in zip(confs, got, gates):
        host_gates = extensions.open_gates(spi)
        assert {a for a in range(len(spi)) if (mask >> a) & 1} == host_gates, spi
        types = {t for t, _ in exts}
        want = extensions.type1_extensions(spi) if host_gates else extensions.type2_extensions(spi)
        assert types == ({1} if host_gates else {2}), spi
        assert {tuple(e) for _, e in exts} == {tuple(e) for _, e in want}, spi
