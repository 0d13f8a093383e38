"""The JNI bridge on a B200: GPUSortingSearch's five native methods (jni_sorter.cu:25-150)
driven through the stand-in VM of tests/jni.  searchForSortingSeq must return int[d][3]
positions that GPUSortingSearch.java:65-74 replays into a valid sorting, an empty array for
a configuration without one, and filterPiPermutations the oracle's rows as byte[k][n]."""
import numpy as np
import pytest

import jni_harness as J
from conftest import load_golden

pytestmark = pytest.mark.gpu

R1375 = float(np.float32(2) / np.float32(1.375))
R15 = float(np.float32(2) / np.float32(1.5))


def test_bridge_searches_and_filters(tmp_path, native_lib, oracle):
    from tdp1375_b200.cases import config_cases
    exe = J.build(str(tmp_path))
    pos_rec = load_golden("cases_3_2.json")["records"][0]
    v1 = {r["case"]: r for r in load_golden("verdicts_config1.json")["cases"]}
    neg_case = next(c for c, r in sorted(v1.items()) if r["full11"] == 0)
    npi, nspi, neven, _ = list(config_cases(1, neg_case + 1))[neg_case]
    cycle, triple = [0, 3, 1, 5, 2], [0, 1, 2]
    lines = [
        "init 1 1 268435456 1048576",
        J.search_line(0, R15, 3, False, oracle.count_even(pos_rec["spi"]), pos_rec["pi"], pos_rec["spi"]),
        J.search_line(0, R1375, 11, True, neven, list(npi), list(nspi)),
        J.search_line(7, R1375, 11, True, neven, list(npi), list(nspi)),
        J.filter_line(False, 7, cycle, triple),
        "cancel 0",
        "destroy",
    ]
    out = J.run(exe, lines, str(tmp_path))
    assert out[0]["exception"] is None
    found = out[1]
    assert found["exception"] is None and found["row_kind"] == "int" and len(found["rows"]) >= 1
    assert all(len(m) == 3 for m in found["rows"])
    ok, _ = oracle.replay_positions(pos_rec["pi"], pos_rec["spi"], found["rows"], oracle.count_even(pos_rec["spi"]),
                                    R15, False)
    assert ok
    assert out[2]["exception"] is None and out[2]["rows"] == []  # no sequence: an empty int[0][]
    assert out[3]["exception"] == "invalid slot"
    hits, rows = oracle.pi_filter(cycle, triple, 7, False)
    assert out[4]["exception"] is None and len(out[4]["rows"]) == hits
    assert sorted(bytes(r) for r in out[4]["rows"]) == sorted(rows)
    assert out[5]["exception"] is None and out[6]["exception"] is None
