"""Case files ("spi->[moves]", AbstractSbtAlgorithm.java:166-179): the writer reproduces the
reference's own case lines byte for byte, parsing inverts it, and applying a recorded
sorting agrees with the oracle's replay."""
import json
import os

import pytest

from conftest import ROOT
from tdp1375_b200 import casefile

FIXTURES = ["cases_3_2.json", "cases_comb.json"]


def records(name):
    return json.load(open(os.path.join(ROOT, "tests", "golden", name)))["records"]


@pytest.mark.parametrize("name", FIXTURES)
def test_writer_reproduces_reference_lines(name):
    for rec in records(name):
        assert casefile.format_line(rec["spi"], rec["moves"]) == rec["line"]
        spi, moves = casefile.parse_line(rec["line"])
        assert spi == rec["spi"] and [list(m) for m in moves] == rec["moves"]


def test_recorded_sortings_reach_the_ratio(oracle):
    """The sortings reach 1.375 (a partial sorting, SortOrExtend's criterion), and applying
    them with casefile.apply_moves gives the oracle's replay."""
    import numpy as np
    rate = np.float32(2) / np.float32(1.375)
    for rec in records("cases_comb.json"):
        out = casefile.apply_moves(rec["spi"], rec["moves"])
        even, final = oracle.replay_symbols(rec["pi"], rec["spi"], rec["moves"])
        assert out == list(final)
        init = oracle.count_even(rec["spi"])
        assert np.float32(even - init) / np.float32(len(rec["moves"])) >= rate


def test_file_round_trip(tmp_path):
    recs = [(r["spi"], [tuple(m) for m in r["moves"]]) for r in records("cases_3_2.json")]
    path = str(tmp_path / "cases.txt")
    casefile.write_case_file(path, recs)
    assert casefile.read_case_file(path) == recs
    assert open(path).read().splitlines() == [r["line"] for r in records("cases_3_2.json")]


def test_bad_lines_are_rejected():
    with pytest.raises(ValueError):
        casefile.parse_line("(0 1 2)(3 4)->[(0 1)]")
    with pytest.raises(ValueError):
        casefile.parse_line("(0 1 2)(4 5 6)->[(0 1 2)]")
