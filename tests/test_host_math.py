"""CPU checks of the kernel arithmetic shared with the host (tdp_math.cuh)."""
import os
import struct
import subprocess

import numpy as np
import pytest

from conftest import ROOT

SRC = os.path.join(ROOT, "tests", "host", "math_check.cpp")


@pytest.fixture(scope="module")
def math_check(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("host") / "math_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-o", exe, SRC], check=True)
    return exe


def test_move_delta_matches_recount(math_check):
    out = subprocess.run([math_check, "delta"], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr


def test_enumeration_restrictions_hold(math_check):
    """Same-cycle pairs (no -2 child useful) and same-cycle triples (only +2 useful, at most
    one even-length cycle) cover every useful child."""
    out = subprocess.run([math_check, "restrict"], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr


def test_triple_list_and_decoder(math_check):
    out = subprocess.run([math_check, "triples"], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr


def test_split_cycle_fields_match_recount(math_check):
    out = subprocess.run([math_check, "split"], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr


def test_tight_bound_is_sound(math_check):
    out = subprocess.run([math_check, "tight"], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr


def test_rule_tables_match_oracle(math_check, oracle):
    """The bit tables the kernel reads equal the oracle's float32 rule, both modes."""
    rate = float(np.float32(2) / np.float32(1.375))
    bits = struct.unpack("<I", struct.pack("<f", rate))[0]
    params = [(n, init, D, full) for n in (3, 9, 12, 18, 24, 33, 63) for init in (0, n // 3, n // 2)
              for D in (1, 4, 8, 11, 15) for full in (0, 1)]
    text = "".join(f"{n} {i} {D} {f} {bits}\n" for n, i, D, f in params)
    out = subprocess.run([math_check, "rules"], input=text, capture_output=True, text=True, check=True)
    for (n, init, D, full), line in zip(params, out.stdout.strip().splitlines()):
        words = [int(v) for v in line.split()]
        for d in range(16):
            sat, expand = words[2 * d], words[2 * d + 1]
            for e in range(min(n, 63) + 1):
                ev = oracle.rule_eval(n, init, rate, D, full, e, d)
                want_sat = bool(ev & 1) and d <= D
                want_exp = bool(ev & 2) and d < D
                assert bool((sat >> e) & 1) == want_sat, (n, init, D, full, e, d)
                assert bool((expand >> e) & 1) == want_exp, (n, init, D, full, e, d)


def test_ceil_hazard_between_java_and_cuda_rules():
    """Java prunes with double ceil (SortingSearch.java:63), CUDA with float ceilf
    (sorting_search.cu:347): they differ exactly at k = 11 for r = 2/1.375."""
    r = np.float32(2) / np.float32(1.375)
    diff = [k for k in range(1, 16) if np.ceil(float(r) * k) != np.ceil(np.float32(r) * np.float32(k))]
    assert diff == [11]
