"""CPU checks of the autotuner's candidate grid and cache lookup (no GPU needed)."""
import json


def test_candidates_cover_the_grid():
    from tdp1375_b200 import autotune
    space = {"blocks_per_sm": [0, 2], "poll_interval": [8, 16, 32], "sparse_enumeration": [1, 0]}
    cands = list(autotune.candidates(space))
    assert len(cands) == 12
    assert len({tuple(sorted(c.items())) for c in cands}) == 12
    assert all(set(c) == set(space) for c in cands)


def test_cached_choice_is_read_back(tmp_path, monkeypatch):
    from tdp1375_b200 import autotune
    monkeypatch.setattr(autotune, "_device_name", lambda: "B200")
    path = tmp_path / "cache.json"
    choice = {"blocks_per_sm": 2, "poll_interval": 16, "sparse_enumeration": 1, "table_entries": 1 << 25,
              "kernel_ms": 12.5}
    path.write_text(json.dumps({"w@B200": {"choice": choice, "tried": [choice], "when": 0}}))
    assert autotune.cached("w", cache_path=str(path)) == choice
    assert autotune.cached("other", cache_path=str(path)) is None
