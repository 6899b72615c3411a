"""Autotuner bookkeeping that needs no GPU: knob encoding and the cache file."""

from __future__ import annotations

from critmc_b200 import autotune


def test_msc_mode_encodes_rows_per_thread():
    for run in autotune.MSC_RUNS:
        code = autotune.msc_mode(run, 3) >> 8
        assert 1 <= code <= 6 and 1 << (code - 1) == run
        assert autotune.msc_mode(run, 3) & 0xFF == 3


def test_cache_round_trip(tmp_path, monkeypatch):
    monkeypatch.setenv("CRITMC_B200_TUNE_CACHE", str(tmp_path / "t.json"))
    assert autotune._load() == {}
    autotune._store("a|b", {"run": 4})
    autotune._store("c|d", {"run": 8})
    assert autotune._load() == {"a|b": {"run": 4}, "c|d": {"run": 8}}


def test_unwritable_cache_is_not_an_error(tmp_path, monkeypatch):
    monkeypatch.setenv("CRITMC_B200_TUNE_CACHE", str(tmp_path / "f" / "t.json"))
    (tmp_path / "f").write_text("a file where a directory should be")
    autotune._store("k", {"x": 1})
    assert autotune._load() == {}
