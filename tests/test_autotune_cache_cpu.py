"""The autotuner's cache file handling (no GPU needed)."""
import json

from sles import autotune


def test_cache_roundtrip(tmp_path, monkeypatch):
    monkeypatch.setenv("SLES_TUNE_CACHE", str(tmp_path / "sub" / "tune.json"))
    assert autotune._load() == {}
    autotune._save({"k": {"variants": {"0": 2}}})
    assert json.loads((tmp_path / "sub" / "tune.json").read_text()) == {"k": {"variants": {"0": 2}}}
    assert autotune._load()["k"]["variants"]["0"] == 2


def test_unreadable_cache_is_empty(tmp_path, monkeypatch):
    p = tmp_path / "tune.json"
    p.write_text("{not json")
    monkeypatch.setenv("SLES_TUNE_CACHE", str(p))
    assert autotune._load() == {}
