"""The autotune cache file (ptk_tune_cache_lookup / ptk_tune_cache_store) on
the host: entries round-trip, are replaced by signature, survive other
entries, and a malformed file is reported and left as it was."""
from __future__ import annotations

import json

import pytest


def test_roundtrip_and_replace(ptk, tmp_path):
    path = tmp_path / "tune.json"
    sig_a = 'sm_100 NVIDIA B200 x148|bf16|frame 5616x3744|grains 2000|rmax 41|r8 0,12,"q"\\'
    sig_b = "sm_100 NVIDIA B200 x148|exact|frame 5616x3744|grains 2000"
    assert ptk.tune_cache_lookup(path, sig_a) is None  # no file yet
    ptk.tune_cache_store(path, sig_a, 1, 4, [2, 3, 4, 6], [1.46, 1.19, 1.2, 1.52])
    ptk.tune_cache_store(path, sig_b, 0, 1, [1, 2], [9.4, 18.2])
    assert ptk.tune_cache_lookup(path, sig_a) == (1, 4)
    assert ptk.tune_cache_lookup(path, sig_b) == (0, 1)
    assert ptk.tune_cache_lookup(path, sig_a + " ") is None
    data = json.loads(path.read_text())  # plain JSON a user can read
    assert data["version"] == 1
    assert data["entries"][sig_a] == {"method": 1, "choice": 4, "values": [2, 3, 4, 6],
                                      "ms": pytest.approx([1.46, 1.19, 1.2, 1.52], rel=1e-5)}
    ptk.tune_cache_store(path, sig_a, 1, 3, [3], [1.1])  # replaces the entry, keeps the other
    assert ptk.tune_cache_lookup(path, sig_a) == (1, 3)
    assert ptk.tune_cache_lookup(path, sig_b) == (0, 1)
    assert len(json.loads(path.read_text())["entries"]) == 2


def test_foreign_keys_and_layout(ptk, tmp_path):
    path = tmp_path / "tune.json"
    path.write_text('{ "note": ["x", {"y": null}], "entries": {"k": {"choice": 6, "extra": true,\n'
                    '"method": 1, "values": [], "ms": []}}, "version": 1 }\n')
    assert ptk.tune_cache_lookup(path, "k") == (1, 6)


@pytest.mark.parametrize("text", ['{"entries": {"k": {"method": 1}}}', '{"entries": [1, 2]}',
                                  '{"entries": {"k": {"method": 1, "choice": 2}}', "not json",
                                  '{"entries": {"k": {"method": 1, "choice": 2}}} trailing'])
def test_malformed_file_is_reported_and_kept(ptk, tmp_path, text):
    path = tmp_path / "tune.json"
    path.write_text(text)
    with pytest.raises(ptk.PtkError):
        ptk.tune_cache_lookup(path, "k")
    with pytest.raises(ptk.PtkError):
        ptk.tune_cache_store(path, "k", 1, 4)
    assert path.read_text() == text


def test_unwritable_location(ptk, tmp_path):
    with pytest.raises(ptk.PtkError):
        ptk.tune_cache_store(tmp_path / "missing_dir" / "tune.json", "k", 1, 4)
