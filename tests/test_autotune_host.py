"""Autotuner bookkeeping without a GPU: cache keys, candidate lists and the
JSON cache round trip."""
from __future__ import annotations

from diffuse_vs_gfm_mms_b200 import abi, autotune


def test_keys_bucket_by_line_length_and_count():
    a = abi.make_desc(2, (1024, 512), (1, 1), [("ideal_gas", 1.4, 0)] * 2)
    b = abi.make_desc(2, (1000, 520), (1, 1), [("ideal_gas", 1.4, 0)] * 2)
    c = abi.make_desc(2, (64, 512), (1, 1), [("ideal_gas", 1.4, 0)] * 2)
    assert autotune.key_for(a, 0) == autotune.key_for(b, 0)
    assert autotune.key_for(a, 0) != autotune.key_for(c, 0)
    assert autotune.key_for(a, 0) != autotune.key_for(a, 1)


def test_candidates_include_staged_and_fused_tiles():
    d = abi.make_desc(3, (64, 64, 64), (1, 1, 1), [("ideal_gas", 1.4, 0)] * 2)
    for direction in range(3):
        c = autotune.candidates(d, direction)
        assert c[0][0] == abi.SCHEDULE_STAGED
        assert any(x[0] == abi.SCHEDULE_FUSED for x in c)
    d.precision = abi.PRECISION_MIXED
    assert autotune.candidates(d, 0) == [(abi.SCHEDULE_STAGED, 0, 0)]


def test_cache_round_trip(tmp_path, monkeypatch):
    monkeypatch.setenv("DIMGPU_TUNE_CACHE", str(tmp_path / "tune.json"))
    autotune._memory.clear()
    autotune._store("k", {"choice": [1, 0, 0]})
    autotune._memory.clear()
    assert autotune._load()["k"]["choice"] == [1, 0, 0]
