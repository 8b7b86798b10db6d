"""The frame autotuner's cache: one JSON file of tile choices keyed by the
GPU and the frame's shape class (host logic; the GPU round trip is in
test_gpu_frame_tuning_cache.py)."""
import json

from sentinel_gpu_processor_b200 import chain

T = {"deramp_rows": 32, "deramp_ctas": 2, "geo_cols": 64, "geo_ctas": 0}


def test_key_buckets_burst_sizes_and_separates_gpus_and_forms():
    a = chain.tuning_key("NVIDIA B200", (10, 0), 148, "c64", True, True, [(1500, 21000), (1510, 22000), (1490, 25000)])
    b = chain.tuning_key("NVIDIA B200", (10, 0), 148, "c64", True, True, [(1505, 21500), (1495, 22500), (1480, 24000)])
    assert a == b  # same shape class
    assert a != chain.tuning_key("NVIDIA B200", (10, 0), 132, "c64", True, True, [(1500, 21000)] * 3)
    assert a != chain.tuning_key("NVIDIA B200", (10, 0), 148, "ci16", True, True, [(1500, 21000)] * 3)
    assert a != chain.tuning_key("NVIDIA B200", (10, 0), 148, "c64", False, True, [(1500, 21000)] * 3)
    assert a != chain.tuning_key("NVIDIA B200", (10, 0), 148, "c64", True, True, [(1500, 21000)] * 4)
    assert a != chain.tuning_key("NVIDIA B200", (10, 0), 148, "c64", True, True, [(750, 11000)] * 3)


def test_store_and_load_round_trip(tmp_path, monkeypatch):
    path = tmp_path / "sub" / "tune.json"
    monkeypatch.setenv("S1B_TUNING_CACHE", str(path))
    assert chain.tuning_cache_path() == str(path)
    assert chain.load_tuning(str(path)) == {}
    chain.store_tuning(str(path), "k1", T)
    chain.store_tuning(str(path), "k2", dict(T, geo_cols=256))
    d = chain.load_tuning(str(path))
    assert d == {"k1": T, "k2": dict(T, geo_cols=256)}
    chain.store_tuning(str(path), "k1", dict(T, deramp_rows=8))  # replaced
    assert chain.load_tuning(str(path))["k1"]["deramp_rows"] == 8
    assert [p.name for p in path.parent.iterdir()] == ["tune.json"]  # no temporary left


def test_unreadable_or_malformed_cache_is_ignored(tmp_path):
    p = tmp_path / "t.json"
    p.write_text("{not json")
    assert chain.load_tuning(str(p)) == {}
    p.write_text(json.dumps({"good": T, "short": {"geo_cols": 64}, "bad": [1, 2], "str": dict(T, geo_ctas="0")}))
    assert chain.load_tuning(str(p)) == {"good": T}
    p.write_text(json.dumps([T]))
    assert chain.load_tuning(str(p)) == {}


def test_default_path_under_the_user_cache(monkeypatch, tmp_path):
    monkeypatch.delenv("S1B_TUNING_CACHE", raising=False)
    monkeypatch.setenv("XDG_CACHE_HOME", str(tmp_path))
    assert chain.tuning_cache_path() == str(tmp_path / "s1b" / "frame_tuning.json")
