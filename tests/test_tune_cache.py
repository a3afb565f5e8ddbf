"""Autotuner bookkeeping that needs no GPU: size buckets and the cache."""
from alya_sma_b200 import tune


def test_buckets_are_powers_of_two():
    assert tune.bucket(1) == 1
    assert tune.bucket(640000) == 1 << 19
    assert tune.bucket(1998848) == 1 << 21
    assert tune.bucket(800) == tune.bucket(1200)


def test_cache_round_trip(tmp_path, monkeypatch):
    monkeypatch.setenv("ALYA_SMA_CACHE", str(tmp_path))
    assert tune.load_cache() == {}
    tune.save_cache({"fp32/cd/1024": {"block": 128, "scatter": "atomic"}})
    assert tune.load_cache()["fp32/cd/1024"]["block"] == 128
    assert tune.cache_path().startswith(str(tmp_path))
