"""Autotuner host logic on the CPU: the fastest built variant is kept,
variants a Riemann solver was not built with are skipped, other errors
propagate, and the per-workload JSON cache short-cuts later trials.  The
batch is a stand-in that returns fixed timings (no device call)."""
import json

import pytest

from bonzo_b200 import _lib, autotune


class FakeBatch:
    def __init__(self, ms, unsupported=(), fail=None):
        self.ms, self.unsupported, self.fail = ms, set(unsupported), fail
        self.timed, self.chosen = [], None

    def time_variant(self, v, steps):
        self.timed.append(v)
        if v == self.fail:
            raise _lib.BnzError(_lib.BNZ_ERR_CUDA, "launch failed")
        if v in self.unsupported:
            raise _lib.BnzError(_lib.BNZ_ERR_UNSUPPORTED, "not built")
        return self.ms[v]

    def set_variant(self, v):
        self.chosen = v


@pytest.fixture
def cache(tmp_path, monkeypatch):
    p = tmp_path / "tune.json"
    monkeypatch.setenv("BNZ_TUNE_CACHE", str(p))
    return p


def _timings(nv):
    return {v: 10.0 - 0.5 * ((v * 7) % nv) for v in range(nv)}


def test_workload_key_buckets():
    assert autotune.workload_key([128] * 64, "hlld", "vl") == "2d|hlld|vl|inst=6|meanN=7"
    # sweeps of similar shape share a bucket
    assert (autotune.workload_key([120, 136] * 32, "hlld", "vl")
            == autotune.workload_key([128] * 64, "hlld", "vl"))
    assert autotune.workload_key([128] * 64, "hll", "mc") != autotune.workload_key([128] * 64, "hlld", "mc")


def test_fastest_variant_kept_and_cached(cache):
    nv = len(_lib.variants())
    ms = _timings(nv)
    b = FakeBatch(ms)
    best, t = autotune.tune_batch(b, [64] * 8, steps=1)
    assert best == min(ms, key=ms.get) and b.chosen == best
    assert b.timed == list(range(nv)) and t == ms
    d = json.loads(cache.read_text())
    key = autotune.workload_key([64] * 8, "hlld", "vl")
    assert d[key]["variant"] == best and len(d[key]["variants"]) == nv
    # a second sweep of the same shape reads the cache and times nothing
    b2 = FakeBatch(ms)
    best2, t2 = autotune.tune_batch(b2, [64] * 8, steps=1)
    assert best2 == best and b2.chosen == best and b2.timed == [] and t2 == ms


def test_unsupported_variants_skipped(cache):
    nv = len(_lib.variants())
    ms = _timings(nv)
    fastest = min(ms, key=ms.get)
    b = FakeBatch(ms, unsupported=[fastest])
    best, t = autotune.tune_batch(b, [64] * 8, rsolver="hll", use_cache=False)
    assert fastest not in t and best != fastest and best == min(t, key=t.get)
    assert not cache.exists()


def test_other_errors_propagate(cache):
    nv = len(_lib.variants())
    b = FakeBatch(_timings(nv), fail=1)
    with pytest.raises(_lib.BnzError) as e:
        autotune.tune_batch(b, [64] * 8)
    assert e.value.code == _lib.BNZ_ERR_CUDA
    assert b.chosen is None and not cache.exists()


def test_unreadable_cache_ignored(cache):
    cache.write_text("{not json")
    nv = len(_lib.variants())
    b = FakeBatch(_timings(nv))
    best, _ = autotune.tune_batch(b, [64] * 8)
    assert b.chosen == best and len(b.timed) == nv
    assert json.loads(cache.read_text())  # rewritten whole
