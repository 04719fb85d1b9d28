"""Autotuner for the fused 2D kernels: tile shape, predictor staging and the
persistent kernels.

Every variant the library was built with (bonzo_b200._lib.variants(): tile
tx x ty, shared-memory staging of the predictor's input or not, persistent
work-queue corrector and predictor or not) is timed on
the batch's own state for a few steps (the state is restored after each
trial) and the fastest is kept.  Choices are cached in a JSON file keyed by
the workload shape, so later runs of a similar sweep skip the trials:

    key = "2d|<rsolver>|<limiter>|inst=<log2 bucket>|meanN=<log2 bucket>"

The cache lives at $BNZ_TUNE_CACHE, else ~/.cache/bonzo_b200/fused_tune.json.
"""
import json
import math
import os

from . import _lib

RS_NAME = {v: k for k, v in _lib.RS.items()}
LIM_NAME = {v: k for k, v in _lib.LIM.items()}


def cache_path():
    return os.environ.get("BNZ_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "bonzo_b200", "fused_tune.json"))


def workload_key(sizes, rsolver, limiter):
    mean_n = sum(sizes) / len(sizes)
    return "2d|%s|%s|inst=%d|meanN=%d" % (rsolver, limiter, round(math.log2(len(sizes))),
                                         round(math.log2(mean_n)))


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except Exception:
        return {}


def _store(d):
    p = cache_path()
    try:
        os.makedirs(os.path.dirname(p), exist_ok=True)
        tmp = p + ".tmp"
        with open(tmp, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, p)
    except OSError:
        pass  # a read-only home only disables the cache


def tune_batch(batch, sizes, rsolver="hlld", limiter="vl", steps=2, use_cache=True):
    """Pick the fastest variant for `batch` (a bonzo_b200._lib.Batch of grids
    with side lengths `sizes`).  Returns (variant, {variant: ms per step})."""
    key = workload_key(sizes, rsolver, limiter)
    if use_cache:
        hit = _load().get(key)
        if hit is not None:
            batch.set_variant(hit["variant"])
            return hit["variant"], {int(k): v for k, v in hit["ms"].items()}
    vs = _lib.variants()
    timings = {}
    for v in range(len(vs)):
        try:
            timings[v] = batch.time_variant(v, steps)
        except _lib.BnzError as e:
            if e.code != _lib.BNZ_ERR_UNSUPPORTED:  # not built for this Riemann solver
                raise
    best = min(timings, key=timings.get)
    batch.set_variant(best)
    if use_cache:
        d = _load()
        d[key] = {"variant": best, "ms": timings, "variants": vs}
        _store(d)
    return best, timings
