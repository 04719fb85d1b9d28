"""Roofline denominators: the measured peaks of this pool's B200s.

MEASURED_PEAKS.json (repo root) holds a STREAM-style copy bandwidth and cuBLAS
bf16 throughput measured on the pool; without it the earlier pool
measurement (6.65 TB/s) is used and labelled as the fallback.
"""
import json
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FALLBACK_HBM_GBS = 6650.0


def hbm_peak():
    """(GB/s, source label)."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, copy)"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback (earlier pool measurement)"
