"""Helpers shared by the tests (inputs, comparisons)."""
from __future__ import annotations

import json
import os

import numpy as np

from sbpom_letkf_v2_b200.params import LETKFParams

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cases.npz")
GOLDEN_CASES = ("letkf", "letkf_rtp", "letkf_k7", "lpf_sr", "lpfgm_mr")


def load_golden(name: str) -> dict:
    z = np.load(GOLDEN)
    pre = name + "__"
    d = {k[len(pre):]: z[k] for k in z.files if k.startswith(pre)}
    d["params"] = LETKFParams(**json.loads(str(d["params"][0])))
    d["grid"] = {k[5:]: v for k, v in d.items() if k.startswith("grid_")}
    d["obs"] = {k[4:]: v for k, v in d.items() if k.startswith("obs_")}
    return d


def field_relerr(a, b) -> float:
    """max |a-b| / max |b| over each variable field, maximised over fields."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    worst = 0.0
    for v in range(b.shape[0]):
        den = np.abs(b[v]).max()
        num = np.abs(a[v] - b[v]).max()
        worst = max(worst, num / den if den > 0 else num)
    return worst


def incr_relerr(a, b, f) -> float:
    """Error of the analysis increment relative to the largest increment."""
    a = np.asarray(a, np.float64) - np.asarray(f, np.float64)
    b = np.asarray(b, np.float64) - np.asarray(f, np.float64)
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / den) if den > 0 else float(np.abs(a - b).max())
