"""Generates tests/golden/cases.npz: small seeded analysis cases with the FP64
oracle's outputs (oracle/letkf_oracle.py), cross-checked against the C
restatement (oracle/letkf_ref.c) before saving.

    python tests/golden/make_golden.py

Cases (all on a 10 x 8 x 3 grid at 0.25 deg, k = 6 unless noted):
  letkf       LETKF, rho = 1.1, RTPP = RTPS = 0
  letkf_rtp   LETKF, rho = 1.05, RTPP = 0.9, RTPS = 0.5 (RTPS overrides RTPP)
  letkf_k7    LETKF with an odd ensemble size (k = 7)
  lpf_sr      LPF, systematic resampling with the reference's offsets, DP,
              nmonte = 6, uniforms from MT19937 streams seeded per (point, draw)
  lpfgm_mr    LPFGM, multinomial resampling, DP, nmonte = 3
"""
from __future__ import annotations

import dataclasses
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import cref, letkf_oracle as O, mt19937 as mt  # noqa: E402
from sbpom_letkf_v2_b200.params import DA_LETKF, DA_LPF, DA_LPFGM, RM_MR, RM_SR  # noqa: E402
from sbpom_letkf_v2_b200.synthetic import WORKLOADS, make_case  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cases.npz")

BASE = WORKLOADS[0].scaled(nlon=10, nlat=8, nlev=3, nmem=6, n_sst=60, n_ssh=20, n_prof=2, seed=2024)

CASES = {
    "letkf": dict(wl={}, params=dict(cov_infl_mul=1.1)),
    "letkf_rtp": dict(wl={}, params=dict(cov_infl_mul=1.05, alpha_rtpp=0.9, alpha_rtps=0.5)),
    "letkf_k7": dict(wl=dict(nmem=7, seed=2025), params=dict(cov_infl_mul=1.1)),
    "lpf_sr": dict(wl=dict(seed=2026, nmem=8), params=dict(iswitch_da=DA_LPF, rm=RM_SR, nmonte=6)),
    "lpfgm_mr": dict(wl=dict(seed=2027), params=dict(iswitch_da=DA_LPFGM, rm=RM_MR, nmonte=3, cov_infl_gm=1.2)),
}


def mt_uniforms(P, nmonte, nmem, rm):
    """Uniforms of each (point, draw): com_rand_seed(nmem, seed) with the
    fixed seed map of oracle.mt19937.pf_seed (SR keeps the first value)."""
    pts = np.repeat(np.arange(P), nmonte)
    drw = np.tile(np.arange(nmonte), P)
    u = mt.com_rand_seed(nmem, mt.pf_seed(pts, drw))
    if rm == RM_SR:
        return u[:, 0].reshape(P, nmonte).copy()
    return u.reshape(P, nmonte, nmem).copy()


def build():
    out = {}
    for name, spec in CASES.items():
        wl = BASE.scaled(**spec["wl"])
        case = make_case(wl, **spec["params"])
        p = case.params
        g = {k: v.numpy() for k, v in case.grid.items()}
        ob = {k: v.numpy() for k, v in case.obs.items()}
        f3, f2 = case.fcst3d.numpy(), case.fcst2d.numpy()
        P = p.nlev * case.nij1
        uni = None
        if p.iswitch_da != DA_LETKF:
            uni = mt_uniforms(P, p.nmonte, p.nmem, p.rm)
        keep = [(k, i) for k in range(p.nlev) for i in range(0, case.nij1, 13)]
        r = O.da_main(p, g, ob, f3, f2, uniforms=uni, keep=keep)
        rc = cref.da_main(p, g, ob, f3, f2, uniforms=uni, rsize=8, want_src=True)
        d3 = np.abs(rc["anal3d"] - r.anal3d).max()
        assert d3 < 1e-12 * np.abs(r.anal3d).max(), (name, d3)
        assert np.array_equal(rc["nobsl"], r.nobsl), name
        pre = f"{name}__"
        for k, v in g.items():
            out[pre + "grid_" + k] = v
        for k, v in ob.items():
            out[pre + "obs_" + k] = v
        out[pre + "fcst3d"] = f3
        out[pre + "fcst2d"] = f2
        out[pre + "anal3d"] = r.anal3d
        out[pre + "anal2d"] = r.anal2d
        out[pre + "nobsl"] = r.nobsl
        out[pre + "params"] = np.array([json.dumps(dataclasses.asdict(p))])
        if uni is not None:
            out[pre + "uniforms"] = uni
            src = np.stack([np.stack([r.src[(k, i)] for (k, i) in keep if (k, i) in r.src])]) if r.src else None
            out[pre + "src_points"] = np.array([k * case.nij1 + i for (k, i) in keep if (k, i) in r.src], np.int64)
            if src is not None:
                out[pre + "src"] = src[0].astype(np.int16)
        kp = [(k, i) for (k, i) in keep if (k, i) in r.wmat]
        out[pre + "w_points"] = np.array([k * case.nij1 + i for (k, i) in kp], np.int64)
        out[pre + "wmat"] = np.stack([r.wmat[q] for q in kp])
        out[pre + "wvec"] = np.stack([r.wvec[q] for q in kp])
        print(f"{name}: P={P} nobs={ob['elm'].size} nobsl max={r.nobsl.max()} |C-numpy|={d3:.2e}")
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    build()
