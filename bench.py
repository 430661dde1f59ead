"""Benchmark of the analysis step: gridpoints/s of one LETKF cycle.

Workload (default): 400 x 300 x 40 grid, k = 100 members, 200k observations
(150k SST, 45k SSH, 500 T/S profiles x 10 levels), sigma_h = 200 km,
sigma_v = 100 m, rho = 1.1 -- seeded synthetic inputs generated in device
memory (sbpom_letkf_v2_b200.synthetic).  One step = one analysis cycle:
observation bucketing (sbletkf_prepare_obs) + the analysis of all 4.8M grid
points (sbletkf_analysis).  Inputs (7.7 GB of state) exceed L2, so no flush
is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|mixed]
    python bench.py --impl reference      # the CPU restatement on the host cores

Multi-GPU (torchrun): the grid's columns are split into contiguous ranges of
nearly equal cost (the reference's MPI decomposition, common_mpi.f90:314);
rank 0's observations are broadcast to every rank (NCCL), and each rank
analyses its own columns with no collective on the data path.  The total work
is fixed as N grows: strong scaling, time = max over ranks.
"""
from __future__ import annotations

import os

os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")

import argparse  # noqa: E402
import json  # noqa: E402
import math  # noqa: E402
import statistics  # noqa: E402
import subprocess  # noqa: E402
import threading  # noqa: E402
import time  # noqa: E402

import numpy as np  # noqa: E402
import torch  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
METRIC = "analysis gridpoints/s per LETKF cycle, mixed vs FP64 on B200 at <=1e-4 rel err"
TC_MAX_CAND_DEFAULT = 12288.0   # library default of sbletkf_params.tc_max_cand

# DRAM bytes per analysed point of the mixed-path analysis kernel (read +
# written), from ncu captures; scaled by the points of a launch.
#   column queue: workload 1 on its full horizontal grid with 2 levels
#     (bench.py --levels 2), which gets the same 8-column queue items;
#   pipelined kernel: workload 1 on its 1/8 grid (bench.py --scale 8).
DRAM_BYTES_PER_POINT_W1 = {"columns": 1073.6e6 / 240000.0, "pipeline": 258.6e6 / 74000.0}
# The same for the LPF: workload 4 on its 1/2 grid (bench.py --workload 4 --scale 2).
DRAM_BYTES_PER_POINT_W4 = 280.6e6 / 61440.0


def _peaks():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def _fp64_peak(dev) -> dict:
    """FP64 roofline denominator: cuBLAS DGEMM 8192^3 through torch.matmul,
    best of 5 (the FP64 counterpart of the bf16 GEMM peak)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return {"tflops": 2.0 * n ** 3 / (best / 1e3) / 1e12,
            "source": "measured in this run: cuBLAS DGEMM 8192^3 via torch.matmul, best of 5"}


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        load = [s for s in sm if s > 0.5 * (max(mx) if mx else 1)] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[j] for r in self.rows for j in range(4) if r[5 + j].lower() == "active"})
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ---------------------------------------------------------------------------
# algorithmic work (per point with n local obs, k members, nv variables)
# ---------------------------------------------------------------------------

def algorithmic_flops(nobsl: np.ndarray, k: int, nv3d: int, nv2d: int, nlev: int, nij1: int,
                      tensor_mask: np.ndarray | None = None) -> dict:
    """Per-launch algorithmic work of the analysis: F_gram = 2 k^2 n,
    F_eig = 9 k^3, F_W = 2k^3 + 2kn + 2k^2 (both where n > 0),
    F_upd = 2 nv k^2.  tensor_mask ([nlev][nij1] bool, optional) marks the
    points whose Gram runs on the tensor cores: F_gram splits into
    gram_tensor and gram_fp64."""
    n = nobsl.astype(np.float64).reshape(nlev, nij1)
    has = n > 0
    nv = np.full_like(n, nv3d, dtype=np.float64)
    nv[nlev - 1, :] += nv2d
    g = 2.0 * k * k * n
    f_gram = float(g.sum())
    tm = np.zeros_like(has) if tensor_mask is None else np.asarray(tensor_mask, bool).reshape(nlev, nij1)
    f_gram_tc = float(g[tm].sum())
    f_eig = float((9.0 * k ** 3) * has.sum())
    f_w = float(((2.0 * k ** 3 + 2.0 * k * n + 2.0 * k * k) * has).sum())
    f_upd = float((2.0 * nv * k * k).sum())
    return {"gram": f_gram, "gram_tensor": f_gram_tc, "gram_fp64": f_gram - f_gram_tc, "eig": f_eig, "w": f_w,
            "upd": f_upd, "total": f_gram + f_eig + f_w + f_upd}


def algorithmic_bytes(nobsl: np.ndarray, k: int, nv3d: int, nv2d: int, nlev: int, nij1: int) -> dict:
    """Per-launch algorithmic HBM bytes: PF weights B_w = 4 n (k+3) per point
    with obs (hdxf row, dep, rloc, rdiag in FP32), PF gather / ensemble update
    B_g = B_upd = 2*4 k nv per point (read forecast, write analysis, FP32)."""
    n = nobsl.astype(np.float64).reshape(nlev, nij1)
    nv = np.full_like(n, nv3d, dtype=np.float64)
    nv[nlev - 1, :] += nv2d
    b_w = float((4.0 * n * (k + 3)).sum())
    b_g = float((8.0 * k * nv).sum())
    return {"weights": b_w, "gather": b_g, "total": b_w + b_g}


def letkf_roofline(fl: dict, kern_ms: float, fp64_peak: dict, peaks: dict, peaks_src: str, traffic) -> dict:
    """Two fractions of the LETKF analysis kernel: the FP64 work (F_eig + F_W,
    plus the Gram of points accumulated in FP64) against the measured FP64
    DGEMM peak, and the tensor-core Gram (F_gram of the tensor-core points)
    against the sustained bf16 peak."""
    t = kern_ms / 1e3
    f64 = fl["eig"] + fl["w"] + fl["gram_fp64"]
    a64 = f64 / t / 1e12
    atc = fl["gram_tensor"] / t / 1e12
    ptc = peaks.get("bf16_tflops_sustained") or peaks.get("bf16_tflops")
    return {"bound": "fp64", "achieved": a64, "peak": fp64_peak["tflops"], "unit": "TFLOP/s",
            "frac": a64 / fp64_peak["tflops"], "traffic": traffic, "kernel": "k_analysis", "kernel_ms": kern_ms,
            "work": "F_eig + F_W (+ F_gram of points on the FP64 Gram)", "peak_source": fp64_peak["source"],
            "flops_per_launch": fl,
            "tensor": {"achieved": atc, "peak": ptc, "unit": "TFLOP/s", "frac": atc / ptc if ptc else None,
                       "work": "F_gram of the points whose Gram runs on tcgen05 (bf16 x3 split)",
                       "peak_source": f"{peaks_src} bf16_tflops_sustained (MEASURED_PEAKS.json)"}}


def mean_spread_error(a3, a2, r3, r2) -> dict:
    """Relative error of the analysis ensemble mean and spread of (a3, a2)
    against (r3, r2), per variable: max |x - r| / max |r| and
    rms(x - r) / rms(r); the worst variable is reported."""
    out = {"mean_max": 0.0, "mean_rms": 0.0, "spread_max": 0.0, "spread_rms": 0.0}
    for a, r in ((a3, r3), (a2, r2)):
        a, r = torch.as_tensor(a), torch.as_tensor(r)
        for v in range(a.shape[0]):
            x, y = a[v].double(), r[v].double()
            for name, fx, fy in (("mean", x.mean(0), y.mean(0)), ("spread", x.std(0), y.std(0))):
                d = fx - fy
                mx = float(d.abs().max() / fy.abs().max().clamp_min(1e-300))
                rms = float(torch.sqrt((d * d).mean() / (fy * fy).mean().clamp_min(1e-300)))
                out[name + "_max"] = max(out[name + "_max"], mx)
                out[name + "_rms"] = max(out[name + "_rms"], rms)
    return out


# ---------------------------------------------------------------------------
# column samples (host side; stratified by the search-box candidate count)
# ---------------------------------------------------------------------------

def box_candidates(params, grid: dict, obs: dict) -> np.ndarray:
    """Observations in each column's search box (common_da.f90:158-161,
    297-348): the candidate count that the selection scans, a host-side proxy
    of the column's nobsl and cost.  numpy; [nij1] int64."""
    nlon, nlat = params.nlon, params.nlat
    idx = np.asarray(obs["idx"], np.int64)
    idy = np.asarray(obs["idy"], np.int64)
    ok = (idx >= 1) & (idx <= nlon - 1) & (idy >= 1) & (idy <= nlat - 1)
    cnt = np.bincount((idy[ok] - 1) * nlon + (idx[ok] - 1), minlength=nlon * nlat).reshape(nlat, nlon)
    sat = np.zeros((nlat + 1, nlon + 1), np.int64)
    sat[1:, 1:] = cnt.cumsum(0).cumsum(1)

    def nint(x):
        return (np.sign(x) * np.floor(np.abs(x) + 0.5)).astype(np.int64)
    g = {k: np.asarray(v, np.float64) for k, v in grid.items()}
    dz = params.dist_zero
    imin = np.clip(nint(g["ri1"] - dz / g["dlon1"]), 1, nlon)
    imax = np.clip(nint(g["ri1"] + dz / g["dlon1"]), 1, nlon)
    jmin = np.clip(nint(g["rj1"] - dz / g["dlat1"]), 1, nlat)
    jmax = np.clip(nint(g["rj1"] + dz / g["dlat1"]), 1, nlat)
    tot = sat[jmax, imax] - sat[jmin - 1, imax] - sat[jmax, imin - 1] + sat[jmin - 1, imin - 1]
    return np.where((imin <= imax) & (jmin <= jmax), tot, 0)


def stratified_columns(cost: np.ndarray, frac: float, nstrata: int = 20, seed: int = 5,
                       min_cols: int = 1) -> np.ndarray:
    """A sample of about frac of the columns, stratified by `cost`: the
    columns sorted by cost are cut into nstrata equal strata and the same
    fraction is drawn at random (seeded) from each.  Sorted column indices."""
    n = cost.size
    want = max(min_cols, int(math.ceil(frac * n)))
    order = np.argsort(cost, kind="stable")
    rng = np.random.default_rng(seed)
    out = []
    for s in range(nstrata):
        lo, hi = s * n // nstrata, (s + 1) * n // nstrata
        if hi <= lo:
            continue
        take = int(round(want * (hi - lo) / n))
        take = min(max(take, 1), hi - lo)
        out.append(rng.choice(order[lo:hi], size=take, replace=False))
    return np.sort(np.concatenate(out))


def split_steps(cols: np.ndarray, cost: np.ndarray, nsteps: int) -> list:
    """Deal the sampled columns to nsteps disjoint parts, round-robin in cost
    order, so every part is itself a stratified sample."""
    order = cols[np.argsort(cost[cols], kind="stable")]
    return [np.sort(order[s::nsteps]) for s in range(nsteps)]


def _column_inputs(case, cols, uniforms=None):
    """numpy grid / forecast blocks of the columns `cols` (and the uniforms of
    their points, point ids k*ncol + j)."""
    dev = case.fcst3d.device
    ct = torch.as_tensor(np.asarray(cols), device=dev)
    g = {k: v.index_select(v.dim() - 1, ct).cpu().numpy() for k, v in case.grid.items()}
    f3 = case.fcst3d.index_select(3, ct).cpu().numpy()
    f2 = case.fcst2d.index_select(2, ct).cpu().numpy()
    uni = None
    if uniforms is not None:
        nlev, nij1 = case.params.nlev, case.nij1
        u = uniforms.view(nlev, nij1, *uniforms.shape[1:]).index_select(1, ct)
        uni = u.reshape(nlev * len(cols), *uniforms.shape[1:]).cpu().numpy()
    return g, f3, f2, uni


def cpu_time_columns(case, p, cols, si, rsize=4, nthreads=0, uniforms=None) -> float:
    """Seconds the C restatement takes for every level of the columns `cols`."""
    from oracle import cref
    g, f3, f2, uni = _column_inputs(case, cols, uniforms)
    ob = {k: v.cpu().numpy() for k, v in case.obs.items()}
    t = time.perf_counter()
    cref.da_main(p, g, ob, f3, f2, uniforms=uni, rsize=rsize, nthreads=nthreads, sorted_inputs=si)
    return time.perf_counter() - t


def cpu_baseline(case, p, frac: float = 0.05, nthreads: int = 0, uniforms=None) -> dict:
    """The C restatement (reference default r_size = binary32 build) on a
    stratified sample of whole grid columns, all levels, timed once on all
    host cores; returns gridpoints/s."""
    from oracle import cref
    nthreads = nthreads or os.cpu_count()
    ob = {k: v.cpu().numpy() for k, v in case.obs.items()}
    si = cref.SortedInputs(p, ob, 4)
    cost = box_candidates(p, {k: v.cpu().numpy() for k, v in case.grid.items()}, ob)
    cols = stratified_columns(cost, frac, min_cols=nthreads)
    cpu_time_columns(case, p, cols[: nthreads], si, nthreads=nthreads, uniforms=uniforms)   # warm-up
    dt = cpu_time_columns(case, p, cols, si, nthreads=nthreads, uniforms=uniforms)
    pts = cols.size * p.nlev
    return {"value": pts / dt, "unit": "gridpoints/s", "cores": nthreads, "kind": "port",
            "sample": f"{cols.size} of {case.nij1} columns ({100.0 * cols.size / case.nij1:.1f} %, all {p.nlev} "
                      f"levels = {pts} points), stratified by search-box candidate count (20 strata), "
                      f"C/OpenMP restatement, r_size=binary32 (reference default build), {dt:.1f} s"}


def oracle_check(case, p, dev, cols_frac=1.0 / 400.0, npts_w=32, uniforms=None) -> dict:
    """The GPU analysis against the FP64 oracle on a stratified column sample
    of the benchmark workload itself: max / rms relative error of the analysis
    mean and spread for the mixed and the FP64 GPU paths, and (LETKF) the
    mixed path's transform W and wvec (letkf_core, common_letkf.f90:191-208)
    through sbletkf_core_batched on sampled points."""
    from oracle import cref
    from oracle import letkf_oracle as O
    from sbpom_letkf_v2_b200.analysis import Analysis, core_batched
    ob = {k: v.cpu().numpy() for k, v in case.obs.items()}
    gfull = {k: v.cpu().numpy() for k, v in case.grid.items()}
    cost = box_candidates(p, gfull, ob)
    cols = stratified_columns(cost, cols_frac, min_cols=32, seed=9)
    g, f3, f2, uni = _column_inputs(case, cols, uniforms)
    t0 = time.perf_counter()
    ref = cref.da_main(p.replace(precision=0), g, ob, f3, f2, uniforms=uni, rsize=8)
    t_oracle = time.perf_counter() - t0
    out = {"sample": f"{cols.size} columns x {p.nlev} levels, stratified by search-box candidates",
           "oracle": "oracle/letkf_ref.c binary64", "oracle_s": t_oracle}
    ct = torch.as_tensor(cols, device=dev)
    gd = {k: v.index_select(v.dim() - 1, ct).contiguous() for k, v in case.grid.items()}
    precs = (0, 1) if p.iswitch_da != 2 else (0,)
    for prec in precs:
        an = Analysis(p.replace(precision=prec), cols.size, ob["elm"].size, device=dev)
        an.prepare_obs(case.obs)
        ud = None if uni is None else torch.as_tensor(uni, device=dev)
        a3, a2 = an.da_main(gd, torch.as_tensor(f3, device=dev, dtype=torch.float64),
                            torch.as_tensor(f2, device=dev, dtype=torch.float64), uniforms=ud)
        nob = an.count_nobsl(gd).cpu().numpy()
        an.close()
        e = mean_spread_error(a3.cpu(), a2.cpu(), torch.as_tensor(ref["anal3d"]), torch.as_tensor(ref["anal2d"]))
        e["nobsl_equal"] = bool(np.array_equal(nob, ref["nobsl"]))
        out["fp64" if prec == 0 else "mixed"] = e
    if p.iswitch_da == 1 and npts_w > 0:
        so = O.sort_obs(ob, p.nlon, p.nlat)
        nob = ref["nobsl"]
        pts = list(zip(*np.nonzero(nob > p.nmem)))
        rng = np.random.default_rng(3)
        pick = [pts[j] for j in rng.choice(len(pts), size=min(npts_w, len(pts)), replace=False)]
        blocks = []
        for k, i in pick:
            cand, dist = O.column_candidates(p, g, so, i)
            _, h, rd, rl, dp, _, _ = O.obs_local(p, so, cand, dist, k, g["depth1"][k, i])
            blocks.append((h, rd, rl, dp))
        nobl = torch.tensor([b[0].shape[0] for b in blocks], dtype=torch.int64, device=dev)
        hd = torch.tensor(np.concatenate([b[0].T.reshape(-1) for b in blocks]), device=dev)
        cat = lambda j: torch.tensor(np.concatenate([b[j] for b in blocks]), device=dev)  # noqa: E731
        wv, wm = core_batched(p.replace(precision=1), nobl, hd, cat(1), cat(2), cat(3))
        ew = ev = 0.0
        for q, (h, rd, rl, dp) in enumerate(blocks):
            rv, rm = O.letkf_core(p, h, rd, rl, dp)
            ew = max(ew, float(np.abs(wm[q].cpu().numpy().T - rm).max() / np.abs(rm).max()))
            ev = max(ev, float(np.abs(wv[q].cpu().numpy() - rv).max() / np.abs(rv).max()))
        out["mixed_W"] = {"w_max": ew, "wvec_max": ev, "points": len(blocks),
                          "nobsl_range": [int(min(b[0].shape[0] for b in blocks)),
                                          int(max(b[0].shape[0] for b in blocks))]}
    return out


def scaled_workload(wl, s: int, levels: int = 0):
    """The workload with nlon, nlat / s and observation counts / s^2, and
    with `levels` vertical levels when levels > 0."""
    if levels > 0:
        wl = wl.scaled(nlev=levels, name=wl.name + f" ({levels} levels)")
    if s <= 1:
        return wl
    q = s * s
    return wl.scaled(nlon=max(8, wl.nlon // s), nlat=max(8, wl.nlat // s), n_sst=wl.n_sst // q,
                     n_ssh=wl.n_ssh // q, n_prof=max(1, wl.n_prof // q), n_hf=wl.n_hf // q,
                     name=wl.name + f" (1/{s} grid)")


def aux_timings(case, p, dev) -> dict:
    """The steps either side of the analysis on the same workload: the
    observation operator (set_obs on the GPU) and the ensemble mean/spread of
    the forecast; CUDA-event times, best of 3."""
    from sbpom_letkf_v2_b200.analysis import ensemble_mean_spread
    from sbpom_letkf_v2_b200.obsop import obs_operator
    g = case.grid
    grid = dict(lon=g["lon1"], lat=g["lat1"], fsm=(g["phi1"] != 1.0).double(), depth=g["depth1"])
    o = case.obs
    raw = dict(elm=o["elm"], lon=o["lon"], lat=o["lat"], lev=o["lev"], err=o["err"], dat=o["dep"])

    def best(fn):
        fn()
        torch.cuda.synchronize()
        t = 1e30
        for _ in range(3):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            t = min(t, a.elapsed_time(b))
        return t
    nobs = int(o["elm"].numel())
    t_op = best(lambda: obs_operator(p, grid, case.fcst3d, case.fcst2d, raw, stats=True))
    t_ms = best(lambda: ensemble_mean_spread(p, case.fcst3d, case.fcst2d))
    es = case.fcst3d.element_size()
    by = (case.fcst3d.numel() + case.fcst2d.numel()) * es + 2 * (case.fcst3d.numel() + case.fcst2d.numel()) // p.nmem * es
    peaks, _ = _peaks()
    return {"obs_operator": {"ms": t_op, "obs_per_s": nobs / (t_op / 1e3), "nobs": nobs, "nmem": p.nmem},
            "ensemble_mean_spread": {"ms": t_ms, "gbs": by / (t_ms / 1e3) / 1e9,
                                     "frac_hbm": by / (t_ms / 1e3) / 1e9 / peaks["hbm_gbs"],
                                     "bytes": by}}


def config_of(wl, p, args, world) -> dict:
    """The workload description shared by both arms' JSON lines."""
    state_gb = 2.0 * 4.0 * wl.nmem * wl.nlon * wl.nlat * (4 * wl.nlev + 1) / 1e9
    pf = p.iswitch_da != 1
    return {"workload": wl.name, "points": wl.npoints, "nmem": p.nmem, "nobs": wl.nobs,
            "precision": args.precision if not pf else "fp64", "nmonte": p.nmonte if pf else None,
            "l2": (f"inputs larger than L2 ({state_gb:.2f} GB FP32 state read + written per step)"
                   if state_gb > 0.126 else f"inputs fit in L2 ({state_gb:.3f} GB), not flushed"),
            "parallelism": (f"column split x{world} (contiguous cost-balanced column ranges, "
                            "observations broadcast)" if world > 1 else "1 GPU")}


# ---------------------------------------------------------------------------
# the multi-GPU column split
# ---------------------------------------------------------------------------

def split_plan(nobsl: np.ndarray, k: int, nlev: int, nij1: int, world: int) -> list:
    """Contiguous column ranges [start, stop), one per rank, of nearly equal
    analysis cost (shard.point_cost summed over each column's levels)."""
    from sbpom_letkf_v2_b200.shard import partition_columns, point_cost
    col_cost = point_cost(np.asarray(nobsl).reshape(nlev, nij1), k).sum(axis=0)
    return partition_columns(col_cost, world)


def local_problem(case, parts: list, rank: int):
    """This rank's grid and forecast blocks (columns parts[rank])."""
    from sbpom_letkf_v2_b200.shard import column_slice
    start, stop = parts[rank]
    return column_slice(case.grid, case.fcst3d, case.fcst2d, start, stop)


def reference_arm(args, rank, world):
    """--impl reference: the CPU restatement, all host cores, each step a
    disjoint part of one stratified sample of >= 5 % of the columns."""
    from oracle import cref
    from sbpom_letkf_v2_b200.synthetic import WORKLOADS, make_case
    if rank != 0:
        return
    dev = "cuda:0" if torch.cuda.is_available() else "cpu"
    wl = scaled_workload(WORKLOADS[args.workload], args.scale, args.levels)
    case = make_case(wl, device=dev, seed=wl.seed)
    p = case.params.replace(precision=0)
    uni = None
    if p.iswitch_da != 1:
        from sbpom_letkf_v2_b200.synthetic import pf_uniforms
        uni = pf_uniforms(wl.npoints, p.nmonte, p.nmem, p.rm, device=dev, seed=11)
    nthreads = os.cpu_count()
    ob = {k: v.cpu().numpy() for k, v in case.obs.items()}
    si = cref.SortedInputs(p, ob, 4)
    cost = box_candidates(p, {k: v.cpu().numpy() for k, v in case.grid.items()}, ob)
    nsteps = max(1, args.steps)
    cols = stratified_columns(cost, args.ref_frac, min_cols=nsteps)
    parts = split_steps(cols, cost, nsteps)
    for _ in range(args.warmup):
        cpu_time_columns(case, p, parts[0], si, nthreads=nthreads, uniforms=uni)
    secs = [cpu_time_columns(case, p, part, si, nthreads=nthreads, uniforms=uni) for part in parts]
    pts = cols.size * p.nlev
    v = pts / sum(secs)
    ms_step = 1e3 * float(np.mean(secs))
    sample = (f"{cols.size} of {case.nij1} columns ({100.0 * cols.size / case.nij1:.1f} %), all {p.nlev} levels "
              f"= {pts} points, stratified by search-box candidate count (20 strata), dealt round-robin to the "
              f"{nsteps} timed steps ({pts // nsteps} points per step); C/OpenMP restatement, r_size=binary32 "
              f"(reference default build), {nthreads} threads")
    line = {"metric": METRIC, "value": v, "unit": "gridpoints/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference",
            "config": config_of(wl, case.params, args, world),
            "step": "one part of the column sample (not the whole grid): ms_per_step is its measured time",
            "extrapolated_full_ms": 1e3 * wl.npoints / v,
            "cpu_baseline": {"value": v, "unit": "gridpoints/s", "cores": nthreads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": v, "unit": "gridpoints/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", type=int, default=1)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--no-fp64-compare", action="store_true",
                    help="skip the one-step FP64-path measurement reported beside the mixed path")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-graph", action="store_true", help="launch eagerly instead of replaying CUDA graphs")
    ap.add_argument("--tune", action="store_true",
                    help="pick schedule and tensor-core routing with the autotuner before timing")
    ap.add_argument("--schedule", choices=["auto", "pipeline", "columns", "point"], default="auto",
                    help="auto (pipelined column queue for the mixed path with 65 <= k <= 112, column queue "
                         "otherwise, one CTA per point for the LPF), or one of those for every path (the LPF "
                         "always uses its default)")
    ap.add_argument("--no-aux", action="store_true",
                    help="skip the timing of the observation operator and the ensemble statistics")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-oracle-check", action="store_true",
                    help="skip the GPU-vs-oracle error on a column sample of the workload")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--ref-frac", type=float, default=0.05,
                    help="reference arm / CPU baseline: fraction of the columns sampled (stratified)")
    ap.add_argument("--scale", type=int, default=1,
                    help="divide nlon and nlat by S and the obs counts by S^2 (same obs density; "
                         "for profiling runs)")
    ap.add_argument("--levels", type=int, default=0,
                    help="use L vertical levels instead of the workload's (for profiling runs: the full "
                         "horizontal grid, so the same column-queue items, at a fraction of the points)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        # host cores only: rank 0 runs, the other ranks exit; no process group
        reference_arm(args, rank, world)
        return
    pg = False
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device(f"cuda:{local}"))
        pg = True

    from sbpom_letkf_v2_b200.analysis import Analysis
    from sbpom_letkf_v2_b200.params import PREC_FP64, PREC_MIXED
    from sbpom_letkf_v2_b200.synthetic import WORKLOADS, make_case, pf_uniforms

    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)
    wl = scaled_workload(WORKLOADS[args.workload], args.scale, args.levels)
    case = make_case(wl, device=dev, seed=wl.seed)        # the same workload on every rank
    if pg:   # rank 0's observations, replicated over NCCL (common_obs.f90:140)
        from sbpom_letkf_v2_b200.shard import broadcast_obs
        case.obs = broadcast_obs(case.obs if rank == 0 else None, src=0, device=dev)
    prec = PREC_MIXED if args.precision == "mixed" else PREC_FP64
    p = case.params.replace(precision=prec)
    nobs = case.obs["elm"].numel()
    pf = p.iswitch_da != 1
    uni_full = pf_uniforms(wl.npoints, p.nmonte, p.nmem, p.rm, device=dev, seed=11) if pf else None

    # nobsl of every point (the cost model of the split, the work formulas)
    an0 = Analysis(p, case.nij1, nobs, device=dev)
    an0.prepare_obs(case.obs)
    nobsl_full = an0.count_nobsl(case.grid).cpu().numpy()
    an0.close()
    parts = split_plan(nobsl_full, p.nmem, p.nlev, case.nij1, world)
    start, stop = parts[rank]
    grid, f3, f2 = local_problem(case, parts, rank)
    ncol = stop - start
    P_local = p.nlev * ncol
    uni = None
    if pf:
        uni = uni_full.view(p.nlev, case.nij1, *uni_full.shape[1:])[:, start:stop]
        uni = uni.reshape(P_local, *uni_full.shape[1:]).contiguous()

    an = Analysis(p, ncol, nobs, device=dev)
    sched = {"auto": Analysis.SCHED_AUTO, "pipeline": Analysis.SCHED_PIPELINE, "columns": Analysis.SCHED_COLUMNS,
             "point": Analysis.SCHED_POINT}[args.schedule]
    if not pf:   # the LPF keeps its default (one CTA per point)
        an.set_schedule(sched)
    tuned = None
    if args.tune:
        from sbpom_letkf_v2_b200 import tune
        tuned = tune.tune(p, grid, f3, f2, case.obs, uniforms=uni, cache=None)
        p = tune.apply(an, p, tuned)
        an.params = p
        an._cp = p.to_c()
    an.prepare_obs(case.obs)
    a3 = torch.empty_like(f3)
    a2 = torch.empty_like(f2)
    s = torch.cuda.current_stream()

    def step():
        an.prepare_obs(case.obs)
        an.da_main(grid, f3, f2, uniforms=uni, anal3d=a3, anal2d=a2, check=False)

    for _ in range(args.warmup):
        step()
    an.raise_status()

    def barrier():
        if pg:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(*vals):
        if not pg:
            return vals
        import torch.distributed as dist
        tt = torch.tensor(vals, device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return tuple(float(x) for x in tt)

    # one cycle = two CUDA graphs (observation bucketing, analysis), so the
    # analysis kernel can be timed with events on this stream between them
    g_prep = g_ana = None
    if not args.no_graph:
        cs = torch.cuda.Stream(device=dev)
        cs.wait_stream(s)
        g_prep, g_ana = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
        with torch.cuda.graph(g_prep, stream=cs):
            an.prepare_obs(case.obs)
        with torch.cuda.graph(g_ana, stream=cs):
            an.da_main(grid, f3, f2, uniforms=uni, anal3d=a3, anal2d=a2, check=False)
        s.wait_stream(cs)
        g_prep.replay()
        g_ana.replay()
        torch.cuda.synchronize()
        an.raise_status()

    # ---- device-timed region: K steps, with the analysis kernel timed inside
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    torch.cuda.synchronize()
    barrier()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    with Clocks(dev.index) as clk:
        t0.record(s)
        for i in range(args.steps):
            if g_prep is not None:
                g_prep.replay()
                ev[i][0].record(s)
                g_ana.replay()
                ev[i][1].record(s)
            else:
                an.prepare_obs(case.obs)
                ev[i][0].record(s)
                an.da_main(grid, f3, f2, uniforms=uni, anal3d=a3, anal2d=a2, check=False)
                ev[i][1].record(s)
        t1.record(s)
        torch.cuda.synchronize()
    barrier()
    ms = t0.elapsed_time(t1) / args.steps
    kern_ms = float(np.mean([a.elapsed_time(b) for a, b in ev]))
    an.raise_status()
    ms, kern_ms_max = max_over_ranks(ms, kern_ms)
    P = wl.npoints
    value = P / (ms / 1e3)

    # ---- end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        hobs = {k: v.cpu().pin_memory() for k, v in case.obs.items()}
        hf3 = f3.cpu().pin_memory()
        hf2 = f2.cpu().pin_memory()
        ha3 = torch.empty_like(hf3).pin_memory()
        ha2 = torch.empty_like(hf2).pin_memory()
        d_obs = {k: torch.empty_like(v, device=dev) for k, v in hobs.items()}
        d3 = torch.empty_like(f3)
        d2 = torch.empty_like(f2)
        hu = uni.cpu().pin_memory() if pf else None
        d_uni = torch.empty_like(uni) if pf else None
        h2d = sum(v.numel() * v.element_size() for v in hobs.values()) + hf3.numel() * 4 + hf2.numel() * 4
        h2d += hu.numel() * 8 if pf else 0
        d2h = ha3.numel() * 4 + ha2.numel() * 4

        def e2e_step():
            for k, v in hobs.items():
                d_obs[k].copy_(v, non_blocking=True)
            d3.copy_(hf3, non_blocking=True)
            d2.copy_(hf2, non_blocking=True)
            if pf:
                d_uni.copy_(hu, non_blocking=True)
            an.prepare_obs(d_obs)
            an.da_main(grid, d3, d2, uniforms=d_uni, anal3d=a3, anal2d=a2, check=False)
            ha3.copy_(a3, non_blocking=True)
            ha2.copy_(a2, non_blocking=True)

        e2e_step()
        torch.cuda.synchronize()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        ne = max(1, min(args.steps, 3))
        e0.record(s)
        for _ in range(ne):
            e2e_step()
        e1.record(s)
        torch.cuda.synchronize()
        barrier()
        ems, = max_over_ranks(e0.elapsed_time(e1) / ne)
        e2e = {"value": P / (ems / 1e3), "unit": "gridpoints/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": ems,
               "note": "per rank: its columns' state, all observations" if world > 1 else None}

    # ---- the FP64 path on the same inputs (one warm-up, one timed step)
    fp64 = None
    if prec == PREC_MIXED and not pf and not args.no_fp64_compare:
        m3, m2 = a3.clone(), a2.clone()
        p64 = p.replace(precision=PREC_FP64)
        an.prepare_obs(case.obs)
        an.da_main(grid, f3, f2, uniforms=uni, anal3d=a3, anal2d=a2, params=p64, check=False)
        torch.cuda.synchronize()
        barrier()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(s)
        an.prepare_obs(case.obs)
        an.da_main(grid, f3, f2, uniforms=uni, anal3d=a3, anal2d=a2, params=p64, check=False)
        f1.record(s)
        torch.cuda.synchronize()
        barrier()
        an.raise_status()
        fms, = max_over_ranks(f0.elapsed_time(f1))
        fp64 = {"value": P / (fms / 1e3), "ms_per_step": fms, "mixed_over_fp64": fms / ms,
                "mixed_vs_fp64_gpu": mean_spread_error(m3, m2, a3, a2)}
        del m3, m2
    an.close()

    aux = None
    if not args.no_aux and rank == 0:
        aux = aux_timings(case, p, dev)
    if rank == 0:
        nob_l = nobsl_full[:, start:stop]
        peaks, src = _peaks()
        if pf:
            by = algorithmic_bytes(nob_l, p.nmem, p.nv3d, p.nv2d, p.nlev, ncol)
            gbs = by["total"] / (kern_ms / 1e3) / 1e9
            traffic = DRAM_BYTES_PER_POINT_W4 * P_local if args.workload == 4 else None
            roof = {"bound": "hbm", "achieved": gbs, "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                    "frac": gbs / peaks["hbm_gbs"] if peaks.get("hbm_gbs") else None, "traffic": traffic,
                    "kernel": "k_analysis (LPF weights + resampling gather)", "kernel_ms": kern_ms,
                    "bytes_per_launch": by, "peak_source": src + " hbm_gbs (copy)",
                    "note": "fused kernel: weights, nmonte draws and gather in one launch"}
        else:
            ob = {k: v.cpu().numpy() for k, v in case.obs.items()}
            cand = box_candidates(p, {k: v[..., start:stop].cpu().numpy() if k == "depth1" else
                                      v[start:stop].cpu().numpy() for k, v in case.grid.items()}, ob)
            tmax = p.tc_max_cand if p.tc_max_cand > 0 else TC_MAX_CAND_DEFAULT
            tmask = np.broadcast_to((cand <= tmax)[None, :], (p.nlev, ncol)) if prec == PREC_MIXED else None
            fl = algorithmic_flops(nob_l, p.nmem, p.nv3d, p.nv2d, p.nlev, ncol, tmask)
            run_sched = (("pipeline" if 65 <= p.nmem <= 112 else "columns") if args.schedule == "auto"
                         else args.schedule)
            traffic = (DRAM_BYTES_PER_POINT_W1[run_sched] * P_local
                       if (args.workload == 1 and prec == PREC_MIXED and run_sched in DRAM_BYTES_PER_POINT_W1) else None)
            roof = letkf_roofline(fl, kern_ms, _fp64_peak(dev), peaks, src, traffic)
        cpu = None
        chk = None
        if world == 1:
            if not args.no_cpu_baseline:
                cpu = cpu_baseline(case, p.replace(precision=PREC_FP64), frac=args.ref_frac, uniforms=uni_full)
            if not args.no_oracle_check:
                chk = oracle_check(case, p, dev, uniforms=uni_full)
        line = {"metric": METRIC, "value": value, "unit": "gridpoints/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None,
                "dtype": "f64" if (prec == PREC_FP64 or pf) else "bf16x3 gram (f32 acc) + f64 eig",
                "data": "synthetic (seeded, generated in device memory)",
                "config": config_of(wl, p, args, world),
                "nobsl": {"mean": float(nobsl_full.mean()), "max": int(nobsl_full.max()),
                          "zero_frac": float((nobsl_full == 0).mean())},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk.summary(), "fp64_path": fp64,
                "oracle_check": chk, "aux": aux,
                "kernel_ms_max_over_ranks": kern_ms_max,
                "gpu_launches": 6 * args.steps, "graph": g_prep is not None,
                "schedule": args.schedule if tuned is None else tuned, "peaks_source": src,
                "hbm_peak_gbs": peaks.get("hbm_gbs")}
        print(json.dumps(line), flush=True)
    if pg:
        import torch.distributed as dist
        del g_prep, g_ana   # no NCCL work in them, but release before tearing the group down
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
