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

Multi-GPU (torchrun): every rank analyses its own copy of the workload
(independent domains, no collective on the data path) -> weak scaling.
"""
from __future__ import annotations

import os

os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")

import argparse  # noqa: E402
import json  # noqa: E402
import statistics  # noqa: E402
import subprocess  # noqa: E402
import threading  # noqa: E402
import time  # noqa: E402

import numpy as np  # noqa: E402
import torch  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
METRIC = "analysis gridpoints/s per LETKF cycle, mixed vs FP64 on B200 at <=1e-4 rel err"


def _peaks():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def _fp64_peak(dev) -> dict:
    """FP64 roofline denominator: cuBLAS DGEMM 8192^3 through torch.matmul,
    best of 5 (the FP64 counterpart of the driver's bf16 GEMM peak)."""
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
            "source": "measured: cuBLAS DGEMM 8192^3 via torch.matmul, best of 5"}


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


def algorithmic_flops(nobsl: np.ndarray, k: int, nv3d: int, nv2d: int, nlev: int, nij1: int) -> dict:
    """Per-launch algorithmic work of the analysis (per point with n local obs):
    F_gram = 2 k^2 n, F_eig = 9 k^3, F_W = 2k^3 + 2kn + 2k^2, F_upd = 2 nv k^2."""
    n = nobsl.astype(np.float64).reshape(nlev, nij1)
    has = n > 0
    nv = np.full_like(n, nv3d, dtype=np.float64)
    nv[nlev - 1, :] += nv2d
    f_gram = float((2.0 * k * k * n).sum())
    f_eig = float((9.0 * k ** 3) * has.sum())
    f_w = float(((2.0 * k ** 3 + 2.0 * k * n + 2.0 * k * k) * has).sum())
    f_upd = float((2.0 * nv * k * k).sum())
    return {"gram": f_gram, "eig": f_eig, "w": f_w, "upd": f_upd, "total": f_gram + f_eig + f_w + f_upd}


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


def mean_spread_error(a3, a2, r3, r2) -> dict:
    """Relative error of the analysis ensemble mean and spread of (a3, a2)
    against (r3, r2), per variable: max |x - r| / max |r| and
    rms(x - r) / rms(r); the worst variable is reported."""
    out = {"mean_max": 0.0, "mean_rms": 0.0, "spread_max": 0.0, "spread_rms": 0.0}
    for a, r in ((a3, r3), (a2, r2)):
        for v in range(a.shape[0]):
            x, y = a[v].double(), r[v].double()
            for name, fx, fy in (("mean", x.mean(0), y.mean(0)), ("spread", x.std(0), y.std(0))):
                d = fx - fy
                mx = float(d.abs().max() / fy.abs().max().clamp_min(1e-300))
                rms = float(torch.sqrt((d * d).mean() / (fy * fy).mean().clamp_min(1e-300)))
                out[name + "_max"] = max(out[name + "_max"], mx)
                out[name + "_rms"] = max(out[name + "_rms"], rms)
    return out


def cpu_baseline(case, p, seconds: float = 15.0, nthreads: int = 0, uniforms=None):
    """The C restatement (reference default r_size = binary32 build) on a
    stratified sample of whole grid columns, all levels; returns gridpoints/s."""
    from oracle import cref
    nthreads = nthreads or os.cpu_count()
    nij1 = case.nij1
    g_all = {k: v.cpu().numpy() for k, v in case.grid.items()}
    ob = {k: v.cpu().numpy() for k, v in case.obs.items()}
    si = cref.SortedInputs(p, ob, 4)

    def run(cols):
        g = {k: (v[:, cols] if v.ndim == 2 else v[cols]) for k, v in g_all.items()}
        ct = torch.as_tensor(cols, device=case.fcst3d.device)
        f3 = case.fcst3d[:, :, :, ct].cpu().numpy()
        f2 = case.fcst2d[:, :, ct].cpu().numpy()
        uni = None
        if uniforms is not None:  # point ids k*nij1+i -> k*ncols+j of the sampled columns
            u = uniforms.view(p.nlev, nij1, *uniforms.shape[1:])[:, ct]
            uni = u.reshape(p.nlev * len(cols), *uniforms.shape[1:]).cpu().numpy()
        t = time.perf_counter()
        cref.da_main(p, g, ob, f3, f2, uniforms=uni, rsize=4, nthreads=nthreads, sorted_inputs=si)
        return time.perf_counter() - t

    rng = np.random.default_rng(5)
    cal = np.sort(rng.choice(nij1, size=max(nthreads, 16), replace=False))
    tc = run(cal)
    ncol = int(min(nij1, max(nthreads, seconds / max(tc, 1e-3) * cal.size)))
    stride = max(1, nij1 // ncol)
    cols = np.arange(0, nij1, stride)[:ncol]
    dt = run(cols)
    pts = cols.size * p.nlev
    return {"value": pts / dt, "unit": "gridpoints/s", "cores": nthreads, "kind": "port",
            "sample": f"{cols.size} of {nij1} columns (every {stride}th, all {p.nlev} levels = {pts} points), "
                      f"C/OpenMP restatement, r_size=binary32 (reference default build), {dt:.1f} s"}


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
            "parallelism": f"replicas x{world}"}


def reference_arm(args, rank, world):
    """--impl reference: the CPU restatement timed per step on a bounded sample."""
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
    vals = []
    for s in range(args.warmup + args.steps):
        r = cpu_baseline(case, p, seconds=args.ref_seconds, uniforms=uni)
        if s >= args.warmup:
            vals.append(r["value"])
    v = float(np.mean(vals))
    line = {"metric": METRIC, "value": v, "unit": "gridpoints/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * wl.npoints / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference",
            "config": config_of(wl, case.params, args, world),
            "cpu_baseline": {"value": v, "unit": "gridpoints/s", "cores": r["cores"], "kind": "port",
                             "sample": r["sample"]},
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
    ap.add_argument("--schedule", choices=["columns", "point"], default="columns",
                    help="persistent column queue with warm-started eigensolves, or one CTA per point")
    ap.add_argument("--no-aux", action="store_true",
                    help="skip the timing of the observation operator and the ensemble statistics")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--ref-seconds", type=float, default=8.0)
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
    case = make_case(wl, device=dev, seed=wl.seed + rank)
    prec = PREC_MIXED if args.precision == "mixed" else PREC_FP64
    p = case.params.replace(precision=prec)
    nobs = case.obs["elm"].numel()
    an = Analysis(p, case.nij1, nobs, device=dev)
    an.set_schedule(Analysis.SCHED_COLUMNS if args.schedule == "columns" else Analysis.SCHED_POINT)
    tuned = None
    if args.tune:
        from sbpom_letkf_v2_b200 import tune
        uni0 = (pf_uniforms(wl.npoints, p.nmonte, p.nmem, p.rm, device=dev, seed=11 + rank)
                if p.iswitch_da != 1 else None)
        tuned = tune.tune(p, case.grid, case.fcst3d, case.fcst2d, case.obs, uniforms=uni0, cache=None)
        p = tune.apply(an, p, tuned)
        an.params = p
        an._cp = p.to_c()
    an.prepare_obs(case.obs)
    nobsl = an.count_nobsl(case.grid).cpu().numpy()
    a3 = torch.empty_like(case.fcst3d)
    a2 = torch.empty_like(case.fcst2d)
    s = torch.cuda.current_stream()
    pf = p.iswitch_da != 1
    uni = pf_uniforms(wl.npoints, p.nmonte, p.nmem, p.rm, device=dev, seed=11 + rank) if pf else None

    def step():
        an.prepare_obs(case.obs)
        an.da_main(case.grid, case.fcst3d, case.fcst2d, uniforms=uni, anal3d=a3, anal2d=a2, check=False)

    for _ in range(args.warmup):
        step()
    an.raise_status()

    def barrier():
        if pg:
            import torch.distributed as dist
            dist.barrier()

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
            an.da_main(case.grid, case.fcst3d, case.fcst2d, uniforms=uni, anal3d=a3, anal2d=a2, check=False)
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
                an.da_main(case.grid, case.fcst3d, case.fcst2d, uniforms=uni, anal3d=a3, anal2d=a2, check=False)
                ev[i][1].record(s)
        t1.record(s)
        torch.cuda.synchronize()
    barrier()
    ms = t0.elapsed_time(t1) / args.steps
    kern_ms = float(np.mean([a.elapsed_time(b) for a, b in ev]))
    an.raise_status()
    if pg:
        import torch.distributed as dist
        tt = torch.tensor([ms, kern_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms, kern_ms = float(tt[0]), float(tt[1])
    P = wl.npoints
    value = P * world / (ms / 1e3)

    # ---- end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        hobs = {k: v.cpu().pin_memory() for k, v in case.obs.items()}
        hf3 = case.fcst3d.cpu().pin_memory()
        hf2 = case.fcst2d.cpu().pin_memory()
        ha3 = torch.empty_like(hf3).pin_memory()
        ha2 = torch.empty_like(hf2).pin_memory()
        d_obs = {k: torch.empty_like(v, device=dev) for k, v in hobs.items()}
        d3 = torch.empty_like(case.fcst3d)
        d2 = torch.empty_like(case.fcst2d)
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
            an.da_main(case.grid, d3, d2, uniforms=d_uni, anal3d=a3, anal2d=a2, check=False)
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
        ems = e0.elapsed_time(e1) / ne
        if pg:
            import torch.distributed as dist
            tt = torch.tensor([ems], device=dev, dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ems = float(tt[0])
        e2e = {"value": P * world / (ems / 1e3), "unit": "gridpoints/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": ems}

    # ---- the FP64 path on the same inputs (one warm-up, one timed step)
    fp64 = None
    if prec == PREC_MIXED and not pf and not args.no_fp64_compare:
        m3, m2 = a3.clone(), a2.clone()
        p64 = p.replace(precision=PREC_FP64)
        an.prepare_obs(case.obs)
        an.da_main(case.grid, case.fcst3d, case.fcst2d, uniforms=uni, anal3d=a3, anal2d=a2, params=p64, check=False)
        torch.cuda.synchronize()
        barrier()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(s)
        an.prepare_obs(case.obs)
        an.da_main(case.grid, case.fcst3d, case.fcst2d, uniforms=uni, anal3d=a3, anal2d=a2, params=p64, check=False)
        f1.record(s)
        torch.cuda.synchronize()
        barrier()
        an.raise_status()
        fms = f0.elapsed_time(f1)
        if pg:
            import torch.distributed as dist
            tt = torch.tensor([fms], device=dev, dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            fms = float(tt[0])
        fp64 = {"value": P * world / (fms / 1e3), "ms_per_step": fms, "mixed_over_fp64": fms / ms,
                "mixed_error": mean_spread_error(m3, m2, a3, a2)}
        del m3, m2

    aux = None
    if not args.no_aux:
        aux = aux_timings(case, p, dev)
    if rank == 0:
        fl = algorithmic_flops(nobsl, p.nmem, p.nv3d, p.nv2d, p.nlev, case.nij1)
        f64 = _fp64_peak(dev)
        peaks, src = _peaks()
        if pf:
            by = algorithmic_bytes(nobsl, p.nmem, p.nv3d, p.nv2d, p.nlev, case.nij1)
            gbs = by["total"] / (kern_ms / 1e3) / 1e9
            # DRAM bytes per launch: an ncu capture of the same kernel on the 1/2
            # grid of workload 4 (bench.py --workload 4 --scale 2) read and
            # wrote 280.6 MB for 61,440 points; scaled by the points of this launch
            traffic = 280.6e6 / 61440.0 * P if args.workload == 4 else None
            roof = {"bound": "hbm", "achieved": gbs, "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                    "frac": gbs / peaks["hbm_gbs"] if peaks.get("hbm_gbs") else None, "traffic": traffic,
                    "kernel": "k_analysis (LPF weights + resampling gather)", "kernel_ms": kern_ms,
                    "bytes_per_launch": by, "peak_source": src + " hbm_gbs (copy)",
                    "note": "fused kernel: weights, nmonte draws and gather in one launch"}
        else:
            achieved = fl["total"] / (kern_ms / 1e3) / 1e12
            # DRAM bytes per launch: an ncu capture of the same kernel on the full
            # horizontal grid with 2 levels (bench.py --levels 2), which gets the
            # same 8-column queue items, read and wrote 1073.6 MB for 240,000
            # points; scaled by the points of this launch
            traffic = (1073.6e6 / 240000.0 * P if (args.workload == 1 and prec == PREC_MIXED
                                                   and args.schedule == "columns") else None)
            roof = {"bound": "fp64", "achieved": achieved, "peak": f64["tflops"], "unit": "TFLOP/s",
                    "frac": achieved / f64["tflops"], "traffic": traffic, "kernel": "k_analysis",
                    "peak_source": f64["source"], "kernel_ms": kern_ms, "flops_per_launch": fl,
                    "note": "FP64 eigensolve bound"}
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            cpu = cpu_baseline(case, p.replace(precision=PREC_FP64), seconds=15.0, uniforms=uni)
        line = {"metric": METRIC, "value": value, "unit": "gridpoints/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None,
                "dtype": "f64" if (prec == PREC_FP64 or pf) else "bf16x3 gram (f32 acc) + f64 eig",
                "data": "synthetic (seeded, generated in device memory)",
                "config": config_of(wl, p, args, world),
                "nobsl": {"mean": float(nobsl.mean()), "max": int(nobsl.max()), "zero_frac": float((nobsl == 0).mean())},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk.summary(), "fp64_path": fp64,
                "aux": aux,
                "gpu_launches": 6 * args.steps, "graph": g_prep is not None, "schedule": args.schedule if tuned is None else tuned, "peaks_source": src,
                "hbm_peak_gbs": peaks.get("hbm_gbs")}
        print(json.dumps(line), flush=True)
    an.close()
    if pg:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
