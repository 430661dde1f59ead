"""Autotuner of the analysis launch.

Two knobs change speed but not the analysis (beyond rounding, and the mixed
path's stated error):

* the schedule: the pipelined column queue (``Analysis.SCHED_PIPELINE``,
  producer warps selecting the next point while consumer warps solve the
  current one), the persistent column queue with warm-started eigensolves
  (``Analysis.SCHED_COLUMNS``) or one CTA per grid point
  (``Analysis.SCHED_POINT``); the warm start pays off where points need the
  k x k eigensolve, not for the LPF;
* for the mixed path, ``tc_max_cand``: the search-box candidate count above
  which a point's Gram is accumulated in FP64 instead of on the tensor cores;
* for the column-queue schedules, the queue-item width (columns per item,
  ``Analysis.set_item_width``), timed on a block of whole latitude rows so
  that the items' columns are real neighbours.

``tune`` times the candidates on a sample of the caller's own columns
(every s-th column of the grid, all levels, the full observation set) with
CUDA events and keeps the fastest configuration whose analysis raised no
status, in a JSON cache keyed by GPU, ensemble size, levels, filter and
precision.  ``apply`` sets it on an ``Analysis`` and returns the parameters
to call it with.
"""
from __future__ import annotations

import json
import os

import torch

CACHE = os.environ.get("SBLETKF_TUNE_CACHE",
                       os.path.join(os.path.expanduser("~"), ".cache", "sbletkf", "tune.json"))
TC_CANDIDATES = (0.0, 6144.0, 3072.0)     # 0: the library default (12288)


def key(params, gpu_name: str) -> str:
    return (f"{gpu_name}|k={params.nmem}|nlev={params.nlev}|da={params.iswitch_da}"
            f"|prec={params.precision}|nmonte={params.nmonte if params.iswitch_da != 1 else 0}")


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(path, table):
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def schedules(params):
    """The launch schedules that apply: the pipelined column queue needs an
    eigensolve (not the LPF) and nmem <= 112."""
    from .analysis import Analysis
    out = [Analysis.SCHED_COLUMNS, Analysis.SCHED_POINT]
    if params.iswitch_da != 2 and params.nmem <= 112:
        out.insert(0, Analysis.SCHED_PIPELINE)
    return out


def candidates(params):
    tcs = TC_CANDIDATES if (params.precision == 1 and params.iswitch_da != 2) else (0.0,)
    return [{"schedule": s, "tc_max_cand": t} for s in schedules(params) for t in tcs]


def column_sample(grid: dict, fcst3d, fcst2d, uniforms, nlev: int, max_cols: int):
    """Every s-th column: grid arrays, state and (PF) uniforms of the sample."""
    nij1 = grid["lon1"].numel()
    stride = max(1, nij1 // max_cols)
    cols = torch.arange(0, nij1, stride, device=fcst3d.device)[:max_cols]
    g = {k: (v.index_select(v.dim() - 1, cols)).contiguous() for k, v in grid.items()}
    f3 = fcst3d.index_select(3, cols).contiguous()
    f2 = fcst2d.index_select(2, cols).contiguous()
    uni = None
    if uniforms is not None:
        u = uniforms.view(nlev, nij1, *uniforms.shape[1:]).index_select(1, cols)
        uni = u.reshape(nlev * cols.numel(), *uniforms.shape[1:]).contiguous()
    return g, f3, f2, uni


def _gpu_measure(params, grid, fcst3d, fcst2d, obs, uniforms, cand, reps):
    """Best-of-reps milliseconds of one analysis with candidate `cand`, or None
    when the analysis latched an error status."""
    from .analysis import Analysis
    p = params.replace(tc_max_cand=cand["tc_max_cand"])
    an = Analysis(p, grid["lon1"].numel(), max(1, obs["elm"].numel()), device=fcst3d.device)
    try:
        an.set_schedule(cand["schedule"])
        an.set_item_width(cand.get("item_width", 0))
        an.prepare_obs(obs)
        a3, a2 = torch.empty_like(fcst3d), torch.empty_like(fcst2d)
        an.da_main(grid, fcst3d, fcst2d, uniforms=uniforms, anal3d=a3, anal2d=a2, check=False)
        if an.status():
            return None
        best = float("inf")
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            an.da_main(grid, fcst3d, fcst2d, uniforms=uniforms, anal3d=a3, anal2d=a2, check=False)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return None if an.status() else best
    finally:
        an.close()


def row_sample(grid: dict, fcst3d, fcst2d, uniforms, nlev: int, nlon: int, max_cols: int):
    """A block of whole latitude rows from the middle of the grid (at most
    max_cols columns): columns nlon apart stay neighbours, as the column
    queue's items assume.  Grid arrays, state and (PF) uniforms of it."""
    nij1 = grid["lon1"].numel()
    nrow = nij1 // nlon
    rows = max(1, min(nrow, max_cols // max(nlon, 1)))
    c0 = (nrow - rows) // 2 * nlon
    cols = torch.arange(c0, c0 + rows * nlon, device=fcst3d.device)
    g = {k: (v.index_select(v.dim() - 1, cols)).contiguous() for k, v in grid.items()}
    f3 = fcst3d.index_select(3, cols).contiguous()
    f2 = fcst2d.index_select(2, cols).contiguous()
    uni = None
    if uniforms is not None:
        u = uniforms.view(nlev, nij1, *uniforms.shape[1:]).index_select(1, cols)
        uni = u.reshape(nlev * cols.numel(), *uniforms.shape[1:]).contiguous()
    return g, f3, f2, uni


WIDTHS = (0, 1, 2, 4, 8)   # columns per queue item (0: the library's choice)


def tune(params, grid: dict, fcst3d, fcst2d, obs: dict, uniforms=None, max_cols: int = 4096, reps: int = 2,
         cache: str | None = CACHE, force: bool = False, gpu_name: str | None = None, measure=None) -> dict:
    """The fastest configuration for this workload: {"schedule", "tc_max_cand",
    "item_width", "ms": {candidate: time}, "ms_width": {width: time}}; read
    from / written to `cache` (None: no cache).  Stage 1 times schedule x
    tensor-core routing on a column sample; stage 2 times the queue-item
    widths of the chosen queue schedule on a block of whole rows."""
    if gpu_name is None:
        gpu_name = torch.cuda.get_device_name(fcst3d.device) if fcst3d.is_cuda else "cpu"
    k = key(params, gpu_name)
    table = _load(cache) if cache else {}
    if not force and k in table:
        return table[k]
    measure = measure or _gpu_measure
    g, f3, f2, uni = column_sample(grid, fcst3d, fcst2d, uniforms, params.nlev, max_cols)
    times = {}
    for cand in candidates(params):
        t = measure(params, g, f3, f2, obs, uni, cand, reps)
        if t is not None:
            times[json.dumps(cand, sort_keys=True)] = t
    if not times:
        raise RuntimeError("no candidate configuration completed without an error status")
    best = json.loads(min(times, key=times.get))
    best["item_width"] = 0
    wtimes = {}
    if best["schedule"] != 0:   # a column-queue schedule: tune its item width
        gr, r3, r2, ur = row_sample(grid, fcst3d, fcst2d, uniforms, params.nlev, params.nlon, max_cols)
        for wd in WIDTHS:
            t = measure(params, gr, r3, r2, obs, ur, dict(best, item_width=wd), reps)
            if t is not None:
                wtimes[str(wd)] = t
        if wtimes:
            best["item_width"] = int(min(wtimes, key=wtimes.get))
    result = dict(best, ms=times, ms_width=wtimes, sample_columns=int(g["lon1"].numel()))
    if cache:
        table = _load(cache)
        table[k] = result
        _store(cache, table)
    return result


def apply(analysis, params, cfg: dict):
    """Set the tuned schedule and item width on `analysis`; return the
    parameters to use."""
    analysis.set_schedule(int(cfg["schedule"]))
    analysis.set_item_width(int(cfg.get("item_width", 0)))
    return params.replace(tc_max_cand=float(cfg["tc_max_cand"]))
