"""Host-side pieces of bench.py on the CPU: workload scaling for profiling
runs, the algorithmic work formulas behind `roofline`, the mixed-path error
metric, and the JSON line of the reference arm (the CPU restatement timed
on a column sample)."""
import json
import os
import subprocess
import sys

import numpy as np
import torch

import bench
from sbpom_letkf_v2_b200.synthetic import WORKLOADS

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_scaled_workload_grid_levels_and_obs_density():
    wl = WORKLOADS[1]
    assert bench.scaled_workload(wl, 1) is wl
    s8 = bench.scaled_workload(wl, 8)
    assert (s8.nlon, s8.nlat, s8.nlev) == (50, 37, 40)
    assert (s8.n_sst, s8.n_ssh, s8.n_prof) == (wl.n_sst // 64, wl.n_ssh // 64, wl.n_prof // 64)
    l2 = bench.scaled_workload(wl, 1, levels=2)
    assert (l2.nlon, l2.nlat, l2.nlev) == (400, 300, 2)
    assert (l2.n_sst, l2.n_ssh, l2.n_prof) == (wl.n_sst, wl.n_ssh, wl.n_prof)   # full horizontal grid
    both = bench.scaled_workload(wl, 4, levels=3)
    assert (both.nlon, both.nlat, both.nlev) == (100, 75, 3)


def test_box_candidates_and_stratified_sample():
    """The host-side candidate count of each column's search box equals the
    oracle's candidate list length, and the stratified sample takes the same
    share of every cost stratum."""
    from oracle import letkf_oracle as O
    from sbpom_letkf_v2_b200.synthetic import make_case
    wl = WORKLOADS[0].scaled(nlon=20, nlat=16, nlev=2, nmem=6, n_sst=300, n_ssh=80, n_prof=4, seed=41)
    case = make_case(wl, sigma_obs=90e3)
    p = case.params
    g = {k: v.numpy() for k, v in case.grid.items()}
    ob = {k: v.numpy() for k, v in case.obs.items()}
    cand = bench.box_candidates(p, g, ob)
    so = O.sort_obs(ob, p.nlon, p.nlat)
    for i in range(case.nij1):
        imin, imax, jmin, jmax = O.search_box(p, g, i)
        assert cand[i] == O.obs_local_sub(so, p.nlon, imin, imax, jmin, jmax).size
    cost = np.arange(1000, dtype=np.float64)[::-1].copy()
    cols = bench.stratified_columns(cost, 0.05, nstrata=10, seed=1)
    assert cols.size == 50 and np.array_equal(cols, np.unique(cols))
    order = np.argsort(cost, kind="stable")
    rank = np.empty(1000, np.int64)
    rank[order] = np.arange(1000)
    assert np.array_equal(np.bincount(rank[cols] // 100, minlength=10), np.full(10, 5))
    parts = bench.split_steps(cols, cost, 3)
    assert sorted(np.concatenate(parts).tolist()) == cols.tolist()
    assert max(p.size for p in parts) - min(p.size for p in parts) <= 1


def test_algorithmic_work_formulas():
    """Per point with n local obs: F_gram = 2k^2 n, F_eig = 9k^3 and
    F_W = 2k^3 + 2kn + 2k^2 only where n > 0, F_upd = 2 nv k^2; bytes
    B_w = 4n(k+3), B_g = 8 k nv; nv includes the 2D variables on the
    surface level (the last one)."""
    k, nv3d, nv2d, nlev, nij1 = 10, 4, 1, 2, 3
    n = np.array([0, 5, 7, 1, 0, 2], dtype=np.int64)        # [nlev][nij1]
    f = bench.algorithmic_flops(n, k, nv3d, nv2d, nlev, nij1)
    has = (n > 0).sum()
    nv = np.array([nv3d] * nij1 + [nv3d + nv2d] * nij1, dtype=np.float64)
    assert f["gram"] == 2.0 * k * k * n.sum()
    assert f["eig"] == 9.0 * k ** 3 * has
    assert f["w"] == float(((2.0 * k ** 3 + 2.0 * k * n + 2.0 * k * k) * (n > 0)).sum())
    assert f["upd"] == float((2.0 * nv * k * k).sum())
    assert f["total"] == f["gram"] + f["eig"] + f["w"] + f["upd"]
    tm = np.array([True, True, False, True, False, False])
    ft = bench.algorithmic_flops(n, k, nv3d, nv2d, nlev, nij1, tm)
    assert ft["gram_tensor"] == 2.0 * k * k * (5 + 1) and ft["gram_fp64"] == 2.0 * k * k * (7 + 0 + 2)
    roof = bench.letkf_roofline(ft, 2.0, {"tflops": 40.0, "source": "x"}, {"bf16_tflops_sustained": 1000.0},
                                "measured", None)
    assert abs(roof["achieved"] - (ft["eig"] + ft["w"] + ft["gram_fp64"]) / 2e-3 / 1e12) < 1e-12
    assert abs(roof["frac"] - roof["achieved"] / 40.0) < 1e-15
    assert abs(roof["tensor"]["frac"] - ft["gram_tensor"] / 2e-3 / 1e12 / 1000.0) < 1e-15
    b = bench.algorithmic_bytes(n, k, nv3d, nv2d, nlev, nij1)
    assert b["weights"] == float((4.0 * n * (k + 3)).sum())
    assert b["gather"] == float((8.0 * k * nv).sum())


def test_mean_spread_error_metric():
    g = torch.Generator().manual_seed(4)
    r3 = torch.randn(2, 16, 3, 5, generator=g, dtype=torch.float64) + 10.0
    r2 = torch.randn(1, 16, 5, generator=g, dtype=torch.float64)
    z = bench.mean_spread_error(r3, r2, r3, r2)
    assert z == {"mean_max": 0.0, "mean_rms": 0.0, "spread_max": 0.0, "spread_rms": 0.0}
    a3 = r3.clone()
    a3[1] += 1e-3                                            # shifts variable 1's mean only
    e = bench.mean_spread_error(a3, r2, r3, r2)
    want = 1e-3 / float(r3[1].mean(0).abs().max())
    # the shift itself rounds at eps * 10 / 1e-3 ~ 2e-12 relative
    assert abs(e["mean_max"] - want) <= 1e-9 * want
    assert e["spread_max"] < 1e-12


def test_reference_arm_json_line():
    """`bench.py --impl reference` prints one JSON line with the contract's
    keys; its e2e moves no bytes between host and device."""
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "0", "--steps", "1",
                        "--warmup", "0", "--ref-frac", "0.01"], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["unit"] == "gridpoints/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["config"]["workload"] == WORKLOADS[0].name
    # the timed step is a part of the sample: value and ms_per_step agree
    pts = int(line["cpu_baseline"]["sample"].split("= ")[1].split(" points")[0])
    assert abs(pts / (line["ms_per_step"] / 1e3) - line["value"]) <= 1e-6 * line["value"]
    assert line["extrapolated_full_ms"] > line["ms_per_step"]


def test_reference_arm_under_torchrun_prints_once():
    """Launched as the multi-GPU contract launches it (torchrun, 2 ranks), the
    reference arm runs on rank 0 only, needs no process group, and prints one
    JSON line; every rank exits 0."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                        "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
                        "--gpus", "2", "--workload", "0", "--steps", "1", "--warmup", "0", "--ref-frac", "0.005"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0


def _split_rank(rank, world, port, outdir):
    """bench.py's multi-GPU code path on gloo ranks: the same workload on every
    rank, rank 0's observations broadcast, split_plan / local_problem cut the
    columns, each rank analyses its own (the oracle stands in for the GPU
    analysis), and the gathered result equals the single-domain analysis."""
    import torch.distributed as dist

    from oracle import letkf_oracle as O
    from sbpom_letkf_v2_b200.shard import broadcast_obs, gather_columns
    from sbpom_letkf_v2_b200.synthetic import make_case
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    wl = WORKLOADS[0].scaled(nlon=14, nlat=10, nlev=3, nmem=10, n_sst=120, n_ssh=30, n_prof=3, seed=7)
    case = make_case(wl, seed=wl.seed, cov_infl_mul=1.1, sigma_obs=60e3)
    case.obs = broadcast_obs(case.obs if rank == 0 else None, src=0)
    p = case.params
    g = {k: v.numpy() for k, v in case.grid.items()}
    ob = {k: v.numpy() for k, v in case.obs.items()}
    nobsl = O.count_nobsl(p, g, ob)
    parts = bench.split_plan(nobsl, p.nmem, p.nlev, case.nij1, world)
    gl, f3, f2 = bench.local_problem(case, parts, rank)
    assert f3.shape[-1] == parts[rank][1] - parts[rank][0]
    r = O.da_main(p, {k: v.numpy() for k, v in gl.items()}, ob, f3.numpy(), f2.numpy())
    a3, a2 = gather_columns(torch.from_numpy(r.anal3d), torch.from_numpy(r.anal2d), parts)
    if rank == 0:
        full = O.da_main(p, g, ob, case.fcst3d.numpy(), case.fcst2d.numpy())
        ok = np.array_equal(a3.numpy(), full.anal3d) and np.array_equal(a2.numpy(), full.anal2d)
        ok = ok and all(b > a for a, b in parts)
        with open(os.path.join(outdir, "result"), "w") as f:
            f.write("ok" if ok else "mismatch")
    dist.barrier()
    dist.destroy_process_group()


def test_bench_column_split_on_two_gloo_ranks(tmp_path):
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    mp.spawn(_split_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    assert (tmp_path / "result").read_text() == "ok"
