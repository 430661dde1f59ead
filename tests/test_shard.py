"""Host logic of the multi-GPU split (sbpom_letkf_v2_b200/shard.py), run as
two gloo ranks on CPU: column partition, observation broadcast, per-rank
analysis of its columns and the gather.  The per-rank analysis here is the
FP64 oracle, so the sharded result must equal the single-domain one exactly
(every point is computed the same way whichever rank owns it)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from sbpom_letkf_v2_b200.shard import column_slice, partition_columns, point_cost


def test_partition_is_contiguous_and_balanced():
    rng = np.random.default_rng(0)
    cost = rng.exponential(size=1000) * (rng.random(1000) < 0.3) + 0.01
    for n in (1, 2, 3, 8):
        parts = partition_columns(cost, n)
        assert parts[0][0] == 0 and parts[-1][1] == 1000
        assert all(parts[r][1] == parts[r + 1][0] for r in range(n - 1))
        loads = [cost[a:b].sum() for a, b in parts]
        assert max(loads) <= cost.sum() / n + cost.max() + 1e-9


def test_point_cost_grows_with_nobsl():
    c = point_cost([0, 1, 10, 1000], 64)
    assert np.all(np.diff(c) > 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, outdir):
    import torch.distributed as dist

    from oracle import letkf_oracle as O
    from sbpom_letkf_v2_b200.shard import broadcast_obs, gather_columns
    from sbpom_letkf_v2_b200.synthetic import WORKLOADS, make_case
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    wl = WORKLOADS[0].scaled(nlon=14, nlat=10, nlev=3, nmem=10, n_sst=120, n_ssh=30, n_prof=3, seed=5)
    case = make_case(wl, cov_infl_mul=1.1, sigma_obs=60e3)       # grid and forecast: every rank builds them
    p = case.params
    obs = broadcast_obs(case.obs if rank == 0 else None, src=0)
    g = {k: v.numpy() for k, v in case.grid.items()}
    ob = {k: v.numpy() for k, v in obs.items()}
    nobsl = O.count_nobsl(p, g, ob)                              # [nlev][nij1]
    parts = partition_columns(point_cost(nobsl, p.nmem).sum(axis=0), world)
    a, b = parts[rank]
    gl, f3, f2 = column_slice(case.grid, case.fcst3d, case.fcst2d, a, b)
    r = O.da_main(p, {k: v.numpy() for k, v in gl.items()}, ob, f3.numpy(), f2.numpy())
    a3, a2 = gather_columns(torch.from_numpy(r.anal3d), torch.from_numpy(r.anal2d), parts)
    if rank == 0:
        full = O.da_main(p, g, ob, case.fcst3d.numpy(), case.fcst2d.numpy())
        ok = np.array_equal(a3.numpy(), full.anal3d) and np.array_equal(a2.numpy(), full.anal2d)
        ok = ok and np.array_equal(ob["dep"], case.obs["dep"].numpy())
        with open(os.path.join(outdir, "result"), "w") as f:
            f.write("ok" if ok else "mismatch")
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_split_equals_single_domain(tmp_path):
    mp.spawn(_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    assert (tmp_path / "result").read_text() == "ok"
