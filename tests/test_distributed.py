"""Ensembles across ranks (world size 2, gloo on CPU): each rank takes its
shard of the models with no data-path collective; the only communication is
the final gather of per-rank statistics, which must cover every model once.
The per-model work here is the oracle's pressure solve (CPU), standing in for
the GPU solve so that the rank logic runs without a GPU."""
import os
import socket

import numpy
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import torch
    from oracle.oracle import OracleModel
    from transportse_b200 import workloads
    from transportse_b200.ensemble import shard
    shapes = [(6, 5, 4), (8, 3, 5), (5, 5, 5), (7, 4, 6), (4, 4, 9)]
    cfgs = [workloads.ensemble_member(seed=50 + i, shape=s) for i, s in enumerate(shapes)]
    mine = shard([c.nx * c.ny * c.nz for c in cfgs], rank, world)
    res = {}
    for i in mine:
        c = cfgs[i]
        m = OracleModel(c)
        z = numpy.zeros(c.P.shape)
        r = m.compute_P(c.P, c.c_f, c.nue, c.rho_f, c.phi, c.Kx, c.Ky, c.Kz, z, z, z, 600.0,
                        c.BP, c.WP, SOR=1.7, max_it=20000, inc_it=1.25, max_dt=1e5,
                        P_conv=1e-10)
        res[i] = (r[5], float(numpy.abs(r[2]).sum()))
    t = torch.zeros(len(cfgs), 2, dtype=torch.float64)
    for i, (it, s) in res.items():
        t[i, 0], t[i, 1] = it, s
    gathered = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(gathered, t)
    if rank == 0:
        torch.save(gathered, os.path.join(out_dir, "gathered.pt"))
    dist.barrier()
    dist.destroy_process_group()


def test_ensemble_shards_over_two_gloo_ranks(tmp_path):
    import torch
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    g = torch.load(os.path.join(tmp_path, "gathered.pt"))
    covered = (g[0][:, 0] > 0).int() + (g[1][:, 0] > 0).int()
    assert covered.tolist() == [1] * 5     # every model on exactly one rank
    # the same solve on one process gives the same answer
    from oracle.oracle import OracleModel
    from transportse_b200 import workloads
    c = workloads.ensemble_member(seed=52, shape=(5, 5, 5))
    z = numpy.zeros(c.P.shape)
    r = OracleModel(c).compute_P(c.P, c.c_f, c.nue, c.rho_f, c.phi, c.Kx, c.Ky, c.Kz, z, z, z,
                                 600.0, c.BP, c.WP, SOR=1.7, max_it=20000, inc_it=1.25,
                                 max_dt=1e5, P_conv=1e-10)
    row = g[0][2] + g[1][2]
    assert int(row[0]) == r[5] and float(row[1]) == float(numpy.abs(r[2]).sum())
