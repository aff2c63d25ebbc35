"""CPU, world size 2 (gloo): the multi-rank plumbing of independent solves.

Each rank solves its own share of a batch of independent systems with the
oracle (the product's solve needs a GPU), then the ranks reduce their device
times with MAX and their solve counts with SUM, exactly as bench.py does
with NCCL.  Checks: the shards partition the batch, every rank sees the same
reduced numbers, and the per-system results equal a single-process run."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import datetime

    import torch.distributed as dist
    from conftest import ISO, load_package
    import oracle as orc
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    mld = load_package()
    from mld2p4_2_b200 import dist as mdist
    systems = [6, 7, 8, 9, 10]          # idim of five independent systems
    mine = mdist.shard(systems, rank, world)
    res = {}
    t_rank = 0.0
    for idim in mine:
        a = orc.gen_pde3d(idim, 1, ISO)
        p = orc.Prec(orc.default_params(smoother=orc.BJAC, coarse_sweeps=4, min_coarse_size=50))
        p.build(a)
        b = orc.spmv(a, np.ones(a.nrows))
        x, it, rr, _ = orc.krylov("FCG", a, p, b, eps=1e-10)
        res[idim] = (it, float(np.abs(x - 1).max()))
        t_rank += 1.0 + rank  # stand-in device time: rank 1 is "slower"
    dist.barrier()
    t_max = mdist.max_over_ranks(t_rank)
    n_done = mdist.sum_over_ranks(len(mine))
    out.put((rank, mine, res, t_max, n_done))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_independent_solves_world2(orc):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got.sort()
    owned = sorted(sum((g[1] for g in got), []))
    assert owned == [6, 7, 8, 9, 10]                    # a partition of the batch
    assert got[0][1] == [6, 8, 10] and got[1][1] == [7, 9]
    assert all(g[3] == got[0][3] for g in got)          # every rank sees the same max
    assert got[0][3] == max(len(g[1]) * (1.0 + g[0]) for g in got)
    assert all(g[4] == 5 for g in got)
    # per-system results equal a single-process run
    from conftest import ISO
    for rank, mine, res, _, _ in got:
        for idim in mine:
            a = orc.gen_pde3d(idim, 1, ISO)
            p = orc.Prec(orc.default_params(smoother=orc.BJAC, coarse_sweeps=4, min_coarse_size=50))
            p.build(a)
            x, it, rr, _ = orc.krylov("FCG", a, p, orc.spmv(a, np.ones(a.nrows)), eps=1e-10)
            assert res[idim][0] == it


def test_shard_helpers(mld):
    from mld2p4_2_b200 import dist as mdist
    units = list(range(64))
    parts = [mdist.shard(units, r, 8) for r in range(8)]
    assert sorted(sum(parts, [])) == units
    assert all(len(p) == 8 for p in parts)
    assert mdist.owner(13, 8) == 5
    assert mdist.job_throughput(3, 8, 1000.0) == 24.0
    with pytest.raises(ValueError):
        mdist.shard(units, 8, 8)
