"""CPU, world size 2 (gloo): the multi-rank plumbing of independent solves.

bench.py deals the 64 independent systems of the batching form to the ranks
with dist.deal_balanced (by size), gives each rank a contiguous block of the
32 right-hand sides with dist.column_block, and gathers the per-unit results
with dist.merge_results; device times are reduced with max_over_ranks.  Here
the same functions run on gloo ranks, each rank solving its dealt systems
with the oracle (the product's solve needs a GPU).  Checks: the dealing is a
partition and balanced, every rank sees the same merged results and reduced
numbers, and the merged per-system results equal a single-process run."""
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
    systems = [6, 11, 7, 9, 10, 8]      # idim of six independent systems
    mine = mdist.deal_balanced([d ** 3 for d in systems], world)[rank]
    results = []
    t_rank = 0.0
    for i in mine:
        a = orc.gen_pde3d(systems[i], 1, ISO)
        p = orc.Prec(orc.default_params(smoother=orc.BJAC, coarse_sweeps=4, min_coarse_size=50))
        p.build(a)
        b = orc.spmv(a, np.ones(a.nrows))
        x, it, rr, _ = orc.krylov("FCG", a, p, b, eps=1e-10)
        results.append((it, float(rr)))
        t_rank += 1.0 + rank  # stand-in device time: rank 1 is "slower"
    merged = mdist.merge_results(mine, results, len(systems))
    lo, hi = mdist.column_block(32, rank, world)
    cols = mdist.merge_results(list(range(lo, hi)), [rank] * (hi - lo), 32)
    dist.barrier()
    t_max = mdist.max_over_ranks(t_rank)
    n_done = mdist.sum_over_ranks(len(mine))
    out.put((rank, mine, merged, t_max, n_done, cols))
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
    got.sort(key=lambda g: g[0])
    systems = [6, 11, 7, 9, 10, 8]
    owned = sorted(sum((g[1] for g in got), []))
    assert owned == list(range(len(systems)))           # a partition of the batch
    loads = [sum(systems[i] ** 3 for i in g[1]) for g in got]
    assert max(loads) <= 0.6 * sum(loads)               # balanced by size
    assert all(g[2] == got[0][2] for g in got)          # every rank sees the same merged list
    assert all(g[3] == got[0][3] for g in got)          # every rank sees the same max
    assert got[0][3] == max(len(g[1]) * (1.0 + g[0]) for g in got)
    assert all(g[4] == len(systems) for g in got)
    assert got[0][5] == [0] * 16 + [1] * 16             # column blocks of the 32 right-hand sides
    # merged per-system results equal a single-process run
    from conftest import ISO
    for i, idim in enumerate(systems):
        a = orc.gen_pde3d(idim, 1, ISO)
        p = orc.Prec(orc.default_params(smoother=orc.BJAC, coarse_sweeps=4, min_coarse_size=50))
        p.build(a)
        x, it, rr, _ = orc.krylov("FCG", a, p, orc.spmv(a, np.ones(a.nrows)), eps=1e-10)
        assert got[0][2][i] == (it, float(rr))


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
    # the batching form's 64 systems (idim 24..96, seed 1) dealt by size
    dims = [int(v) for v in np.random.default_rng(1).integers(24, 97, 64)]
    for world in (1, 2, 4, 8):
        deal = mdist.deal_balanced([d ** 3 for d in dims], world)
        assert sorted(sum(deal, [])) == list(range(64))
        loads = [sum(dims[i] ** 3 for i in p) for p in deal]
        assert max(loads) - min(loads) <= max(d ** 3 for d in dims)
        blocks = [mdist.column_block(32, r, world) for r in range(world)]
        assert blocks[0][0] == 0 and blocks[-1][1] == 32
        assert all(blocks[r][1] == blocks[r + 1][0] for r in range(world - 1))
    assert mdist.merge_results([2, 0, 1], ["c", "a", "b"], 3) == ["a", "b", "c"]
    with pytest.raises(ValueError):
        mdist.merge_results([0, 0], [1, 2], 2)
