"""The multi-process layer on CPU (gloo, world size 2): the group reduction
callback that replaces the reference's MPI_Allreduce of the KPM moments
(SRC/kpmdos.c:160-176), and the sharing of vectors and slices by
pEVSL_Part1d.  No GPU: the library is only loaded for its host functions."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from pevsl_b200.distributed import GroupReduce, part1d
        red = GroupReduce()
        buf = np.arange(302, dtype=np.float64) * (rank + 1)
        out = red.sum_inplace(buf.copy())
        shares = [part1d(60, world, r) for r in range(world)]
        gathered = [None] * world
        dist.all_gather_object(gathered, dict(rank=rank, share=part1d(60, world, rank)))
        q.put(dict(rank=rank, out=out, calls=red.calls, shares=shares, gathered=gathered))
    finally:
        dist.destroy_process_group()


def test_group_reduce_sums_across_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = np.arange(302, dtype=np.float64) * 3  # 1x + 2x
    for r in res:
        assert np.array_equal(r["out"], want)
        assert r["calls"] == 1
        # the shares tile the 60 vectors, in rank order, every rank agreeing
        assert r["shares"] == [(0, 30), (30, 60)]
        assert [g["share"] for g in r["gathered"]] == r["shares"]


@pytest.mark.parametrize("n,parts", [(60, 4), (10, 4), (2, 4), (7, 1), (30, 8)])
def test_part1d_tiles(n, parts):
    from pevsl_b200.distributed import part1d
    spans = [part1d(n, parts, p) for p in range(parts)]
    assert spans[0][0] == 0 and spans[-1][1] == n
    assert all(spans[i][1] == spans[i + 1][0] for i in range(parts - 1))
    sizes = [b - a for a, b in spans]
    assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)
