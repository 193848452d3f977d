"""The multi-process slicing run on the GPU: pevsl_b200.distributed.
solve_interval_distributed with two ranks (gloo process group, host
buffers), both on cuda:0.  The one exchange of the path, the all-reduce of
the KPM moments and count (SRC/kpmdos.c:160-176), runs through the
library's group-reduction callback; the ranks then solve their own shares of
the slices (pEVSL_Part1d) and rank 0 gathers them.  The ranks never wait on
each other inside a kernel: the only synchronisation is the host-side
all-reduce and gather.

Checked against one process running pevsl_b200.solve_interval on the same
inputs: moments within 1e-13 relative (the Gaussian stream draws exactly
each rank's share of the one-process vectors), slice ends within 1e-12,
identical per-slice counts, filter degrees and Lanczos steps, eigenvalues
within 1e-10 relative, residuals <= 1e-8.
"""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

GRID = (20, 20, 20)
SPEC = dict(a_lo=0.6, b_hi=1.2, nslices=5, bounds_mode=1, Mdeg=300, nvec=60, rng_mode=1, seed=0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        import pevsl_b200 as pv
        from pevsl_b200.distributed import GroupReduce, solve_interval_distributed
        from pevsl_b200.problems import laplacian
        assert pv.load().pEVSL_B200_SetDevice(0) == 0
        n, ia, ja, a = laplacian(*GRID)
        M = pv.Matrix.from_csr(n, ia, ja, a)
        red = GroupReduce()

        def gather(obj):
            out = [None] * world
            dist.all_gather_object(out, obj)
            return out
        r = solve_interval_distributed(M, pv.SliceRun(**SPEC), rank, world, red, gather)
        M.free()
        q.put(dict(rank=rank, calls=red.calls, res=None if r is None else dict(
            status=r.status, mu=r.mu, sli=r.sli, deg=r.deg, nev=r.nev, its=r.its, lam=r.lam,
            res=r.res, ecount=r.ecount)))
    except Exception as e:  # reported to the parent, which fails the test
        q.put(dict(rank=rank, error=repr(e)))
    finally:
        dist.destroy_process_group()


def test_distributed_solve_matches_one_process(gpu):
    import pevsl_b200 as pv
    from pevsl_b200.problems import laplacian
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for g in got:
        assert "error" not in g, g
        assert g["calls"] == 1  # one all-reduce of the moments per rank
    d = next(g["res"] for g in got if g["rank"] == 0)

    n, ia, ja, a = laplacian(*GRID)
    M = pv.Matrix.from_csr(n, ia, ja, a)
    one = pv.solve_interval(M, pv.SliceRun(**SPEC), batched=True)
    M.free()
    assert d["status"] == 0 and one.status == 0
    assert np.max(np.abs(d["mu"] - one.mu)) <= 1e-13 * np.max(np.abs(one.mu))
    assert abs(d["ecount"] - one.ecount) <= 1e-12 * abs(one.ecount)
    assert np.max(np.abs(d["sli"] - one.sli)) <= 1e-12 * np.max(np.abs(one.sli))
    assert list(d["nev"]) == list(one.nev)
    assert list(d["deg"]) == list(one.deg) and list(d["its"]) == list(one.its)
    for la, lb, rs in zip(d["lam"], one.lam, d["res"]):
        assert np.max(np.abs(la - lb)) <= 1e-10 * np.max(np.abs(lb))
        assert np.all(rs < 1e-8) and np.all(rs / np.abs(la) <= 1e-8)
