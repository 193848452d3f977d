"""One process per GPU: the reference's group decomposition (TESTS/Lap/
LapPLanN.c with ngroups; SRC/kpmdos.c:97-102,160-176) over a
torch.distributed process group.

The path has one exchange: the KPM random vectors are shared out over the
ranks (pEVSL_Part1d) and the moments and count are summed across them -- a
single all-reduce of Mdeg + 2 doubles, installed into the library as the
instance's group reduction (pEVSL_B200_SetGroupReduce).  Everything else is
independent: every rank computes the same bounds and slices, then solves its
own contiguous share of the slices; rank 0 gathers the results.  The
all-reduce runs on the group's backend (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import (PevslData, SliceResult, Instance, Matrix, Vector, findpol, load, set_rng,
               spslicer_kpm, cheblannr_batch)

REDUCE_FN = C.CFUNCTYPE(None, C.POINTER(C.c_double), C.c_int, C.c_void_p)


def part1d(n: int, nparts: int, part: int):
    """[start, end) of part `part` of n items split into nparts contiguous
    pieces, the first n % nparts one longer: the library's pEVSL_Part1d
    (SRC/utils.c:128-149), which pEVSL_Kpmdos uses for the vectors."""
    idx, j1, j2 = C.c_int(part), C.c_int(), C.c_int()
    load().pEVSL_Part1d(n, nparts, C.byref(idx), C.byref(j1), C.byref(j2), 1)
    return j1.value, j2.value


class GroupReduce:
    """The cross-rank sum of a buffer of doubles on a torch.distributed group,
    as a C callback for pEVSL_B200_SetGroupReduce."""

    def __init__(self, group=None, device=None):
        import torch
        import torch.distributed as dist
        self.dist, self.torch, self.group = dist, torch, group
        if device is None:
            backend = dist.get_backend(group)
            device = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" \
                else torch.device("cpu")
        self.device = device
        self.calls = 0

        def _cb(buf, count, ctx):
            a = np.ctypeslib.as_array(buf, shape=(count,))
            t = self.torch.from_numpy(a.copy()).to(self.device)
            self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
            a[:] = t.cpu().numpy()
            self.calls += 1

        self._py = _cb
        self.fn = REDUCE_FN(_cb)

    def sum_inplace(self, a: np.ndarray):
        """The callback on a numpy buffer (what the library calls)."""
        a = np.ascontiguousarray(a, dtype=np.float64)
        self.fn(a.ctypes.data_as(C.POINTER(C.c_double)), a.size, None)
        return a

    def install(self, ev: Instance):
        load().pEVSL_B200_SetGroupReduce(ev.p, C.cast(self.fn, C.c_void_p), None)

    def remove(self, ev: Instance):
        load().pEVSL_B200_SetGroupReduce(ev.p, None, None)


def kpmdos_groups(ev: Instance, Mdeg, damping, nvec, intv, reduce: GroupReduce, rank, world):
    """pEVSL_Kpmdos with the vectors shared out over the ranks and summed by
    `reduce`: every rank returns the moments of all nvec vectors."""
    reduce.install(ev)
    try:
        return ev.kpmdos(Mdeg, damping, nvec, intv, ngroups=world, groupid=rank)
    finally:
        reduce.remove(ev)


def solve_interval_distributed(A: Matrix, s, rank: int, world: int, reduce: GroupReduce | None,
                               gather=None) -> SliceResult | None:
    """The slicing run of pevsl_b200.solve_interval over `world` ranks: the
    KPM vectors split across the ranks (summed through `reduce`), the slices
    in contiguous shares; `gather(obj) -> list` (e.g. all_gather_object)
    brings the per-slice results to every rank, rank 0 returns them in a
    SliceResult (other ranks: None)."""
    lib = load()
    set_rng(s.rng_mode, s.seed)
    with Instance(A) as ev:
        set_rng(s.rng_mode, s.seed)
        vinit = Vector(A.n)
        lib.pEVSL_ParvecRand(C.byref(vinit.pv))
        if s.bounds_mode == 1:
            lo, hi = C.c_double(), C.c_double()
            r = lib.pEVSL_LanTrbounds(ev.p, s.lan_lanm, s.lan_maxit, s.lan_tol, C.byref(vinit.pv),
                                      s.lan_bndtype, C.byref(lo), C.byref(hi), None)
            if r:
                raise RuntimeError(f"pEVSL_LanTrbounds returned {r}")
            lmin, lmax = lo.value, hi.value
        else:
            lmin, lmax = s.lmin, s.lmax
        intv = [s.a_lo, s.b_hi, lmin, lmax]
        if world > 1 and reduce is not None:
            r, mu, ecount = kpmdos_groups(ev, s.Mdeg, s.kpm_damping, s.nvec, intv, reduce, rank, world)
        else:
            r, mu, ecount = ev.kpmdos(s.Mdeg, s.kpm_damping, s.nvec, intv)
        if r:
            raise RuntimeError(f"pEVSL_Kpmdos returned {r}")
        npts = int(10 * ecount)
        r, sli = spslicer_kpm(mu, s.Mdeg, intv, s.nslices, npts)
        if r:
            raise RuntimeError(f"pEVSL_SpslicerKpm returned {r}")
        s0, s1 = part1d(s.nslices, world, rank)
        nev = int(1 + ecount / float(s.nslices)) + 2
        mlan = min(max(5 * nev, s.mlan_min), A.n)
        mine = []
        if s1 > s0:
            intvs, filters = [], []
            for sl in range(s0, s1):
                iv = [sli[sl], sli[sl + 1], lmin, lmax]
                r, f = findpol(iv, s.pol_max_deg, s.pol_damping, s.thresh_int, s.thresh_ext)
                if r:
                    raise RuntimeError(f"pEVSL_FindPol returned {r}")
                filters.append(f)
                intvs.append(iv)
            r, outs = cheblannr_batch(ev, intvs, [mlan] * len(filters), s.tol, vinit, filters)
            for sl, f, o in zip(range(s0, s1), filters, outs):
                mine.append(dict(slice=sl, deg=f.deg, nev=o["nev"], its=o["its"],
                                 lam=o.get("lam", np.zeros(0)), res=o.get("res", np.zeros(0)),
                                 status=o["status"]))
        vinit.free()
    parts = gather(mine) if gather is not None else [mine]
    if rank != 0:
        return None
    res = SliceResult(lmin, lmax, ecount, npts, 0, np.asarray(mu), np.asarray(sli))
    for d in sorted((d for p in parts for d in p), key=lambda d: d["slice"]):
        res.deg.append(d["deg"])
        res.nev.append(d["nev"])
        res.its.append(d["its"])
        res.lam.append(d["lam"])
        res.res.append(d["res"])
        if d["status"] and not res.status:
            res.status = 300 + abs(d["status"])
    return res


__all__ = ["GroupReduce", "kpmdos_groups", "part1d", "solve_interval_distributed", "PevslData"]
