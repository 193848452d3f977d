#!/usr/bin/env python
"""Eigenpairs/s of pEVSL's spectrum-slicing path on B200 (one process per GPU).

A step is one whole run of the path on the workload (bounds by thick-restart
Lanczos, KPM density of states, slicing, then filtered Lanczos on every
slice), through the C-ABI library libpevsl_b200.so:

  value : matrix resident in HBM; device time (CUDA events on the library
          stream) of K steps after W warm-up steps; eigenpairs accepted at
          residual <= 1e-8 per second, summed over ranks / max rank time.
  e2e   : the same through the public API from pinned host buffers: every step
          uploads the CSR (pEVSL_ParcsrSetup), solves, reads the eigenvalues and
          residuals back, frees the matrix.

Default workload (the metric's configuration): 3D 7-point Laplacian
100^3 (n = 1e6, nnz = 6.94e6), interval [0.80, 0.82], 4 slices, KPM Mdeg 300
with 30 seeded Gaussian vectors, tol 1e-8.  With N > 1 GPUs every rank
solves its own copy with its own seed (weak scaling, no collective on the
data path); rank 0 prints the JSON line.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")

import numpy as np  # noqa: E402

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "lap100_4slices": dict(grid=(100, 100, 100), a=0.80, b=0.82, nslices=4, Mdeg=300, nvec=30),
    "lap20_5slices": dict(grid=(20, 20, 20), a=0.6, b=1.2, nslices=5, Mdeg=300, nvec=60),
    # 32 shifted 2D/3D Laplacians, n 1e4..5e5, 2..8 slices each (a count
    # interpretation of "~2% of the spectrum": 20 eigenvalues per slice)
    "lap_multi_32": dict(multi=True, count=32, seed=2024, per_slice=20),
    # the generalized problem of TESTS/Gen_Lap/LapPLanN.c scaled up: A the 3D
    # Laplacian, B the 1D Laplacian (diagonal 4) of the same size; B-solve
    # by the least-squares 1/x on [2, 6] (degree 24 at tol 1e-10, rounding
    # level), L^{-T} by the least-squares 1/sqrt(x) (max degree 50, 1e-6)
    "genlap24": dict(gen=True, grid=(24, 24, 24), a=1.0, b=1.0094, nslices=2, Mdeg=100, nvec=30,
                     bsol=("lsrec", 80, 1e-10), ltsol=("lssqrt", 50, 1e-6), brange=(2.0, 6.0)),
}
DEFAULT_WORKLOAD = "lap100_4slices"
METRIC = "eigenpairs/s at residual <= 1e-8 (3D Laplacian 100^3, [0.80,0.82], 4 slices, FP64)"


def metric_of(w):
    """The metric string of a single-problem workload."""
    g = w["grid"]
    if w.get("gen"):
        return (f"eigenpairs/s at ||A x - lam B x|| <= 1e-8 (A x = lam B x: A 3D Laplacian "
                f"{g[0]}^3, B 1D Laplacian, [{w['a']:.4f},{w['b']:.4f}], {w['nslices']} slices, "
                f"FP64)")
    return (f"eigenpairs/s at residual <= 1e-8 (3D Laplacian {g[0]}^3, [{w['a']:.2f},{w['b']:.2f}], "
            f"{w['nslices']} slices, FP64)")


class GenSetup:
    """B (1D Laplacian of the same size as A) on the device and the
    B-solvers of a generalized workload; install(ev) makes an instance
    generalized (pEVSL_SetBParcsr, SetBSol, SetLTSol, SetGenEig)."""

    def __init__(self, w, n, pinned=None):
        import pevsl_b200 as pv
        from pevsl_b200.problems import laplacian
        if pinned is None:
            _, ib, jb, b = laplacian(n, 1, 1)
        else:
            ib, jb, b = pinned
        self.B = pv.Matrix.from_csr(n, ib, jb, b)
        lo, hi = w["brange"]
        k, deg, tol = w["bsol"]
        self.bsol = pv.BSolver(self.B, k, lo, hi, deg, tol)
        k, deg, tol = w["ltsol"]
        self.ltsol = pv.BSolver(self.B, k, lo, hi, deg, tol)

    def install(self, ev):
        ev.set_generalized(self.B, self.bsol, self.ltsol)

    def free(self):
        self.bsol.free()
        self.ltsol.free()
        self.B.free()


def slice_run(w, seed):
    import pevsl_b200 as pv
    return pv.SliceRun(w["a"], w["b"], w["nslices"], bounds_mode=1, Mdeg=w["Mdeg"],
                       kpm_damping=1, nvec=w["nvec"], pol_damping=2, pol_max_deg=3000,
                       thresh_int=0.8, thresh_ext=0.2, tol=1e-8, rng_mode=pv.RNG_GAUSS, seed=seed)


# ---------------------------------------------------------------- distributed
class Dist:
    def __init__(self, n_gpus):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.dev = "cpu"
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            # the group carries host-side barriers and the ranks' timings only
            backend = os.environ.get("PEVSL_BENCH_BACKEND", "gloo")
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                self.dev = torch.device("cuda", self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples every 200 ms while the timed region runs."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.QUERY,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- helpers
def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic(workload):
    """dram bytes per launch of the fused filter kernel from the committed ncu
    summary (profiles/), or None."""
    path = os.path.join(ROOT, "profiles", "cheb_step_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        e = d.get(workload)
        return e.get("dram_bytes_per_launch") if e else None
    except (OSError, ValueError, AttributeError):
        return None


def cpu_reference_sample(n, ia, ja, a, fil, seconds_budget=30.0):
    """Time the reference's own pEVSL_ChebAv (oracle/_ref, compiled from the
    reference sources) on this matrix with one slice's filter, on one core.
    Returns seconds per filter degree (one SpMV + the recurrence's BLAS1)."""
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libpevsl_ref.so"))
    deg = fil.deg
    # bounded sample: enough degrees for ~seconds_budget at ~10 ms each
    mu = np.ascontiguousarray(fil.mu[: deg + 1])
    v = np.cos(np.arange(n) * 0.1)
    y = np.zeros(n)
    P = lambda x: x.ctypes.data_as(C.c_void_p)  # noqa: E731
    # probe: a short filter of degree 20 to estimate the per-degree time
    t = time.perf_counter()
    lib.oref_chebav(n, P(ia), P(ja), P(a), 20, C.c_double(fil.cc), C.c_double(fil.dd), P(mu), P(v),
                    P(y))
    per = (time.perf_counter() - t) / 20
    d = int(max(20, min(deg, seconds_budget / max(per, 1e-9))))
    t = time.perf_counter()
    lib.oref_chebav(n, P(ia), P(ja), P(a), d, C.c_double(fil.cc), C.c_double(fil.dd), P(mu), P(v),
                    P(y))
    return (time.perf_counter() - t) / d, d


def cpu_reference_gen_sample(w, n, ia, ja, a, fil, seconds_budget=30.0):
    """Time the reference's generalized pEVSL_ChebAv (oracle/_ref): per
    degree one B-solve (its least-squares polynomial, pEVSL_LSPolSol) and
    one A matvec, on one core.  Returns seconds per degree."""
    from pevsl_b200.problems import laplacian
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libpevsl_ref.so"))
    _, ib, jb, b = laplacian(n, 1, 1)
    mu = np.ascontiguousarray(fil.mu[: fil.deg + 1])
    v = np.cos(np.arange(n) * 0.1)
    y = np.zeros(n)
    P = lambda x: x.ctypes.data_as(C.c_void_p)  # noqa: E731
    k, lsdeg, lstol = w["bsol"]
    lo, hi = w["brange"]

    def run(d):
        t = time.perf_counter()
        lib.oref_gen_chebav(n, P(ia), P(ja), P(a), P(ib), P(jb), P(b), lsdeg, C.c_double(lstol),
                            C.c_double(lo), C.c_double(hi), d, C.c_double(fil.cc),
                            C.c_double(fil.dd), P(mu), P(v), P(y))
        return time.perf_counter() - t
    per = run(10) / 10
    d = int(max(10, min(fil.deg, seconds_budget / max(per, 1e-9))))
    return run(d) / d, d


# ---------------------------------------------------------------- our arm
def run_b200(args, dist):
    import pevsl_b200 as pv
    from pevsl_b200.problems import laplacian
    w = WORKLOADS[args.workload]
    pv.load()
    pv.load().pEVSL_B200_SetDevice(dist.local)
    lib = pv.load()
    n, ia, ja, a = laplacian(*w["grid"])
    nnz = int(ia[-1])
    distributed = args.mode == "distributed" and dist.world > 1 and not w.get("gen")
    # replicas: every rank its own seed; distributed: one problem, one seed
    seed = 0 if distributed else 1000 * dist.rank
    spec = slice_run(w, seed)
    reduce, gather = None, None
    if distributed:
        from pevsl_b200.distributed import GroupReduce

        reduce = GroupReduce()

        def gather(obj):
            out = [None] * dist.world
            dist.pg.all_gather_object(out, obj)
            return out
    # pinned host copies of the inputs: every step uploads them
    ia_p, p1 = pv.pinned_empty(n + 1, np.int32)
    ja_p, p2 = pv.pinned_empty(nnz, np.int32)
    a_p, p3 = pv.pinned_empty(nnz, np.float64)
    ia_p[:], ja_p[:], a_p[:] = ia, ja, a
    gen = bool(w.get("gen"))
    bpins = []
    if gen:
        _, ib, jb, bv = laplacian(n, 1, 1)
        bpins = [pv.pinned_empty(n + 1, np.int32), pv.pinned_empty(len(jb), np.int32),
                 pv.pinned_empty(len(jb), np.float64)]
        bpins[0][0][:], bpins[1][0][:], bpins[2][0][:] = ib, jb, bv
    batched = args.path == "batched"

    # One loop of W + K steps.  Every step goes through the public API from
    # pinned host memory: upload the CSR (pEVSL_ParcsrSetup; for the
    # generalized workload B and its solvers too), solve, read the
    # eigenvalues and residuals back, free the matrix.  `value` is the device
    # time of the solve alone (CUDA events on the library stream, the matrix
    # resident); `e2e` is the wall time of the whole step, copies included.
    # The L2 is flushed before every step, outside both clocks.
    eig = 0
    results = []
    ms = 0.0
    wall = 0.0
    d2h = 0
    clocks = ClockSampler(dist.local)
    for it in range(args.warmup + args.steps):
        timed = it >= args.warmup
        if it == args.warmup:
            dist.barrier()
            clocks.start()
            lib.pEVSL_B200_Sync()
            lib.pEVSL_B200_ResetFilterCounters()
            lib.pEVSL_B200_ResetGenCounters()
            l0 = pv.launch_count()
        lib.pEVSL_B200_FlushL2(0)
        lib.pEVSL_B200_Sync()
        t0 = time.perf_counter()
        M = pv.Matrix.from_csr(n, ia_p, ja_p, a_p)
        gs = GenSetup(w, n, (bpins[0][0], bpins[1][0], bpins[2][0])) if gen else None
        lib.pEVSL_B200_EventRecord(0)
        if distributed:
            from pevsl_b200.distributed import solve_interval_distributed
            r = solve_interval_distributed(M, spec, dist.rank, dist.world, reduce, gather)
        else:
            r = pv.solve_interval(M, spec, batched=batched, setup=gs.install if gen else None)
        lib.pEVSL_B200_EventRecord(1)
        step_ms = lib.pEVSL_B200_EventElapsedMs(0, 1)
        if gs:
            gs.free()
        M.free()
        lib.pEVSL_B200_Sync()
        step_wall = time.perf_counter() - t0
        if distributed:
            # rank 0 gathered every slice; the others count nothing
            nev = sum(r.nev) if r is not None else 0
        else:
            nev = sum(r.nev)
        if timed:
            ms += step_ms
            wall += step_wall
            if r is not None:
                results.append(r)
                d2h += sum(len(x) for x in r.lam) * 16
            eig += nev
        print(f"[bench] {'step' if timed else 'warmup'} {it + 1}/{args.warmup + args.steps}: "
              f"{nev} eigenpairs, solve {step_ms / 1e3:.2f} s, step {step_wall:.2f} s",
              file=sys.stderr, flush=True)
    clk = clocks.stop()
    launches = pv.launch_count() - l0
    f_launch, f_bytes, f_ms = pv.filter_counters()
    if gen:
        # the generalized filter: one "launch" is one filter degree (the
        # B-solve's fused degrees on B and the fused A step), timed per
        # application (CUDA graph replays)
        _, f_launch, f_bytes, f_ms = pv.gen_counters()
    dist.barrier()
    t_max = dist.max(ms / 1e3)
    eig_all = dist.sum(float(eig))
    value = eig_all / t_max
    e2e_t = dist.max(wall)
    e2e_val = eig_all / e2e_t
    # roofline of the dominant kernel (fused Chebyshev filter degree)
    peak, peak_kind = measured_peak()
    per_launch_bytes = f_bytes / max(f_launch, 1)
    per_launch_ms = f_ms / max(f_launch, 1)
    achieved = per_launch_bytes / (per_launch_ms * 1e-3) / 1e9 if f_launch else None
    if not results:  # a distributed rank other than 0: rank 0 prints the line
        return None
    r0 = results[0]
    out = {
        "metric": metric_of(w),
        "value": value,
        "unit": "eigenpairs/s",
        "n_gpus": dist.world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_max * 1e3 / args.steps,
        "higher_is_better": True,
        "scaling": "strong" if distributed else "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": ("synthetic: 3D Dirichlet Laplacian A" + (" and 1D Laplacian B (diagonal 4)"
                 if gen else "") + " generated on the host, seeded Philox Gaussian random "
                 "vectors (" + ("seed 0, one problem over the ranks" if distributed else
                                "seed 1000*rank") + ")"),
        "config": {"workload": args.workload, "n": n, "nnz": nnz, "interval": [w["a"], w["b"]],
                   **({"problem": "generalized A x = lam B x (pEVSL_SetGenEig)",
                       "b_solve": "least-squares 1/x on [2, 6], pEVSL_SetupLSPolRec(80, 1e-10)",
                       "lt_solve": "least-squares 1/sqrt(x), pEVSL_SetupLSPolSqrt(50, 1e-6)"}
                      if gen else {}),
                   "nslices": w["nslices"], "kpm_mdeg": w["Mdeg"], "kpm_nvec": w["nvec"],
                   "bounds": "thick-restart Lanczos (50, 200, 1e-8)", "tol": 1e-8,
                   "precision": "fp64",
                   "path": ("all slices in lockstep (pEVSL_B200_ChebLanNrBatch), bit-identical to "
                            "the slice-by-slice drop-in path" if batched else
                            "slice by slice (pEVSL_ChebLanNr, the drop-in path)"),
                   "eigenpairs_per_step": sum(r0.nev), "nev_per_slice": r0.nev,
                   "lanczos_steps_per_slice": r0.its, "filter_degree_per_slice": r0.deg,
                   "l2": "256 MiB written between timed steps (L2 flush); within a step the "
                         "working set streams thousands of times",
                   "parallelism": (f"one problem over {dist.world} ranks: KPM vectors split "
                                   "and summed by one all-reduce, slices shared out "
                                   "(pevsl_b200.distributed)" if distributed else
                                   f"replicas x{dist.world}")},
        "gpu_launches": int(launches),
        "clocks": clk,
        "roofline": {
            "kernel": ("generalized filter degree (B-solve: fused Chebyshev degrees on B; A step "
                       "fused with the recurrence), CUDA-graph replays; one launch = one degree"
                       if gen else
                       "cheb_step_il (fused SpMV + Chebyshev recurrence, all slices per launch with "
                       "row-interleaved vectors in groups of two that stay in L2, filter sum updated "
                       "every third degree: k_cheb_il2_e on the ELL copy of the packed entries; one "
                       "live slice: k_cheb_il_e<1>), all filter launches of the timed steps"
                       if batched else "cheb_step (fused SpMV + Chebyshev recurrence, CSR-stream, "
                       "packed entries)"),
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak if achieved else None, "peak_source": peak_kind,
            "bytes_per_launch": per_launch_bytes, "launches": f_launch,
            "avg_launch_us": per_launch_ms * 1e3,
            "traffic": ncu_traffic(args.workload) if batched and not gen else None},
        "e2e": {"value": e2e_val, "unit": "eigenpairs/s",
                "h2d_bytes_per_step": int(4 * (n + 1) + 12 * nnz +
                                          (4 * (n + 1) + 12 * (3 * n - 2) if gen else 0)),
                "d2h_bytes_per_step": int(d2h // max(args.steps, 1)),
                "how": "same steps as value: wall time of upload from pinned memory + solve + "
                       "results to host + free, summed over the K timed steps"},
    }
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline and gen:
        try:
            r, fil = pv.findpol([r0.sli[0], r0.sli[1], r0.lmin, r0.lmax], 3000, 2, 0.8, 0.2)
            per, d = cpu_reference_gen_sample(w, n, ia, ja, a, fil)
            degs = sum(dg * (it + 1) for dg, it in zip(r0.deg, r0.its)) + w["Mdeg"] * w["nvec"] + 200
            out["cpu_baseline"] = {
                "value": sum(r0.nev) / (per * degs), "unit": "eigenpairs/s", "cores": 1,
                "kind": "reference",
                "sample": f"reference generalized pEVSL_ChebAv (oracle/_ref, least-squares B-solve, "
                          f"OpenBLAS 1 thread) of degree {d} with slice 0's filter: "
                          f"{per*1e3:.2f} ms per degree; extrapolated to this run's "
                          f"{degs} degrees (filters x Lanczos steps, KPM, <=200 bounds steps)"}
        except Exception as e:
            out["cpu_baseline"] = {"value": None, "unavailable": str(e)}
    elif dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        try:
            r, fil = pv.findpol([r0.sli[0], r0.sli[1], r0.lmin, r0.lmax], 3000, 2, 0.8, 0.2)
            per, d = cpu_reference_sample(n, ia, ja, a, fil)
            # whole-run CPU time: every slice's filter degrees (degree x
            # (Lanczos steps + 1), the reference's pEVSL_ChebAv calls) and every
            # KPM / bounds SpMV at the measured per-degree cost
            # (reorthogonalisation, ~1-2% of the reference's time on this
            # workload, not counted)
            kpm = w["Mdeg"] * w["nvec"]
            slice_degs = sum(dg * (it + 1) for dg, it in zip(r0.deg, r0.its))
            cpu_t = per * (slice_degs + kpm + 200)
            out["cpu_baseline"] = {
                "value": sum(r0.nev) / cpu_t, "unit": "eigenpairs/s", "cores": 1,
                "kind": "reference",
                "sample": f"reference pEVSL_ChebAv (oracle/_ref, OpenBLAS 1 thread) of degree {d} "
                          f"with slice 0's filter on this matrix: {per*1e3:.2f} ms per degree; "
                          f"extrapolated to the run's {slice_degs} slice filter degrees + "
                          f"{kpm} KPM + <=200 bounds matvecs"}
        except Exception as e:  # the baseline is reported, never required
            out["cpu_baseline"] = {"value": None, "unavailable": str(e)}
    for p in [p1, p2, p3] + [bp[1] for bp in bpins]:
        pv.free_pinned(p)
    return out


def run_b200_multi(args, dist):
    """The batched-problem workload: 32 independent Laplacians (problems.
    multi_laplacian_set), every slice of every problem solved; batched = all
    slices of all problems in lockstep (pEVSL_B200_ChebLanNrMulti), plain =
    one pEVSL_ChebLanNr per slice.  Spectrum bounds and slices come from the
    analytic spectrum (the workload's definition), the start vectors are
    seeded Gaussian."""
    import pevsl_b200 as pv
    from pevsl_b200.problems import laplacian_shifted, multi_laplacian_set
    w = WORKLOADS[args.workload]
    lib = pv.load()
    lib.pEVSL_B200_SetDevice(dist.local)
    P = multi_laplacian_set(w["count"], w["seed"] + 7919 * dist.rank, w["per_slice"])
    host, probs = [], []
    for i, p in enumerate(P):
        n, ia, ja, a = laplacian_shifted(*p["grid"], p["shift"])
        pins = [pv.pinned_empty(n + 1, np.int32), pv.pinned_empty(len(ja), np.int32),
                pv.pinned_empty(len(ja), np.float64)]
        pins[0][0][:], pins[1][0][:], pins[2][0][:] = ia, ja, a
        intvs = [[p["intv"][k], p["intv"][k + 1], p["lmin"], p["lmax"]] for k in range(p["nslices"])]
        fl = [pv.findpol(iv, max_deg=8000)[1] for iv in intvs]
        maxits = [max(5 * (c + 2), 150) for c in p["counts"]]
        v = np.random.default_rng(100 + i + 7919 * dist.rank).standard_normal(n)
        host.append((n, pins, intvs, fl, maxits, v))
    batched = args.path == "batched"

    def solve(mats):
        eig = 0
        if batched:
            insts = [pv.Instance(M) for M in mats]
            r, outs = pv.cheblannr_multi([(ev, h[2], h[4], 1e-8, h[5], h[3])
                                          for ev, h in zip(insts, host)])
            eig = sum(o["nev"] for per in outs for o in per)
            for ev in insts:
                ev.close()
        else:
            for M, h in zip(mats, host):
                with pv.Instance(M) as ev:
                    for k, iv in enumerate(h[2]):
                        eig += ev.cheblannr(iv, h[4][k], 1e-8, h[5], h[3][k])["nev"]
        return eig

    # one loop of W + K steps, each from pinned host memory: upload the 32
    # matrices, solve (device time between CUDA events), results to host,
    # free; e2e is the wall time of the same steps
    clocks = ClockSampler(dist.local)
    eig, ms, wall, h2d = 0, 0.0, 0.0, 0
    for it in range(args.warmup + args.steps):
        timed = it >= args.warmup
        if it == args.warmup:
            dist.barrier()
            clocks.start()
            lib.pEVSL_B200_Sync()
            lib.pEVSL_B200_ResetFilterCounters()
            l0 = pv.launch_count()
        lib.pEVSL_B200_FlushL2(0)
        lib.pEVSL_B200_Sync()
        t0 = time.perf_counter()
        mats = [pv.Matrix.from_csr(h[0], h[1][0][0], h[1][1][0], h[1][2][0]) for h in host]
        lib.pEVSL_B200_EventRecord(0)
        e = solve(mats)
        lib.pEVSL_B200_EventRecord(1)
        step_ms = lib.pEVSL_B200_EventElapsedMs(0, 1)
        for M in mats:
            M.free()
        lib.pEVSL_B200_Sync()
        step_wall = time.perf_counter() - t0
        if timed:
            eig += e
            ms += step_ms
            wall += step_wall
            h2d += sum(4 * (h[0] + 1) + 12 * len(h[1][1][0]) for h in host)
        print(f"[bench] {'step' if timed else 'warmup'} {it + 1}/{args.warmup + args.steps}: "
              f"{e} eigenpairs, solve {step_ms / 1e3:.2f} s, step {step_wall:.2f} s",
              file=sys.stderr, flush=True)
    clk = clocks.stop()
    launches = pv.launch_count() - l0
    f_launch, f_bytes, f_ms = pv.filter_counters()
    dist.barrier()
    t_max = dist.max(ms / 1e3)
    value = dist.sum(float(eig)) / t_max
    e2e_eig = eig
    e2e_t = dist.max(wall)
    peak, peak_kind = measured_peak()
    per_launch_bytes = f_bytes / max(f_launch, 1)
    per_launch_ms = f_ms / max(f_launch, 1)
    achieved = per_launch_bytes / (per_launch_ms * 1e-3) / 1e9 if f_launch else None
    out = {
        "metric": "eigenpairs/s at residual <= 1e-8 (32 shifted 2D/3D Laplacians, n 1e4..5e5, "
                  "2..8 slices each, FP64)",
        "value": value, "unit": "eigenpairs/s", "n_gpus": dist.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: seeded shifted Laplacians generated on the host, seeded Gaussian "
                "start vectors",
        "config": {"workload": args.workload, "problems": len(P),
                   "slices": sum(p["nslices"] for p in P),
                   "rows": [p["n"] for p in P], "eigenpairs_per_step": eig // max(args.steps, 1),
                   "interval": "starts 0.5% of the spectral width above the bottom, 20 "
                               "eigenvalues per slice",
                   "path": ("all slices of all problems in lockstep (pEVSL_B200_ChebLanNrMulti)"
                            if batched else "one pEVSL_ChebLanNr per slice (the drop-in path)"),
                   "l2": "working set far above the 126 MB L2 (25 GB of Lanczos bases)",
                   "parallelism": f"replicas x{dist.world}"},
        "gpu_launches": int(launches), "clocks": clk,
        "roofline": {"kernel": "one filter degree for every live slice: cheb_step_il per problem "
                               "(interleaved slices, n >= 2^16), cheb_step_batch for the rest",
                     "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if achieved else None, "peak_source": peak_kind,
                     "bytes_per_launch": per_launch_bytes, "launches": f_launch,
                     "avg_launch_us": per_launch_ms * 1e3, "traffic": None},
        "e2e": {"value": dist.sum(float(e2e_eig)) / e2e_t, "unit": "eigenpairs/s",
                "h2d_bytes_per_step": int(h2d // max(args.steps, 1)),
                "d2h_bytes_per_step": int(16 * e2e_eig // max(args.steps, 1))},
        "cpu_baseline": {"value": None, "unavailable": "the reference CPU path is timed on the "
                         "default workload (lap100_4slices)"},
    }
    for h in host:
        for p_ in h[1]:
            pv.free_pinned(p_[1])
    return out


# ---------------------------------------------------------------- reference arm
def _ref_slice_worker(q, n, ia, ja, a, deg, cc, dd, mu, budget):
    os.environ["OPENBLAS_NUM_THREADS"] = "1"

    class F:
        pass
    f = F()
    f.deg, f.cc, f.dd, f.mu = deg, cc, dd, mu
    q.put(cpu_reference_sample(n, ia, ja, a, f, budget))


def ref_golden(workload):
    """The reference build's own run of a workload (tests/golden, written by
    tests/golden/make_golden.py from oracle/_ref on the same inputs: seeded
    Gaussian vectors, thick-restart bounds, KPM, slicing, ChebLanNr): its
    bounds, slice ends and per-slice filter degrees, Lanczos steps and
    accepted counts, or None when the fixture is absent."""
    name, key = {"lap100_4slices": ("lap100_c2.json", None),
                 "lap20_5slices": ("pipelines.json", "lap20_lantr_gauss")}.get(workload, (None, None))
    if name is None:
        return None
    try:
        with open(os.path.join(ROOT, "tests", "golden", name)) as f:
            g = json.load(f)
    except OSError:
        return None
    g = g[key] if key else g
    return {k: g[k] for k in ("lmin", "lmax", "sli", "deg", "its", "nev")} | {
        "eigenpairs": int(sum(g["nev"])), "seconds_per_slice": g.get("seconds_per_slice"),
        "fixture": name + (f":{key}" if key else "")}


def reference_sample_seconds(warmup, steps):
    """Seconds of the reference's pEVSL_ChebAv each slice process runs per
    step of the reference arm: 180 s over all steps, between 2 and 20 s."""
    return min(20.0, max(2.0, 180.0 / max(1, warmup + steps)))


def run_reference(args, dist):
    """The reference's own CPU code (oracle/_ref, compiled from its sources)
    on this workload, one process per slice as the reference's MPI groups.
    A step times a bounded sample: each process runs the reference's
    pEVSL_ChebAv with its slice's filter (pEVSL_FindPol on the reference's
    own slice ends) for 180 s / (warm-up + timed steps), between 2 and 20 s,
    so that the whole arm ends within about four minutes at any step count
    (the driver's 25 steps: about 7 s each); the time of the whole run is
    extrapolated from it to the per-slice filter degrees and Lanczos steps
    of the reference's own run of the workload (ref_golden)."""
    if dist.rank != 0:
        return None
    w = WORKLOADS[args.workload]
    if w.get("gen") or w.get("multi"):
        return {"impl": "reference", "unavailable": "the reference arm times the single-problem "
                "Laplacian workloads (lap100_4slices, lap20_5slices)"}
    g = ref_golden(args.workload)
    if g is None:
        return {"impl": "reference", "unavailable": "the reference build's run of this workload "
                "(tests/golden) is missing"}
    import multiprocessing as mp

    from pevsl_b200.problems import laplacian
    n, ia, ja, a = laplacian(*w["grid"])
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libpevsl_ref.so"))
    P = lambda x: x.ctypes.data_as(C.c_void_p)  # noqa: E731

    def ref_findpol(intv, max_deg=3000, damping=2, thresh_int=0.8, thresh_ext=0.2):
        """the reference's own pEVSL_SetPolDef + pEVSL_FindPol (this arm
        runs none of the library's code)"""
        iv = np.ascontiguousarray(intv, dtype=np.float64)
        mu = np.zeros(max_deg + 1)
        t, d = C.c_int(), C.c_int()
        gam, bar, cc, dd = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        r = lib.oref_findpol(P(iv), max_deg, damping, C.c_double(thresh_int),
                             C.c_double(thresh_ext), 0, C.byref(t), C.byref(d), C.byref(gam),
                             C.byref(bar), C.byref(cc), C.byref(dd), P(mu))
        if r:
            raise RuntimeError(f"reference pEVSL_FindPol returned {r} for {list(intv)}")
        return d.value, cc.value, dd.value, np.ascontiguousarray(mu[: d.value + 1])
    nsl = w["nslices"]
    sli = g["sli"]
    filters = [ref_findpol([sli[s], sli[s + 1], g["lmin"], g["lmax"]]) for s in range(nsl)]
    assert [f[0] for f in filters] == g["deg"], "filter degrees differ from the reference run"
    cores = min(os.cpu_count() or 1, nsl)
    ctx = mp.get_context("spawn")
    times, per = [], []
    sample_target = reference_sample_seconds(args.warmup, args.steps)
    for it in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        q = ctx.Queue()
        procs = []
        for s in range(nsl):
            deg, cc, dd, mu = filters[s]
            p = ctx.Process(target=_ref_slice_worker,
                            args=(q, n, ia, ja, a, deg, cc, dd, mu, sample_target))
            p.start()
            procs.append(p)
        per = [q.get() for _ in procs]
        for p in procs:
            p.join()
        if it >= args.warmup:
            times.append(time.perf_counter() - t0)
    per_deg = float(np.mean([x[0] for x in per]))
    kpm = w["Mdeg"] * w["nvec"]
    # slices run concurrently (one process each): the slowest slice sets
    # the time; the KPM vectors are split across the same processes
    slice_t = max(per_deg * (its + 1) * deg for its, deg in zip(g["its"], g["deg"]))
    total_t = slice_t + per_deg * (kpm / cores + 200)
    value = g["eigenpairs"] / total_t
    sample_s = float(np.mean(times)) if times else 0.0
    measured = g.get("seconds_per_slice")
    how = (f"reference pEVSL_ChebAv (oracle/_ref, one core per process, {nsl} processes in "
           f"parallel) for ~{sample_target:.0f} s per slice and step with each slice's own "
           f"filter: {per_deg*1e3:.2f} ms per "
           f"degree; extrapolated x{total_t / max(sample_s, 1e-9):.0f} to the reference run's "
           f"per-slice Lanczos steps {g['its']} and filter degrees {g['deg']} "
           f"({g['fixture']}) + the KPM matvecs split over {cores} processes + <=200 bounds "
           f"matvecs" + (f"; the full reference run that wrote the fixture took "
                         f"{[round(x) for x in measured]} s per slice on one core each"
                         if measured else ""))
    return {"metric": metric_of(w), "value": value, "unit": "eigenpairs/s", "n_gpus": dist.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sample_s,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: 3D Dirichlet Laplacian", "impl": "reference",
            "config": {"workload": args.workload, "n": n, "nnz": int(ia[-1]),
                       "slice_ends": sli, "filter_degree_per_slice": g["deg"],
                       "lanczos_steps_per_slice": g["its"], "nev_per_slice": g["nev"],
                       "estimated_seconds_per_run": total_t},
            "cpu_baseline": {"value": value, "unit": "eigenpairs/s", "cores": cores,
                             "kind": "reference", "sample": how},
            "e2e": {"value": value, "unit": "eigenpairs/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def kernel_case(args):
    """A few launches of one kernel on a matrix larger than L2, for ncu, on
    the 3D Laplacian of side --grid:
      cheb_step  two degree-16 filter applications (32 fused filter-degree
                 launches, one vector);
      cheb_batch --batch slices of [0.8, 4.0] with filters of degree
                 --degree (16) in lockstep, 3 Lanczos steps; prints the
                 filter's live timing per degree;
      kpm_step   8 KPM degrees for 16 vectors;
      gen_filter two degree-16 generalized filter applications on the
                 genlap24 problem scaled to --grid (B-solve: least-squares
                 1/x of degree 24, 25 launches per degree);
      c4_filter  the C4 matrix (random symmetric, n = 2e6, ~17 entries per
                 row, offsets within +-5000; seed 1): 3 Lanczos steps with
                 a degree-16 filter on one slice, then on 16 interior slices
                 in lockstep; prints the filter's live timing (CUDA events)
                 and HBM fraction per degree;
    (a forced degree d gives a filter of degree d - 1, as in the reference)
      pipeline   one whole batched solve of --workload (for launch lists);
      gemm       the DMMA products: Ritz vectors U = V Y and Gram matrix
                 V' U with n = --grid^3, k = --degree, m = 128 (device
                 time and TFLOP/s of each)."""
    import pevsl_b200 as pv
    from pevsl_b200.problems import laplacian
    if args.kernel_case == "c4_filter":
        from pevsl_b200.problems import random_sparse_symmetric
        n, ia, ja, a = random_sparse_symmetric(2000000, 16, 5000, 1)
        # Gershgorin enclosure of the spectrum
        rows = np.repeat(np.arange(n), np.diff(ia))
        diag = np.zeros(n)
        np.add.at(diag, rows[ja == rows], a[ja == rows])
        rad = np.bincount(rows, weights=np.abs(a), minlength=n) - np.abs(diag)
        lmin, lmax = float(np.min(diag - rad)), float(np.max(diag + rad))
        M = pv.Matrix.from_csr(n, ia, ja, a)
        wdt = lmax - lmin
        edges = np.linspace(lmin + 0.1 * wdt, lmax - 0.1 * wdt, 17)
        intvs = [[edges[i], edges[i + 1], lmin, lmax] for i in range(16)]
        fl = [pv.findpol(iv, deg_in=16)[1] for iv in intvs]
        v = np.cos(np.arange(n) * 0.1)
        peak, kind = measured_peak()
        out = {"kernel_case": "c4_filter", "n": n, "nnz": int(ia[-1]), "bounds": [lmin, lmax]}
        with pv.Instance(M) as ev:
            for label, k in (("one_slice", 1), ("16_slices", 16)):
                pv.load().pEVSL_B200_ResetFilterCounters()
                if k == 1:
                    ev.cheblannr(intvs[0], 3, 1e-8, v, fl[0])
                else:
                    pv.cheblannr_batch(ev, intvs, [3] * 16, 1e-8, v, fl)
                l, b, ms = pv.filter_counters()
                out[label] = {"launches": l, "us_per_launch": 1e3 * ms / l,
                              "bytes_per_launch": b / l, "GBps": b / ms / 1e6,
                              "frac": b / ms / 1e6 / peak, "peak": peak, "peak_source": kind}
        M.free()
        print(json.dumps(out))
        return
    if args.kernel_case == "gemm":
        # the two DMMA products at the size of one C2 slice's Ritz step:
        # U = V Y (n = 1e6, k = --degree Lanczos vectors, m = 128 Ritz vectors)
        # and the Gram matrix C = V' W (W = U)
        lib = pv.load()
        for f in (lib.pEVSL_B200_GemmNN, lib.pEVSL_B200_GemmTN):
            f.argtypes = [C.c_long, C.c_int, C.c_int, C.c_void_p, C.c_long, C.c_void_p, C.c_long,
                          C.c_void_p, C.c_long]
        n, k, m = args.grid ** 3, args.degree, 128
        V = pv.Vector(n * k, np.cos(np.arange(n * k) * 1e-3))
        Y = pv.Vector(k * m, np.sin(np.arange(k * m) * 0.1))
        U, G = pv.Vector(n * m), pv.Vector(k * m)
        # one untimed call of each first: the vectors are managed memory
        # filled on the host, and the first touch migrates their pages
        lib.pEVSL_B200_GemmNN(n, k, m, V.pv.data, n, Y.pv.data, k, U.pv.data, n)
        lib.pEVSL_B200_GemmTN(n, k, m, V.pv.data, n, U.pv.data, n, G.pv.data, k)
        lib.pEVSL_B200_Sync()
        lib.pEVSL_B200_EventRecord(0)
        for _ in range(2):
            lib.pEVSL_B200_GemmNN(n, k, m, V.pv.data, n, Y.pv.data, k, U.pv.data, n)
        lib.pEVSL_B200_EventRecord(1)
        for _ in range(2):
            lib.pEVSL_B200_GemmTN(n, k, m, V.pv.data, n, U.pv.data, n, G.pv.data, k)
        lib.pEVSL_B200_EventRecord(2)
        t_nn = lib.pEVSL_B200_EventElapsedMs(0, 1) / 2
        t_tn = lib.pEVSL_B200_EventElapsedMs(1, 2) / 2
        fl = 2.0 * n * k * m
        print(json.dumps({"kernel_case": "gemm", "n": n, "k": k, "m": m,
                          "gemm_nn_ms": t_nn, "gemm_nn_tflops": fl / t_nn / 1e9,
                          "gemm_tn_ms": t_tn, "gemm_tn_tflops": fl / t_tn / 1e9,
                          "gemm_nn_GBps": 8.0 * (n * k * ((m + 63) // 64) + n * m) / t_nn / 1e6}))
        for x in (V, Y, U, G):
            x.free()
        return
    if args.kernel_case == "pipeline":
        w = WORKLOADS[args.workload]
        n, ia, ja, a = laplacian(*w["grid"])
        M = pv.Matrix.from_csr(n, ia, ja, a)
        r = pv.solve_interval(M, slice_run(w, 0), batched=True)
        print(json.dumps({"kernel_case": "pipeline", "workload": args.workload,
                          "nev": [int(x) for x in r.nev], "status": r.status}))
        return
    g = args.grid
    n, ia, ja, a = laplacian(g, g, g)
    M = pv.Matrix.from_csr(n, ia, ja, a)
    pv.set_rng(pv.RNG_GAUSS, 0)
    if args.kernel_case == "gen_filter":
        gs = GenSetup(WORKLOADS["genlap24"], n)
        r, f = pv.findpol([0.5, 2.0, 0.02, 4.1], deg_in=16)
        v = np.cos(np.arange(n) * 0.1)
        with pv.Instance(M) as ev:
            gs.install(ev)
            pol, keep = pv._polparams(f)
            vv, yv = pv.Vector(n, v), pv.Vector(n)
            for _ in range(2):
                st = ev.lib.pEVSL_B200_ChebAvGen(ev.p, C.byref(pol), vv.pv.data, yv.pv.data)
            vv.free()
            yv.free()
        gs.free()
        print(json.dumps({"kernel_case": "gen_filter", "n": n, "status": st}))
        return
    extra = {}
    with pv.Instance(M) as ev:
        if args.kernel_case == "cheb_step":
            r, f = pv.findpol([0.8, 4.0, 0.0, 12.0], deg_in=16)
            v = np.cos(np.arange(n) * 0.1)
            for _ in range(2):
                ev.chebav(f, v)
        elif args.kernel_case == "cheb_batch":
            S = args.batch
            edges = np.linspace(0.8, 4.0, S + 1)
            intvs = [[edges[i], edges[i + 1], 0.0, 12.0] for i in range(S)]
            fl = [pv.findpol(iv, deg_in=args.degree)[1] for iv in intvs]
            v = np.cos(np.arange(n) * 0.1)
            pv.load().pEVSL_B200_ResetFilterCounters()
            pv.cheblannr_batch(ev, intvs, [3] * S, 1e-8, v, fl)
            l, b, ms = pv.filter_counters()
            peak, kind = measured_peak()
            extra = {"batch": S, "launches": l, "us_per_launch": 1e3 * ms / l,
                     "bytes_per_launch": b / l, "GBps": b / ms / 1e6,
                     "frac": b / ms / 1e6 / peak, "peak": peak, "peak_source": kind}
        else:
            ev.kpmdos(8, 1, 16, [0.80, 0.82, 0.0, 12.0])
    print(json.dumps({"kernel_case": args.kernel_case, "n": n, "nnz": int(ia[-1]), **extra}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--path", default="batched", choices=["batched", "plain"],
                    help="batched: slices in lockstep; plain: one pEVSL_ChebLanNr per slice")
    ap.add_argument("--mode", default="replicas", choices=["replicas", "distributed"],
                    help="N > 1: replicas (every rank solves its own copy, weak scaling) or "
                         "distributed (one problem over the ranks: KPM vectors split and summed "
                         "by an all-reduce, slices shared out; strong scaling)")
    ap.add_argument("--degree", type=int, default=16,
                    help="filter degree of the cheb_batch kernel case")
    ap.add_argument("--kernel-case", choices=["cheb_step", "cheb_batch", "kpm_step", "gen_filter",
                                              "c4_filter", "pipeline", "gemm"],
                    help="run a few launches of one kernel (for ncu) and exit")
    ap.add_argument("--grid", type=int, default=128)
    ap.add_argument("--batch", type=int, default=4)
    args = ap.parse_args()
    if args.kernel_case:
        kernel_case(args)
        return
    if args.warmup < 3:
        args.warmup = 3
    dist = Dist(args.gpus)
    if args.impl == "reference":
        out = run_reference(args, dist)
    elif WORKLOADS[args.workload].get("multi"):
        out = run_b200_multi(args, dist)
    else:
        out = run_b200(args, dist)
    if dist.rank == 0 and out is not None:
        print(json.dumps(out), flush=True)
    dist.close()


if __name__ == "__main__":
    main()
