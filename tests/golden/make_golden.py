"""Generate the golden fixtures in tests/golden/ from the pEVSL reference.

Runs oracle/_ref/libpevsl_ref.so (the reference compiled from its own sources
by oracle/Makefile; needs the reference tree, so this runs where the
reference is mounted, never on a GPU box) and writes small JSON files that
the CPU tests use to pin the oracle restatement and the GPU tests use as
known answers.  Floats are written with repr() so they round-trip exactly.

    python tests/golden/make_golden.py [mm | gen | findpol | c2]
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from checkers import Checker, RunSpec, laplacian  # noqa: E402


def fl(x):
    return [float(v) for v in np.asarray(x).ravel()]


def dump(name, obj):
    path = os.path.join(HERE, name)
    with open(path, "w") as f:
        json.dump(obj, f, indent=1)
    print("wrote", path, os.path.getsize(path), "bytes")


def pipeline_case(ref, grid, spec: RunSpec):
    A = laplacian(*grid)
    r = ref.pipeline(A, spec)
    return dict(
        grid=list(grid), spec=spec.__dict__, status=r.status, lmin=r.lmin, lmax=r.lmax,
        ecount=r.ecount, npts=r.npts, mu=fl(r.mu) if spec.dos_type == 0 else None,
        sli=fl(r.sli), deg=[int(v) for v in r.deg], ptype=[int(v) for v in r.ptype],
        gam=fl(r.gam), bar=fl(r.bar), nev=[int(v) for v in r.nev], its=[int(v) for v in r.its],
        lam=[fl(x) for x in r.lam], res=[fl(x) for x in r.res])


def main():
    ref = Checker("ref")

    # 1. SpMV, input sin(i) as TESTS0/Matvec/test1.c:70-85 (3D and 2D grids)
    mv = {}
    for grid in ((8, 8, 8), (12, 10, 1)):
        A = laplacian(*grid)
        x = np.sin(np.arange(A.n, dtype=np.float64))
        mv["x".join(map(str, grid))] = dict(grid=list(grid), y=fl(ref.matvec(A, x)))
    dump("matvec_sin.json", mv)

    # 2. KPM moments + slicer + filters on the README matrix (hand-set bounds)
    A = laplacian(20, 20, 20)
    intv = [0.6, 1.2, 0.0, 12.0]
    kpm = {}
    for mode in (0, 1):
        ref.set_rng(mode, 0)
        r, mu, ec = ref.kpmdos(A, 300, 1, 60, intv)
        npts = int(10 * ec)
        rs, sli = ref.spslicer_kpm(mu, 300, intv, 5, npts)
        pols = []
        for sl in range(5):
            _, p = ref.findpol([sli[sl], sli[sl + 1], 0.0, 12.0])
            pols.append(dict(intv=[float(sli[sl]), float(sli[sl + 1]), 0.0, 12.0],
                             type=p["type"], deg=p["deg"], gam=p["gam"], bar=p["bar"],
                             cc=p["cc"], dd=p["dd"], mu=fl(p["mu"])))
        kpm["glibc" if mode == 0 else "gauss"] = dict(
            status=r, mu=fl(mu), ecount=ec, npts=npts, slicer_status=rs, sli=fl(sli), pols=pols)
    dump("lap20_kpm.json", dict(grid=[20, 20, 20], intv=intv, Mdeg=300, damping=1, nvec=60,
                                seed=0, cases=kpm))

    findpol_cases(ref)

    # 4. Slicer edge cases: one slice, many slices, invalid interval
    ref.set_rng(1, 7)
    A = laplacian(10, 10, 10)
    intv = [0.5, 3.0, 0.0, 12.0]
    _, mu, ec = ref.kpmdos(A, 80, 1, 20, intv)
    sl_cases = []
    for n_int, npts in ((1, 50), (4, int(10 * ec)), (9, 30), (4, 3)):
        r, sli = ref.spslicer_kpm(mu, 80, intv, n_int, npts)
        sl_cases.append(dict(n_int=n_int, npts=npts, status=r, sli=fl(sli)))
    r, _ = ref.spslicer_kpm(mu, 80, [3.0, 0.5, 0.0, 12.0], 4, 40)
    sl_cases.append(dict(n_int=4, npts=40, intv=[3.0, 0.5, 0.0, 12.0], status=r))
    dump("spslicer_cases.json", dict(grid=[10, 10, 10], intv=intv, Mdeg=80, mu=fl(mu),
                                     ecount=ec, cases=sl_cases))

    # 5. Lanczos DOS + its slicer, and thick-restart bounds
    A = laplacian(12, 12, 12)
    ref.set_rng(1, 3)
    r, xd, yd, ne = ref.landos(A, 10, 40, 200, [0.5, 6.0, 0.0, 12.0])
    sli = ref.spslicer_lan(xd, yd, 4)
    v0 = np.cos(np.arange(A.n, dtype=np.float64))
    bnd = {}
    for bt in (1, 2):
        ref.set_rng(1, 3)
        rb, lo, hi = ref.lantrbounds(A, 50, 200, 1e-8, v0, bt)
        bnd[str(bt)] = dict(status=rb, lmin=lo, lmax=hi)
    dump("lanczos_cases.json", dict(grid=[12, 12, 12], landos=dict(
        nvec=10, msteps=40, npts=200, intv=[0.5, 6.0, 0.0, 12.0], seed=3, status=r, xdos=fl(xd),
        ydos=fl(yd), neig=ne, sli4=fl(sli)), lantrbounds=dict(v0="cos(i)", lanm=50, maxit=200,
                                                              tol=1e-8, cases=bnd)))

    # 6. Whole runs: small 3D and 2D Laplacians, and the README matrix with
    #    (a) hand-set bounds / glibc stream, (b) LanTrbounds / Gaussian stream,
    #    (c) Lanczos DOS
    runs = {}
    runs["lap10_kpm_gauss"] = pipeline_case(
        ref, (10, 10, 10), RunSpec(0.6, 2.0, 3, Mdeg=100, nvec=20, rng_mode=1, seed=11))
    runs["lap30x30_kpm_glibc"] = pipeline_case(
        ref, (30, 30, 1), RunSpec(1.0, 2.0, 2, lmax=8.0, Mdeg=120, nvec=20, rng_mode=0, seed=5))
    runs["lap20_readme_glibc"] = pipeline_case(ref, (20, 20, 20), RunSpec(0.6, 1.2, 5))
    runs["lap20_lantr_gauss"] = pipeline_case(
        ref, (20, 20, 20), RunSpec(0.6, 1.2, 5, bounds_mode=1, rng_mode=1, seed=0))
    runs["lap12_landos_gauss"] = pipeline_case(
        ref, (12, 12, 12), RunSpec(0.5, 2.5, 3, dos_type=1, nvec=10, rng_mode=1, seed=2))
    dump("pipelines.json", runs)

    # 7. Lucky breakdown and restart (SRC/cheblanNr.c:248-281): a diagonal
    #    matrix with 10 distinct eigenvalues of multiplicity 40; the Krylov
    #    space exhausts after a few steps and every restart draws a new
    #    random vector from the glibc stream.
    n = 400
    d = np.repeat(np.arange(1.0, 11.0), 40)
    ia = np.arange(n + 1, dtype=np.int32)
    ja = np.arange(n, dtype=np.int32)
    from checkers import Csr
    D = Csr(n, ia, ja, d.copy())
    intv = [3.5, 5.5, 0.5, 10.5]
    _, pol = ref.findpol(intv)
    ref.set_rng(0, 9)
    v0 = np.cos(np.arange(n, dtype=np.float64) * 0.37)
    out = ref.cheblannr(D, intv, 300, 1e-8, v0, pol)
    dump("breakdown_case.json", dict(n=n, diag="repeat(1..10, 40)", intv=intv, maxit=300,
                                     tol=1e-8, v0="cos(0.37 i)", seed=9, deg=pol["deg"],
                                     status=out["status"], nev=out["nev"], its=out["its"],
                                     lam=fl(out["lam"]), res=fl(out["res"])))


def findpol_cases(ref):
    """Filter design edge cases: end intervals (chext), forced degree, every
    damping type, invalid intervals (check_intv codes), and slices on which
    a degree below 2 + 0.5/(normalised width) already meets the threshold
    (the reference's search starts at degree 2, SRC/chebpol.c:434): three
    slices of a random-coefficient 41^3 Laplacian's spectrum bound [0, 24]
    and a slice of width 1.4e-4 (normalised) with max_deg 3000, 20000 and a
    forced degree 100."""
    narrow = [0.4845065036442954, 0.4850594098995861, 0.4435124791600489, 8.445429558871442]
    cases = []
    for intv_c, kw in (([0.0, 0.5, 0.0, 12.0], {}), ([-1.0, 0.5, 0.0, 12.0], {}),
                       ([11.0, 12.0, 0.0, 12.0], {}), ([11.5, 13.0, 0.0, 12.0], {}),
                       ([0.8, 0.82, 0.0, 12.0], {}), ([3.0, 3.5, 0.0, 12.0], {"damping": 0}),
                       ([3.0, 3.5, 0.0, 12.0], {"damping": 1}), ([3.0, 3.5, 0.0, 12.0], {"deg_in": 40}),
                       ([0.0, 0.5, 0.0, 12.0], {"deg_in": 25}),
                       ([2.0, 2.5, 0.0, 8.0], {"thresh_int": 0.6, "thresh_ext": 0.15}),
                       ([1.0, 0.5, 0.0, 12.0], {}), ([13.0, 14.0, 0.0, 12.0], {}),
                       ([0.10, 0.123, 0.0, 24.0], {}), ([0.123, 0.143, 0.0, 24.0], {}),
                       ([0.143, 0.165, 0.0, 24.0], {}),
                       (narrow, {"max_deg": 3000}), (narrow, {"max_deg": 20000}),
                       (narrow, {"max_deg": 3000, "deg_in": 100})):
        r, p = ref.findpol(intv_c, **kw)
        c = dict(intv=intv_c, kw=kw, status=r)
        if p is not None:
            c.update(type=p["type"], deg=p["deg"], gam=p["gam"], bar=p["bar"], cc=p["cc"],
                     dd=p["dd"], mu=fl(p["mu"]))
        cases.append(c)
    dump("findpol_cases.json", dict(cases=cases))


def mm_case(refdir=None):
    """The reference's Matrix Market driver (TESTS/MM/MMPLanN.c, built by
    `make -C oracle drivers` against the reference build) on its own
    MATRICES/A.mtx (stiff1) with the first two intervals of TESTS/MM/matfile.
    Writes mm_stiff1.npz: the matrix's coordinate entries exactly as the
    file lists them (one triangle, 1-based), and the driver's output."""
    import subprocess
    import tempfile

    from checkers import REFERENCE_TREE
    refdir = refdir or REFERENCE_TREE
    root = os.path.dirname(os.path.dirname(HERE))
    exe = os.path.join(root, "oracle", "_ref", "MMPLanN")
    src = os.path.join(refdir, "MATRICES", "A.mtx")
    with open(src) as f:
        lines = [ln for ln in f if not ln.startswith("%")]
    nr, nc, nz = (int(x) for x in lines[0].split())
    ent = np.array([ln.split() for ln in lines[1:1 + nz]])
    I, J = ent[:, 0].astype(np.int32), ent[:, 1].astype(np.int32)
    V = ent[:, 2].astype(np.float64)
    intervals = [(0.10, 0.12, 3), (0.12, 0.14, 2)]
    with tempfile.TemporaryDirectory() as d:
        write_mm(os.path.join(d, "stiff1.mtx"), nr, I, J, V)
        write_matfile(os.path.join(d, "matfile"), "stiff1.mtx", intervals)
        os.makedirs(os.path.join(d, "OUT"))
        subprocess.run([exe, "-matfile", "matfile", "-ngroups", "1"], cwd=d, check=True,
                       capture_output=True, env=dict(os.environ, OPENBLAS_NUM_THREADS="1"))
        with open(os.path.join(d, "OUT", "LapPLanN_G0.out")) as f:
            out = f.read()
    path = os.path.join(HERE, "mm_stiff1.npz")
    np.savez_compressed(path, n=nr, i=I, j=J, v=V, intervals=np.array(intervals),
                        output=np.array(out))
    print("wrote", path, os.path.getsize(path), "bytes")


def gen_case():
    """The generalized problem.  (1) The reference's B-solvers on the 1D
    Laplacian B of TESTS/Gen_Lap/LapPLanN.c (n = 512, diagonal 4): the
    least-squares coefficients of 1/x and 1/sqrt(x) and one solve each, and
    Chebyshev-iteration solves -> gen_bsolve.json.  (2) That driver, built
    against the reference with the Chebyshev B-solver of tests/dropin/shim
    (`make -C oracle drivers`), with KPM and with Lanczos DOS -> genlap8.json
    (its screen output and OUT/LapPLanN_G0.out)."""
    import subprocess
    import tempfile
    ref = Checker("ref")
    B = laplacian(512, 1, 1)
    b = np.cos(0.1 * np.arange(B.n, dtype=np.float64)) + 0.5
    ls = []
    for kind, max_deg, tol in ((0, 50, 1e-6), (1, 50, 1e-6), (0, 80, 1e-10), (1, 120, 1e-12)):
        deg, mu, cc, dd, x = ref.lspol(kind, max_deg, tol, 2.0, 6.0, B, b)
        ls.append(dict(kind=kind, max_deg=max_deg, tol=tol, lmin=2.0, lmax=6.0, deg=deg,
                       mu=fl(mu), cc=cc, dd=dd, x=fl(x)))
    ci = []
    for kind, deg in ((1, 1), (1, 12), (2, 0), (2, 12), (2, 40)):
        ci.append(dict(kind=kind, deg=deg, lmin=2.0, lmax=6.0,
                       x=fl(ref.chebiter(kind, 2.0, 6.0, deg, B, b))))
    dump("gen_bsolve.json", dict(B="laplacian(512,1,1)", b="cos(0.1 i) + 0.5", lspol=ls,
                                 chebiter=ci))
    root = os.path.dirname(os.path.dirname(HERE))
    exe = os.path.join(root, "oracle", "_ref", "GenLapPLanN")
    runs = {}
    for name, args in (("kpm", ["-ngroups", "1"]),
                       ("landos", ["-ngroups", "1", "-dostype", "1", "-nslices", "3"])):
        with tempfile.TemporaryDirectory() as d:
            os.makedirs(os.path.join(d, "OUT"))
            r = subprocess.run([exe] + args, cwd=d, check=True, capture_output=True, text=True,
                               env=dict(os.environ, OPENBLAS_NUM_THREADS="1"))
            with open(os.path.join(d, "OUT", "LapPLanN_G0.out")) as f:
                runs[name] = dict(args=args, stdout=r.stdout, out=f.read())
    dump("genlap8.json", runs)


def write_mm(path, n, I, J, V):
    """A symmetric Matrix Market file with the given entries (repr floats:
    they read back to the same doubles)."""
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real symmetric\n")
        f.write(f"{n} {n} {len(V)}\n")
        f.writelines(f"{i} {j} {v!r}\n" for i, j, v in zip(I.tolist(), J.tolist(), V.tolist()))


def write_matfile(path, mtx, intervals):
    """TESTS/MM/matfile's format: the count, then one line per problem."""
    with open(path, "w") as f:
        f.write(f"{len(intervals)}\n")
        for a, b, ns in intervals:
            f.write(f"{mtx} stiff1 MM1 {a} {b} {ns}\n")


# The 100^3 Laplacian run of the benchmark: interval [0.80, 0.82], 4 slices,
# thick-restart bounds (50, 200, 1e-8), KPM Mdeg 300 with 30 Philox Gaussian
# vectors (seed 0), filters FindPol(damping 2, max_deg 3000, 0.8 / 0.2),
# ChebLanNr tol 1e-8.
C2_GRID = (100, 100, 100)
C2_SPEC = dict(a_lo=0.80, b_hi=0.82, nslices=4, bounds_mode=1, Mdeg=300, nvec=30, kpm_damping=1,
               pol_damping=2, pol_max_deg=3000, thresh_int=0.8, thresh_ext=0.2, tol=1e-8,
               rng_mode=1, seed=0)


def _c2_slice(args):
    """One slice of the run in its own process (the reference build on one
    core): bounds, KPM and slicing in full, then ChebLanNr on this slice."""
    grid, spec, sl = args
    import time
    t = time.time()
    ref = Checker("ref")
    r = ref.pipeline(laplacian(*grid), RunSpec(**spec), cap=1000, slices=(sl, sl + 1))
    return sl, r, time.time() - t


def c2_case(grid=C2_GRID, spec=None, name="lap100_c2.json", procs=None):
    """The benchmark's run on the reference build, one process per slice
    (a few hours of CPU on 100^3): slice ends, filters, per-slice Lanczos
    steps, accepted counts, eigenvalues and residuals -> lap100_c2.json."""
    import multiprocessing as mp
    import time
    spec = dict(C2_SPEC if spec is None else spec)
    ns = spec["nslices"]
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    t0 = time.time()
    with mp.get_context("spawn").Pool(procs or ns) as pool:
        parts = {}
        for sl, r, dt in pool.imap_unordered(_c2_slice, [(grid, spec, k) for k in range(ns)]):
            parts[sl] = (r, dt)
            print(f"slice {sl}: its {int(r.its[sl])} nev {int(r.nev[sl])} deg {int(r.deg[sl])} "
                  f"({dt:.0f} s)", flush=True)
    r0 = parts[0][0]
    for sl in range(1, ns):  # every process computed the same bounds, moments and slices
        r = parts[sl][0]
        assert (r.lmin, r.lmax, r.ecount) == (r0.lmin, r0.lmax, r0.ecount)
        assert np.array_equal(r.sli, r0.sli) and np.array_equal(r.mu, r0.mu)
    pick = lambda f: [f(parts[sl][0], sl) for sl in range(ns)]  # noqa: E731
    dump(name, dict(
        grid=list(grid), spec=spec, status=max(parts[sl][0].status for sl in range(ns)),
        lmin=r0.lmin, lmax=r0.lmax, ecount=r0.ecount, npts=r0.npts, mu=fl(r0.mu), sli=fl(r0.sli),
        deg=pick(lambda r, k: int(r.deg[k])), ptype=pick(lambda r, k: int(r.ptype[k])),
        gam=pick(lambda r, k: float(r.gam[k])), bar=pick(lambda r, k: float(r.bar[k])),
        nev=pick(lambda r, k: int(r.nev[k])), its=pick(lambda r, k: int(r.its[k])),
        lam=pick(lambda r, k: fl(r.lam[k])), res=pick(lambda r, k: fl(r.res[k])),
        seconds_per_slice=[round(parts[sl][1], 1) for sl in range(ns)],
        wall_seconds=round(time.time() - t0, 1),
        how="reference build (oracle/_ref), one process per slice, one core each"))


if __name__ == "__main__":
    if sys.argv[1:] == ["c2"]:
        c2_case()
    elif sys.argv[1:] == ["c2-check"]:
        # the same machinery on the README matrix, against pipelines.json
        c2_case((20, 20, 20), dict(a_lo=0.6, b_hi=1.2, nslices=5, bounds_mode=1, rng_mode=1,
                                   seed=0), name="_c2_check.json")
    elif sys.argv[1:] == ["mm"]:
        mm_case()
    elif sys.argv[1:] == ["findpol"]:
        findpol_cases(Checker("ref"))
    elif sys.argv[1:] == ["gen"]:
        gen_case()
    else:
        main()
        mm_case()
        gen_case()
