"""Pin the oracle restatement (oracle/pevsl_oracle.c) to the reference.

The golden fixtures in tests/golden/ were produced by the pEVSL reference
compiled from its own sources (tests/golden/make_golden.py); the oracle must
reproduce them before it is trusted as the checker of the CUDA path.
Tolerances: integer outputs (degrees, counts, iterations, filter types,
return codes) exact; moments / endpoints / filter data 1e-12 relative;
eigenvalues 1e-10 relative; the known answers of ExactEigLap3 to 1e-12.
"""
import numpy as np
import pytest

from checkers import RunSpec, exact_eig_lap, laplacian
from conftest import golden


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_matvec_golden(oracle):
    for key, case in golden("matvec_sin.json").items():
        A = laplacian(*case["grid"])
        y = oracle.matvec(A, np.sin(np.arange(A.n, dtype=np.float64)))
        assert rel(y, case["y"]) <= 1e-15, key


def test_laplacian_generator_matches_oracle_c(oracle):
    import ctypes as C
    for grid in ((20, 20, 20), (7, 5, 3), (30, 30, 1)):
        A = laplacian(*grid)
        n = A.n
        ia = np.zeros(n + 1, np.int32)
        ja = np.zeros(7 * n, np.int32)
        a = np.zeros(7 * n)
        nnz = oracle.lib.orc_lap3(*grid, ia.ctypes.data_as(C.c_void_p),
                                  ja.ctypes.data_as(C.c_void_p), a.ctypes.data_as(C.c_void_p))
        assert nnz == A.nnz
        assert np.array_equal(ia, A.ia) and np.array_equal(ja[:nnz], A.ja)
        assert np.array_equal(a[:nnz], A.a)
    # nnz of the README matrix: 7n - 2*3*400
    assert laplacian(20, 20, 20).nnz == 53600


@pytest.mark.parametrize("mode", ["glibc", "gauss"])
def test_kpm_slicer_filters_golden(oracle, mode):
    g = golden("lap20_kpm.json")
    case = g["cases"][mode]
    A = laplacian(*g["grid"])
    oracle.set_rng(0 if mode == "glibc" else 1, g["seed"])
    r, mu, ec = oracle.kpmdos(A, g["Mdeg"], g["damping"], g["nvec"], g["intv"])
    assert r == case["status"] == 0
    assert rel(mu, case["mu"]) <= 1e-12
    assert abs(ec - case["ecount"]) <= 1e-10 * abs(case["ecount"])
    assert int(10 * ec) == case["npts"]
    rs, sli = oracle.spslicer_kpm(np.array(case["mu"]), g["Mdeg"], g["intv"], 5, case["npts"])
    assert rs == case["slicer_status"]
    assert rel(sli, case["sli"]) <= 1e-12
    for p in case["pols"]:
        r, q = oracle.findpol(p["intv"])
        assert r == 0 and q["deg"] == p["deg"] and q["type"] == p["type"]
        for k in ("gam", "bar", "cc", "dd"):
            assert abs(q[k] - p[k]) <= 1e-12 * max(1.0, abs(p[k])), k
        assert rel(q["mu"], p["mu"]) <= 1e-12


def test_findpol_edge_cases_golden(oracle):
    for c in golden("findpol_cases.json")["cases"]:
        r, q = oracle.findpol(c["intv"], **c["kw"])
        assert r == c["status"], c
        if r == 0:
            assert q["type"] == c["type"] and q["deg"] == c["deg"], c
            assert abs(q["gam"] - c["gam"]) <= 1e-12 and abs(q["bar"] - c["bar"]) <= 1e-12
            assert rel(q["mu"], c["mu"]) <= 1e-12


def test_spslicer_edge_cases_golden(oracle):
    g = golden("spslicer_cases.json")
    for c in g["cases"]:
        iv = c.get("intv", g["intv"])
        r, sli = oracle.spslicer_kpm(np.array(g["mu"]), g["Mdeg"], iv, c["n_int"], c["npts"])
        assert r == c["status"], c
        if "sli" in c:
            assert rel(sli, c["sli"]) <= 1e-12, c


def test_lanczos_dos_and_bounds_golden(oracle):
    g = golden("lanczos_cases.json")
    A = laplacian(*g["grid"])
    d = g["landos"]
    oracle.set_rng(1, d["seed"])
    r, xd, yd, ne = oracle.landos(A, d["nvec"], d["msteps"], d["npts"], d["intv"])
    assert r == d["status"]
    assert rel(xd, d["xdos"]) <= 1e-15
    assert rel(yd, d["ydos"]) <= 1e-10
    assert abs(ne - d["neig"]) <= 1e-10 * abs(d["neig"])
    sli = oracle.spslicer_lan(xd, yd, 4)
    assert rel(sli, d["sli4"]) <= 1e-12
    b = g["lantrbounds"]
    v0 = np.cos(np.arange(A.n, dtype=np.float64))
    for bt, c in b["cases"].items():
        r, lo, hi = oracle.lantrbounds(A, b["lanm"], b["maxit"], b["tol"], v0, int(bt))
        assert r == c["status"]
        # bounds are converged to tol = 1e-8 (SRC/lantrbnd.c:369); the
        # restated dense eigensolver agrees with LAPACK to rounding
        assert abs(lo - c["lmin"]) <= 1e-10 * max(1, abs(c["lmin"]))
        assert abs(hi - c["lmax"]) <= 1e-10 * abs(c["lmax"])


@pytest.mark.parametrize("name", ["lap10_kpm_gauss", "lap30x30_kpm_glibc", "lap12_landos_gauss"])
def test_pipeline_golden_small(oracle, name):
    g = golden("pipelines.json")[name]
    A = laplacian(*g["grid"])
    s = RunSpec(**g["spec"])
    r = oracle.pipeline(A, s)
    check_pipeline(r, g)


@pytest.mark.slow
@pytest.mark.parametrize("name", ["lap20_readme_glibc", "lap20_lantr_gauss"])
def test_pipeline_golden_readme(oracle, name):
    g = golden("pipelines.json")[name]
    A = laplacian(*g["grid"])
    r = oracle.pipeline(A, RunSpec(**g["spec"]))
    check_pipeline(r, g)


def check_pipeline(r, g):
    assert r.status == g["status"] == 0
    assert abs(r.lmin - g["lmin"]) <= 1e-10 * max(1, abs(g["lmin"]))
    assert abs(r.lmax - g["lmax"]) <= 1e-10 * abs(g["lmax"])
    assert abs(r.ecount - g["ecount"]) <= 1e-10 * abs(g["ecount"])
    assert r.npts == g["npts"]
    assert rel(r.sli, g["sli"]) <= 1e-12
    assert list(r.deg) == g["deg"] and list(r.ptype) == g["ptype"]
    assert list(r.nev) == g["nev"]
    assert list(r.its) == g["its"]
    for sl in range(len(g["nev"])):
        assert rel(r.lam[sl], g["lam"][sl]) <= 1e-10
        assert np.all(r.res[sl] < g["spec"]["tol"])
        # known answer: the analytic Laplacian spectrum (TESTS/COMMON/lapl.c:139-169)
        ex = exact_eig_lap(*g["grid"], g["sli"][sl], g["sli"][sl + 1])
        assert len(ex) == g["nev"][sl]
        assert np.max(np.abs(r.lam[sl] - ex)) <= 1e-12


def test_exact_eigs_known_answer_readme():
    """The README's per-slice counts are the analytic counts of its slices
    (README.md:111-115 lists computed == exact)."""
    g = golden("pipelines.json")["lap20_readme_glibc"]
    counts = [len(exact_eig_lap(20, 20, 20, g["sli"][i], g["sli"][i + 1])) for i in range(5)]
    assert counts == g["nev"] == [21, 24, 27, 19, 27]


def test_oracle_against_live_reference(oracle, reference):
    """Where the reference build is present, compare the two checkers live on
    a case that is not in the fixtures (a 3D Laplacian with unequal sides)."""
    A = laplacian(9, 11, 8)
    s = RunSpec(1.0, 2.5, 3, Mdeg=80, nvec=12, rng_mode=1, seed=123, lmax=12.0)
    r1 = reference.pipeline(A, s)
    r2 = oracle.pipeline(A, s)
    assert r1.status == r2.status == 0
    assert rel(r2.mu, r1.mu) <= 1e-12 and rel(r2.sli, r1.sli) <= 1e-12
    assert list(r2.nev) == list(r1.nev) and list(r2.deg) == list(r1.deg)
    for a, b in zip(r2.lam, r1.lam):
        assert rel(a, b) <= 1e-10


def test_breakdown_restart_golden(oracle):
    """Repeated lucky breakdowns with random restarts (SRC/cheblanNr.c:248-281)
    on a diagonal matrix with 10 distinct eigenvalues of multiplicity 40."""
    from checkers import Csr
    g = golden("breakdown_case.json")
    n = g["n"]
    D = Csr(n, np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32),
            np.repeat(np.arange(1.0, 11.0), 40))
    _, pol = oracle.findpol(g["intv"])
    assert pol["deg"] == g["deg"]
    oracle.set_rng(0, g["seed"])
    out = oracle.cheblannr(D, g["intv"], g["maxit"], g["tol"], np.cos(np.arange(n) * 0.37), pol)
    assert (out["status"], out["nev"], out["its"]) == (g["status"], g["nev"], g["its"])
    assert rel(out["lam"], g["lam"]) <= 1e-10


@pytest.mark.slow
def test_random_pipelines_against_reference(oracle, reference):
    """Twelve random whole runs (2D and 3D Laplacians of 216 to 1728 rows,
    1 to 4 slices, either bounds mode and DOS type, both random streams)
    through the oracle and the reference build: status, slice ends (1e-12),
    filter types and degrees, eigenvalue counts and eigenvalues (1e-10) as
    the reference's.  Lanczos step counts may differ by whole test cycles
    of 20 steps: the restricted-trace test compares a change with 2e-12,
    and where that change sits within rounding the two builds' dot products
    and tridiagonal eigensolvers (LAPACK DSTEV there) decide differently."""
    rng = np.random.default_rng(3)
    cycles = 0
    for _ in range(12):
        d3 = rng.random() < 0.5
        g = (int(rng.integers(6, 13)),) * 3 if d3 else \
            (int(rng.integers(12, 40)), int(rng.integers(12, 40)), 1)
        top = 12.0 if d3 else 8.0
        a = float(rng.uniform(0.2, top * 0.6))
        b = a + float(rng.uniform(0.1, 1.2))
        spec = RunSpec(a_lo=a, b_hi=b, nslices=int(rng.integers(1, 5)),
                       bounds_mode=int(rng.integers(0, 2)), lmin=0.0, lmax=top,
                       dos_type=int(rng.integers(0, 2)), Mdeg=int(rng.choice([100, 200, 300])),
                       nvec=int(rng.choice([10, 20, 40])), rng_mode=int(rng.integers(0, 2)),
                       seed=int(rng.integers(0, 100)), thresh_int=float(rng.choice([0.6, 0.8])))
        A = laplacian(*g)
        r1, r2 = reference.pipeline(A, spec), oracle.pipeline(A, spec)
        assert r1.status == r2.status
        assert np.max(np.abs(r1.sli - r2.sli)) <= 1e-12 * max(1.0, np.max(np.abs(r1.sli)))
        assert list(r1.ptype) == list(r2.ptype) and list(r1.deg) == list(r2.deg)
        assert list(r1.nev) == list(r2.nev)
        for x, y, i1, i2 in zip(r1.lam, r2.lam, r1.its, r2.its):
            assert (i1 - i2) % 20 == 0
            cycles += i1 != i2
            if len(x):
                assert np.max(np.abs(np.sort(x) - np.sort(y))) <= 1e-10 * np.max(np.abs(x))
    assert cycles <= 3


@pytest.mark.slow
def test_random_matrix_pipelines_against_reference(oracle, reference):
    """Whole runs on matrices other than the constant-coefficient Laplacian:
    random sparse symmetric (800 to 3000 rows, offsets up to 300) and
    random-coefficient 3D Laplacians (8^3 to 12^3), bounds by thick-restart
    Lanczos, KPM or Lanczos DOS, 1 to 3 slices.  Bounds to 1e-12
    (relative), slice ends to 1e-12, filter degrees, eigenvalue counts and
    eigenvalues (1e-10) as the reference build's; step counts up to whole
    convergence-test cycles."""
    from pevsl_b200.problems import random_coef_laplacian, random_sparse_symmetric

    from checkers import Csr
    rng = np.random.default_rng(4)
    for t in range(6):
        if t % 2 == 0:
            n, ia, ja, a = random_sparse_symmetric(int(rng.integers(800, 3000)), 8,
                                                   int(rng.integers(10, 300)),
                                                   int(rng.integers(0, 99)))
        else:
            g = int(rng.integers(8, 13))
            n, ia, ja, a = random_coef_laplacian(g, g, g, seed=int(rng.integers(0, 99)))
        A = Csr(n, ia, ja, a)
        _, lo, hi = reference.lantrbounds(A, 50, 200, 1e-8, np.cos(np.arange(n) * 0.37))
        w = hi - lo
        aa = lo + w * rng.uniform(0.1, 0.6)
        spec = RunSpec(a_lo=aa, b_hi=aa + w * rng.uniform(0.02, 0.1),
                       nslices=int(rng.integers(1, 4)), bounds_mode=1,
                       dos_type=int(rng.integers(0, 2)), Mdeg=200, nvec=20,
                       rng_mode=int(rng.integers(0, 2)), seed=t)
        r1, r2 = reference.pipeline(A, spec), oracle.pipeline(A, spec)
        assert r1.status == r2.status == 0
        scale = max(abs(r1.lmin), abs(r1.lmax))
        assert abs(r1.lmin - r2.lmin) <= 1e-12 * scale and abs(r1.lmax - r2.lmax) <= 1e-12 * scale
        assert np.max(np.abs(r1.sli - r2.sli)) <= 1e-12 * scale
        assert list(r1.deg) == list(r2.deg) and list(r1.nev) == list(r2.nev)
        for x, y, i1, i2 in zip(r1.lam, r2.lam, r1.its, r2.its):
            assert (i1 - i2) % 20 == 0
            if len(x):
                assert np.max(np.abs(np.sort(x) - np.sort(y))) <= 1e-10 * np.max(np.abs(x))
