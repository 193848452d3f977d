"""Parity of the CUDA path with the oracle and the reference's golden outputs.

Every test calls the product through its C-ABI (libpevsl_b200.so via
pevsl_b200) and checks it against the plain-C oracle on the same inputs
and/or the fixtures generated from the reference.  Tolerances (FP64 path):

  SpMV                     1e-14 relative (summation order only)
  random vectors           glibc stream exact; Philox Gaussian 1e-14 relative
                           (device log/sincos vs host libm)
  KPM moments / ecount     1e-12 relative;  npts identical
  slice endpoints          1e-12 relative;  filter degree/type identical
  filter application       1e-11 relative
  bounds (LanTrbounds)     1e-10 relative
  eigenvalues              1e-10 relative;  per-slice counts identical
  residuals                ||Ax - lam x|| < tol = 1e-8 and ||Ax - lam x||/|lam| <= 1e-8
"""
import ctypes as C

import numpy as np
import pytest

import pevsl_b200 as pv
from checkers import Csr, RunSpec, exact_eig_lap, laplacian
from conftest import golden

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def dev_matrix(A: Csr) -> pv.Matrix:
    return pv.Matrix.from_csr(A.n, A.ia, A.ja, A.a)


def random_csr(n, per_row, seed, sym=False):
    rng = np.random.default_rng(seed)
    rows = []
    for i in range(n):
        k = int(per_row[i]) if hasattr(per_row, "__len__") else per_row
        cols = np.sort(rng.choice(n, size=min(k, n), replace=False))
        rows.append(cols)
    ia = np.zeros(n + 1, np.int32)
    ia[1:] = np.cumsum([len(r) for r in rows])
    ja = np.concatenate(rows).astype(np.int32)
    a = rng.standard_normal(len(ja))
    return Csr(n, ia, ja, a)


# ---------------------------------------------------------------- SpMV
def test_matvec_golden(gpu):
    for key, case in golden("matvec_sin.json").items():
        A = laplacian(*case["grid"])
        M = dev_matrix(A)
        y = M.matvec(np.sin(np.arange(A.n, dtype=np.float64)))
        assert rel(y, case["y"]) <= 1e-14, key


@pytest.mark.parametrize("per_row", [1, 3, 7, 13, 29, 70, "ragged", "ragged_short"])
def test_spmv_lane_widths(gpu, oracle, per_row):
    """Rows of 1..70 entries select the CSR-stream kernel (short rows) or a
    lane width of 1..32 threads per row; 'ragged' mixes empty and long rows."""
    n = 3001
    if per_row in ("ragged", "ragged_short"):
        rng = np.random.default_rng(5)
        pr = rng.integers(0, 120 if per_row == "ragged" else 40, size=n)
        pr[::7] = 0
        pr[-40:] = 0
        A = random_csr(n, pr, 1)
    else:
        A = random_csr(n, per_row, per_row)
    x = np.random.default_rng(2).standard_normal(n)
    y = dev_matrix(A).matvec(x)
    ref = oracle.matvec(A, x)
    assert np.max(np.abs(y - ref)) <= 1e-14 * max(1.0, np.max(np.abs(ref))) * 8


@pytest.mark.parametrize("lanes", [0, 1, 2, 4, 8, 16, 32])
def test_every_spmv_kernel_on_one_matrix(gpu, oracle, monkeypatch, lanes):
    """PEVSL_B200_LANES forces each kernel variant on the same ragged matrix;
    the CSR-stream kernel (lanes 0) sums in the reference's order without
    fused multiply-adds, so it matches the sequential row loop exactly."""
    monkeypatch.setenv("PEVSL_B200_LANES", str(lanes))
    rng = np.random.default_rng(11)
    pr = rng.integers(0, 300, size=2000)
    pr[5:9] = 0
    A = random_csr(2000, pr, 3)
    x = rng.standard_normal(2000)
    y = dev_matrix(A).matvec(x)
    ref = oracle.matvec(A, x)
    if lanes == 0:
        assert np.array_equal(y, ref)
    else:
        assert np.max(np.abs(y - ref)) <= 1e-13 * max(1.0, np.max(np.abs(ref)))


def test_spmv_empty_and_tiny(gpu, oracle):
    for n in (1, 2, 33):
        A = laplacian(n, 1, 1) if n > 1 else Csr(1, np.array([0, 1], np.int32),
                                                 np.array([0], np.int32), np.array([2.5]))
        x = np.linspace(-1, 1, n)
        assert rel(dev_matrix(A).matvec(x), oracle.matvec(A, x)) <= 1e-15


# ---------------------------------------------------------------- vectors / RNG
def test_parvec_blas(gpu):
    lib = pv.load()
    n = 100003
    rng = np.random.default_rng(0)
    xa, ya = rng.standard_normal(n), rng.standard_normal(n)
    x, y = pv.Vector(n, xa), pv.Vector(n, ya)
    t = C.c_double()
    lib.pEVSL_ParvecDot(C.byref(x.pv), C.byref(y.pv), C.byref(t))
    assert abs(t.value - xa @ ya) <= 1e-12 * np.sqrt(n)
    lib.pEVSL_ParvecNrm2(C.byref(x.pv), C.byref(t))
    assert abs(t.value - np.linalg.norm(xa)) <= 1e-13 * np.linalg.norm(xa)
    lib.pEVSL_ParvecSum(C.byref(x.pv), C.byref(t))
    assert abs(t.value - xa.sum()) <= 1e-11
    lib.pEVSL_ParvecAxpy(0.5, C.byref(x.pv), C.byref(y.pv))
    assert rel(y.get(), ya + 0.5 * xa) <= 1e-15
    lib.pEVSL_ParvecScal(C.byref(y.pv), -2.0)
    assert rel(y.get(), -2.0 * (ya + 0.5 * xa)) <= 1e-15
    lib.pEVSL_ParvecCopy(C.byref(x.pv), C.byref(y.pv))
    assert np.array_equal(y.get(), xa)
    lib.pEVSL_ParvecSetScalar(C.byref(y.pv), 3.0)
    assert np.all(y.get() == 3.0)
    lib.pEVSL_ParvecSetZero(C.byref(y.pv))
    assert np.all(y.get() == 0.0)
    # managed memory: the host reads the data pointer directly, as
    # TESTS0/Matvec/test1.c does
    host = np.ctypeslib.as_array(C.cast(x.pv.data, C.POINTER(C.c_double)), shape=(n,))
    assert np.array_equal(host, xa)
    assert lib.pEVSL_B200_LastError() == 0


def test_parvecs_gemv_gemtv(gpu):
    lib = pv.load()
    n, k = 5000, 37
    rng = np.random.default_rng(1)
    Vh = rng.standard_normal((k, n))
    X = pv.Parvecs()
    lib.pEVSL_ParvecsCreate(n, k, n, n, 0, 1, C.byref(X))
    lib.pEVSL_B200_Memcpy(X.data, Vh.ctypes.data, Vh.nbytes)
    v = pv.Vector(n, rng.standard_normal(n))
    w = np.zeros(k)
    lib.pEVSL_ParvecsGemtv(1.0, C.byref(X), k, C.byref(v.pv), 0.0,
                           w.ctypes.data_as(C.POINTER(C.c_double)))
    assert rel(w, Vh @ v.get()) <= 1e-13
    coef = rng.standard_normal(k)
    y0 = v.get()
    lib.pEVSL_ParvecsGemv(-1.0, C.byref(X), k, coef.ctypes.data_as(C.POINTER(C.c_double)), 1.0,
                          C.byref(v.pv))
    assert rel(v.get(), y0 - Vh.T @ coef) <= 1e-13
    lib.pEVSL_ParvecsFree(C.byref(X))


@pytest.mark.parametrize("n,k,m", [(10007, 53, 70), (777, 300, 129), (65, 4, 1), (3, 17, 64)])
def test_dense_products_on_tensor_cores(gpu, n, k, m):
    """The DMMA products of the solvers (Ritz vectors U = V Y, Gram
    matrices C = V' W) against numpy's FP64 products on ragged shapes (tiles
    of 64 and panels of 16 cut through rows, columns and the inner
    dimension), within 1e-13 of the largest entry, and identical bits on a
    second call (fixed reduction order)."""
    lib = pv.load()
    for f in (lib.pEVSL_B200_GemmNN, lib.pEVSL_B200_GemmTN):
        f.argtypes = [C.c_long, C.c_int, C.c_int, C.c_void_p, C.c_long, C.c_void_p, C.c_long,
                      C.c_void_p, C.c_long]
    rng = np.random.default_rng(n + k + m)
    ldv = n + 3
    V = rng.standard_normal((k, ldv))   # column-major n x k with leading dimension ldv
    Y = rng.standard_normal((m, k))     # column-major k x m
    W = rng.standard_normal((m, ldv))   # column-major n x m
    dV, dY, dW = pv.Vector(k * ldv, V.ravel()), pv.Vector(m * k, Y.ravel()), pv.Vector(m * ldv, W.ravel())
    dU, dC = pv.Vector(m * n), pv.Vector(k * m)
    outs = []
    for _ in range(2):
        assert lib.pEVSL_B200_GemmNN(n, k, m, dV.pv.data, ldv, dY.pv.data, k, dU.pv.data, n) == 0
        assert lib.pEVSL_B200_GemmTN(n, k, m, dV.pv.data, ldv, dW.pv.data, ldv, dC.pv.data, k) == 0
        assert lib.pEVSL_B200_Sync() == 0
        outs.append((dU.get().reshape(m, n), dC.get().reshape(m, k)))
    Vn, Wn = V[:, :n].T, W[:, :n].T
    U_ref, C_ref = Vn @ Y.T, Vn.T @ Wn
    assert np.max(np.abs(outs[0][0].T - U_ref)) <= 1e-13 * np.max(np.abs(U_ref))
    assert np.max(np.abs(outs[0][1].T - C_ref)) <= 1e-13 * np.max(np.abs(C_ref))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
    for x in (dV, dY, dW, dU, dC):
        x.free()


def test_rng_glibc_stream_matches_reference_formula(gpu, oracle):
    lib = pv.load()
    n = 7777
    pv.set_rng(pv.RNG_GLIBC, 5)
    v = pv.Vector(n)
    lib.pEVSL_ParvecRand(C.byref(v.pv))
    got = v.get()
    oracle.lib.orc_set_rng(0, C.c_uint64(5))
    exp = np.zeros(n)
    oracle.lib.orc_rand_vector(exp.ctypes.data_as(C.c_void_p), n)
    assert np.array_equal(got, exp)
    assert np.all(np.abs(got) <= 1.0)


def test_rng_gauss_matches_oracle(gpu, oracle):
    lib = pv.load()
    n = 10001
    pv.set_rng(pv.RNG_GAUSS, 1234)
    oracle.lib.orc_set_rng(1, C.c_uint64(1234))
    for draw in range(3):
        v = pv.Vector(n)
        lib.pEVSL_ParvecRand(C.byref(v.pv))
        exp = np.zeros(n)
        oracle.lib.orc_rand_vector(exp.ctypes.data_as(C.c_void_p), n)
        assert np.max(np.abs(v.get() - exp)) <= 1e-14 * np.max(np.abs(exp)), draw
    assert int(lib.pEVSL_B200_RngDraws()) == 3
    assert abs(exp.mean()) < 0.05 and abs(exp.std() - 1.0) < 0.05


# ---------------------------------------------------------------- KPM, filter
@pytest.mark.parametrize("mode", ["glibc", "gauss"])
def test_kpm_golden(gpu, mode):
    g = golden("lap20_kpm.json")
    case = g["cases"][mode]
    A = dev_matrix(laplacian(*g["grid"]))
    with pv.Instance(A) as ev:
        pv.set_rng(0 if mode == "glibc" else 1, g["seed"])
        r, mu, ec = ev.kpmdos(g["Mdeg"], g["damping"], g["nvec"], g["intv"])
    assert r == 0
    assert rel(mu, case["mu"]) <= 1e-12
    assert abs(ec - case["ecount"]) <= 1e-10 * abs(case["ecount"])
    assert int(10 * ec) == case["npts"]
    r, sli = pv.spslicer_kpm(mu, g["Mdeg"], g["intv"], 5, int(10 * ec))
    assert r == 0 and rel(sli, case["sli"]) <= 1e-12


def test_kpm_more_than_one_block(gpu, oracle):
    """nvec = 150 runs as blocks of 64 + 64 + 22 vectors."""
    A = laplacian(9, 10, 11)
    intv = [1.0, 3.0, 0.0, 12.0]
    with pv.Instance(dev_matrix(A)) as ev:
        pv.set_rng(pv.RNG_GAUSS, 77)
        r, mu, ec = ev.kpmdos(60, 2, 150, intv)
    oracle.set_rng(1, 77)
    _, mu_o, ec_o = oracle.kpmdos(A, 60, 2, 150, intv)
    assert r == 0 and rel(mu, mu_o) <= 1e-12 and abs(ec - ec_o) <= 1e-10 * abs(ec_o)


def test_chebav_matches_oracle(gpu, oracle):
    A = laplacian(20, 20, 20)
    for intv in ([0.6, 0.7482233502538076, 0.0, 12.0], [0.0, 0.5, 0.0, 12.0], [11.0, 12.0, 0, 12]):
        r, f = pv.findpol(intv)
        v = np.cos(np.arange(A.n) * 0.1)
        with pv.Instance(dev_matrix(A)) as ev:
            y = ev.chebav(f, v)
        yo = oracle.chebav(A, dict(deg=f.deg, cc=f.cc, dd=f.dd, mu=f.mu), v)
        assert rel(y, yo) <= 1e-11, intv


# ---------------------------------------------------------------- Lanczos pieces
def test_lantrbounds_golden(gpu):
    g = golden("lanczos_cases.json")
    A = dev_matrix(laplacian(*g["grid"]))
    b = g["lantrbounds"]
    v0 = np.cos(np.arange(A.n, dtype=np.float64))
    for bt, c in b["cases"].items():
        with pv.Instance(A) as ev:
            pv.set_rng(pv.RNG_GAUSS, 3)
            r, lo, hi = ev.lantrbounds(b["lanm"], b["maxit"], b["tol"], v0, int(bt))
        assert r == c["status"] == 0
        assert abs(lo - c["lmin"]) <= 1e-10 * max(1, abs(c["lmin"]))
        assert abs(hi - c["lmax"]) <= 1e-10 * abs(c["lmax"])


def test_landos_golden(gpu):
    g = golden("lanczos_cases.json")
    d = g["landos"]
    A = dev_matrix(laplacian(*g["grid"]))
    with pv.Instance(A) as ev:
        pv.set_rng(pv.RNG_GAUSS, d["seed"])
        r, xd, yd, ne = ev.landos(d["nvec"], d["msteps"], d["npts"], d["intv"])
    assert r == 0
    assert rel(xd, d["xdos"]) <= 1e-15
    assert rel(yd, d["ydos"]) <= 1e-10
    assert abs(ne - d["neig"]) <= 1e-10 * abs(d["neig"])
    assert rel(pv.spslicer_lan(xd, yd, 4), d["sli4"]) <= 1e-12


def test_cheblannr_slice_matches_oracle(gpu, oracle):
    A = laplacian(20, 20, 20)
    intv = [0.6, 0.7482233502538076, 0.0, 12.0]
    r, f = pv.findpol(intv)
    v0 = np.sin(np.arange(A.n) * 0.7)
    with pv.Instance(dev_matrix(A)) as ev:
        out = ev.cheblannr(intv, 300, 1e-8, v0, f, want_vectors=True)
    ref = oracle.cheblannr(A, intv, 300, 1e-8, v0, dict(deg=f.deg, type=f.type, gam=f.gam,
                                                         bar=f.bar, cc=f.cc, dd=f.dd, mu=f.mu))
    assert out["status"] == 0
    assert out["nev"] == ref["nev"] == 21 and out["its"] == ref["its"]
    assert rel(out["lam"], ref["lam"]) <= 1e-10
    assert np.all(out["res"] < 1e-8)
    # eigenvectors: residuals recomputed on the host from the returned vectors
    W = out["W"]
    for lam, w in zip(out["lam"], W):
        r = oracle.matvec(A, w) - lam * w
        assert np.linalg.norm(r) / abs(lam) <= 1e-8 and abs(np.linalg.norm(w) - 1) < 1e-12


def test_breakdown_restart_golden(gpu):
    g = golden("breakdown_case.json")
    n = g["n"]
    D = Csr(n, np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32),
            np.repeat(np.arange(1.0, 11.0), 40))
    r, f = pv.findpol(g["intv"])
    assert f.deg == g["deg"]
    with pv.Instance(dev_matrix(D)) as ev:
        pv.set_rng(pv.RNG_GLIBC, g["seed"])
        out = ev.cheblannr(g["intv"], g["maxit"], g["tol"], np.cos(np.arange(n) * 0.37), f)
    assert (out["status"], out["nev"], out["its"]) == (g["status"], g["nev"], g["its"])
    assert rel(out["lam"], g["lam"]) <= 1e-10


# ---------------------------------------------------------------- whole runs
def check_pipeline(r: pv.SliceResult, g, grid):
    assert r.status == g["status"] == 0
    assert abs(r.lmin - g["lmin"]) <= 1e-10 * max(1, abs(g["lmin"]))
    assert abs(r.lmax - g["lmax"]) <= 1e-10 * abs(g["lmax"])
    assert abs(r.ecount - g["ecount"]) <= 1e-10 * abs(g["ecount"])
    assert r.npts == g["npts"]
    assert rel(r.sli, g["sli"]) <= 1e-12
    assert r.deg == g["deg"] and r.ptype == g["ptype"]
    assert r.nev == g["nev"], (r.nev, g["nev"])
    assert r.its == g["its"]
    for sl in range(len(g["nev"])):
        lam = r.lam[sl]
        assert rel(lam, g["lam"][sl]) <= 1e-10
        assert np.all(r.res[sl] < g["spec"]["tol"])
        assert np.all(r.res[sl] / np.abs(lam) <= 1e-8)
        ex = exact_eig_lap(*grid, g["sli"][sl], g["sli"][sl + 1])
        assert len(ex) == len(lam) and np.max(np.abs(lam - ex)) <= 1e-12


@pytest.mark.parametrize("name", ["lap10_kpm_gauss", "lap30x30_kpm_glibc", "lap12_landos_gauss",
                                  "lap20_readme_glibc", "lap20_lantr_gauss"])
def test_pipeline_golden(gpu, name):
    g = golden("pipelines.json")[name]
    A = dev_matrix(laplacian(*g["grid"]))
    r = pv.solve_interval(A, pv.SliceRun(**g["spec"]))
    check_pipeline(r, g, g["grid"])


# ---------------------------------------------------------------- error paths
def test_error_codes(gpu):
    A = dev_matrix(laplacian(6, 6, 6))
    with pv.Instance(A) as ev:
        r, _, _ = ev.kpmdos(20, 1, 2, [1.0, 0.5, 0.0, 12.0])
        assert r == -1
        r, _, _ = ev.kpmdos(20, 1, 2, [13.0, 14.0, 0.0, 12.0])
        assert r == -1
        r, f = pv.findpol([1.0, 2.0, 0.0, 12.0])
        out = ev.cheblannr([2.0, 1.0, 0.0, 12.0], 50, 1e-8, np.ones(A.n), f)
        assert out["status"] == 0 and out["nev"] == 0
        bad = pv.Filter(f.type, f.deg, 1.5, f.bar, f.cc, f.dd, f.mu)
        out = ev.cheblannr([1.0, 2.0, 0.0, 12.0], 50, 1e-8, np.ones(A.n), bad)
        assert out["status"] == -1
        v = np.ones(A.n)
        v[3] = np.nan
        out = ev.cheblannr([1.0, 2.0, 0.0, 12.0], 50, 1e-8, v, f)
        assert out["status"] == pv.ERR_NONFINITE
    assert pv.findpol([1.0, 0.5, 0.0, 12.0])[0] == -1
    assert pv.spslicer_kpm(np.ones(11), 10, [3.0, 1.0, 0, 12], 3, 40)[0] == -1


def test_user_matvec_callback(gpu):
    """pEVSL_SetAMatvec with a callback that receives device pointers; the
    unfused path must give the fused path's results."""
    lib = pv.load()
    A = laplacian(12, 12, 12)
    M = dev_matrix(A)
    intv = [1.0, 1.6, 0.0, 12.0]
    r, f = pv.findpol(intv)
    v0 = np.cos(np.arange(A.n) * 0.3)

    @pv.MVFUNC
    def mv(x, y, data):
        lib.pEVSL_ParcsrMatvec0(x, y, C.addressof(M.A))

    with pv.Instance(M) as ev:
        fused = ev.cheblannr(intv, 300, 1e-8, v0, f)
        pv.set_rng(pv.RNG_GAUSS, 4)
        _, mu_f, ec_f = ev.kpmdos(40, 1, 8, intv)
    with pv.Instance(None) as ev:
        lib.pEVSL_SetProbSizes(ev.p, A.n, A.n, 0)
        lib.pEVSL_SetAMatvec(ev.p, mv, None)
        cb = ev.cheblannr(intv, 300, 1e-8, v0, f)
        pv.set_rng(pv.RNG_GAUSS, 4)
        _, mu_c, ec_c = ev.kpmdos(40, 1, 8, intv)
    assert cb["status"] == 0 and cb["nev"] == fused["nev"] and cb["its"] == fused["its"]
    assert rel(cb["lam"], fused["lam"]) <= 1e-10
    assert rel(mu_c, mu_f) <= 1e-12 and abs(ec_c - ec_f) <= 1e-10 * abs(ec_f)


# ---------------------------------------------------------------- batched slices
@pytest.mark.parametrize("name", ["lap10_kpm_gauss", "lap30x30_kpm_glibc", "lap12_landos_gauss",
                                  "lap20_readme_glibc", "lap20_lantr_gauss"])
def test_batched_pipeline_golden_and_bitwise(gpu, name):
    """All slices in lockstep (pEVSL_B200_ChebLanNrBatch): same goldens, and
    bit-for-bit the results of the slice-by-slice drop-in path (2, 3 and 5
    slices: batch widths 2, 4 and 8 with padded entries)."""
    g = golden("pipelines.json")[name]
    A = dev_matrix(laplacian(*g["grid"]))
    rb = pv.solve_interval(A, pv.SliceRun(**g["spec"]), batched=True)
    check_pipeline(rb, g, g["grid"])
    rs = pv.solve_interval(A, pv.SliceRun(**g["spec"]), batched=False)
    assert rb.its == rs.its and rb.nev == rs.nev
    for a, b in zip(rb.lam, rs.lam):
        assert np.array_equal(a, b)
    for a, b in zip(rb.res, rs.res):
        assert np.array_equal(a, b)


def test_batch_mixed_statuses(gpu):
    """Invalid interval (no pairs, status 0), filter centre outside [-1,1]
    (status -1) and valid slices in one batch."""
    A = laplacian(10, 10, 10)
    M = dev_matrix(A)
    good = [[0.6, 1.0, 0.0, 12.0], [1.0, 1.5, 0.0, 12.0]]
    filters = [pv.findpol(iv)[1] for iv in good]
    bad = pv.Filter(filters[0].type, filters[0].deg, 2.0, filters[0].bar, filters[0].cc,
                    filters[0].dd, filters[0].mu)
    intvs = [good[0], [1.5, 1.0, 0.0, 12.0], good[1], good[0]]
    fl = [filters[0], filters[0], filters[1], bad]
    v0 = np.cos(np.arange(A.n) * 0.2)
    with pv.Instance(M) as ev:
        r, outs = pv.cheblannr_batch(ev, intvs, [300] * 4, 1e-8, v0, fl)
        single = [ev.cheblannr(iv, 300, 1e-8, v0, f) for iv, f in zip(good, filters)]
    assert r == -1
    assert [o["status"] for o in outs] == [0, 0, 0, -1]
    assert outs[1]["nev"] == 0
    for o, s in zip([outs[0], outs[2]], single):
        assert o["nev"] == s["nev"] and o["its"] == s["its"]
        assert np.array_equal(o["lam"], s["lam"])
        ex = exact_eig_lap(10, 10, 10, *(good[0][:2] if s is single[0] else good[1][:2]))
        assert len(ex) == o["nev"]


# ---------------------------------------------------------------- mixed precision
@pytest.mark.parametrize("name", ["lap20_lantr_gauss", "lap10_kpm_gauss", "lap20_readme_glibc"])
def test_mixed_precision_counts_and_residuals(gpu, name):
    """FP32 filter + FP32 KPM moments, FP64 basis / reorthogonalisation /
    one FP64 filtered Rayleigh-Ritz sweep (slices whose refined pairs miss
    tol are solved again in FP64): every slice holds exactly the eigenvalues
    of A inside it, each within 1e-10 (relative) of the exact value, with
    ||Ax - lam x|| < 1e-8 and ||Ax - lam x||/|lam| <= 1e-8.  The FP32 KPM
    moves the slice ends by at most 1e-5 (relative); where the slices are
    the FP64 run's, so are the per-slice counts."""
    g = golden("pipelines.json")[name]
    A = dev_matrix(laplacian(*g["grid"]))
    r = pv.solve_interval(A, pv.SliceRun(**g["spec"]), batched=True, precision=pv.PREC_MIXED)
    assert r.status == 0
    assert 0 <= r.fallbacks <= len(r.nev)
    assert rel(r.sli, g["sli"]) <= 1e-5, (r.sli, g["sli"])
    if rel(r.sli, g["sli"]) <= 1e-12:
        assert r.nev == g["nev"]
    for sl in range(len(r.nev)):
        lam = r.lam[sl]
        assert np.all(r.res[sl] / np.abs(lam) <= 1e-8) and np.all(r.res[sl] < 1e-8)
        ex = exact_eig_lap(*g["grid"], r.sli[sl], r.sli[sl + 1])
        assert len(lam) == len(ex), (sl, len(lam), len(ex))
        assert np.max(np.abs(lam - ex) / np.abs(ex)) <= 1e-10


def test_mixed_precision_per_eigenvalue_against_fp64_run(gpu):
    """The mixed form against the FP64 run on the same inputs, eigenvalue by
    eigenvalue (README matrix, thick-restart bounds, Gaussian stream): every
    slice whose ends the FP32 moments leave in place has the FP64 run's
    count, and each of its eigenvalues agrees with the FP64 run's within
    1e-10 relative (the largest error is reported in the message)."""
    g = golden("pipelines.json")["lap20_lantr_gauss"]
    A = dev_matrix(laplacian(*g["grid"]))
    spec = pv.SliceRun(**g["spec"])
    r64 = pv.solve_interval(A, spec, batched=True, precision=pv.PREC_FP64)
    r32 = pv.solve_interval(A, spec, batched=True, precision=pv.PREC_MIXED)
    assert r64.status == 0 and r32.status == 0
    worst = 0.0
    for sl in range(len(r64.nev)):
        if rel(r32.sli[sl:sl + 2], r64.sli[sl:sl + 2]) > 1e-12:
            continue  # the FP32 moments moved this slice's ends
        assert r32.nev[sl] == r64.nev[sl]
        err = np.abs(r32.lam[sl] - r64.lam[sl]) / np.abs(r64.lam[sl])
        worst = max(worst, float(err.max()))
    assert worst <= 1e-10, f"largest per-eigenvalue error against FP64: {worst:.3e}"


# ---------------------------------------------------------------- batching forms
def _lap_slices(grid, a, b, ns, seed=3):
    """Bounds from the analytic spectrum, slices evenly spaced, filters."""
    L = laplacian(*grid)
    ev = exact_eig_lap(*grid, 0.0, 100.0)
    lmin, lmax = ev[0] - 1e-6, ev[-1] + 1e-6
    edges = np.linspace(a, b, ns + 1)
    intvs = [[edges[i], edges[i + 1], lmin, lmax] for i in range(ns)]
    fl = [pv.findpol(iv)[1] for iv in intvs]
    return pv.Matrix.from_csr(L.n, L.ia, L.ja, L.a), intvs, fl


def test_filter_forms_bit_identical(gpu):
    """One launch per degree, one persistent launch for all degrees, and the
    launches replayed from a CUDA graph give the same bits (same per-row
    arithmetic, any schedule)."""
    lib = pv.load()
    M, intvs, fl = _lap_slices((14, 13, 12), 0.5, 1.3, 4)
    v = np.cos(np.arange(M.n) * 0.37)
    outs = []
    try:
        for form in (0, 1, 2):
            assert lib.pEVSL_B200_SetFilterForm(form) == 0
            with pv.Instance(M) as ev:
                r, o = pv.cheblannr_batch(ev, intvs, [150] * 4, 1e-8, v, fl)
            assert r == 0
            outs.append(o)
    finally:
        lib.pEVSL_B200_SetFilterForm(-1)
    for other in outs[1:]:
        for a, b in zip(outs[0], other):
            assert a["nev"] == b["nev"] and a["its"] == b["its"]
            assert np.array_equal(a["lam"], b["lam"]) and np.array_equal(a["res"], b["res"])


def test_persistent_barrier_timeout_reports_error(gpu):
    """The persistent filter's grid barrier gives up after its spin limit:
    with the arrival counter preset so that no arrival completes it and a
    short limit (4096 polls, well under a millisecond), the kernel returns,
    the lockstep call reports PEVSL_ERR_CUDA right after that filter
    application, and the next call on the same context runs normally and
    gives the bits of the default form."""
    lib = pv.load()
    lib.pEVSL_B200_SetBarrierSpins.argtypes = [C.c_uint]
    lib.pEVSL_B200_SeedBarrierArrivals.argtypes = [C.c_uint]
    M, intvs, fl = _lap_slices((14, 13, 12), 0.5, 1.3, 4)
    v = np.cos(np.arange(M.n) * 0.37)
    with pv.Instance(M) as ev:
        r, ref = pv.cheblannr_batch(ev, intvs, [150] * 4, 1e-8, v, fl)
    assert r == 0
    try:
        assert lib.pEVSL_B200_SetFilterForm(1) == 0
        assert lib.pEVSL_B200_SetBarrierSpins(4096) == 0
        assert lib.pEVSL_B200_SeedBarrierArrivals(1 << 30) == 0
        with pv.Instance(M) as ev:
            r, outs = pv.cheblannr_batch(ev, intvs, [150] * 4, 1e-8, v, fl)
        assert r == pv.ERR_CUDA
        assert lib.pEVSL_B200_SetBarrierSpins(0) == 0
        with pv.Instance(M) as ev:
            r, again = pv.cheblannr_batch(ev, intvs, [150] * 4, 1e-8, v, fl)
        assert r == 0
    finally:
        lib.pEVSL_B200_SetBarrierSpins(0)
        lib.pEVSL_B200_SetFilterForm(-1)
    for a, b in zip(ref, again):
        assert a["nev"] == b["nev"] and a["its"] == b["its"]
        assert np.array_equal(a["lam"], b["lam"])


def test_multi_problem_equals_separate(gpu):
    """pEVSL_B200_ChebLanNrMulti over problems of different sizes, slice
    counts and filter degrees gives every slice the bits of solving its
    problem alone, and the exact per-slice counts."""
    specs = [((11, 10, 9), 0.6, 1.4, 3), ((30, 29, 1), 0.3, 0.7, 2), ((9, 9, 9), 1.0, 2.2, 4)]
    probs, sep = [], []
    insts = []
    for grid, a, b, ns in specs:
        M, intvs, fl = _lap_slices(grid, a, b, ns)
        v = np.sin(np.arange(M.n) * 0.11 + ns)
        ev = pv.Instance(M)
        insts.append(ev)
        r, o = pv.cheblannr_batch(ev, intvs, [160] * ns, 1e-8, v, fl)
        assert r == 0
        sep.append((grid, intvs, o))
        probs.append((ev, intvs, [160] * ns, 1e-8, v, fl))
    r, multi = pv.cheblannr_multi(probs)
    assert r == 0
    for (grid, intvs, o1), o2 in zip(sep, multi):
        for iv, a, b in zip(intvs, o1, o2):
            assert a["nev"] == b["nev"] and a["its"] == b["its"]
            assert np.array_equal(a["lam"], b["lam"])
            ex = exact_eig_lap(*grid, iv[0], iv[1])
            assert b["nev"] == len(ex)
            assert np.max(np.abs(b["lam"] - ex)) <= 1e-10 * np.max(np.abs(ex))
    for ev in insts:
        ev.close()


def test_interleaved_filter_bit_identical(gpu):
    """Slices of one matrix of at least 2^16 rows run the interleaved filter
    (row-interleaved vectors, one gather for all slices); every slice gets
    the bits of solving it alone (one-vector kernel) and the exact count."""
    grid = (41, 41, 41)  # 68 921 rows
    M, intvs, fl = _lap_slices(grid, 0.3, 0.36, 3)
    assert M.n >= 65536
    v = np.cos(np.arange(M.n) * 0.37)
    with pv.Instance(M) as ev:
        r, batch = pv.cheblannr_batch(ev, intvs, [200] * 3, 1e-8, v, fl)
    assert r == 0
    for iv, f, b in zip(intvs, fl, batch):
        with pv.Instance(M) as ev:
            r, (one,) = pv.cheblannr_batch(ev, [iv], [200], 1e-8, v, [f])
        assert r == 0
        assert one["nev"] == b["nev"] and one["its"] == b["its"]
        assert np.array_equal(one["lam"], b["lam"]) and np.array_equal(one["res"], b["res"])
        ex = exact_eig_lap(*grid, iv[0], iv[1])
        assert b["nev"] == len(ex)
        assert np.max(np.abs(b["lam"] - ex)) <= 1e-10 * np.max(np.abs(ex))


def test_interleaved_groups_one_after_another_bit_identical(gpu, monkeypatch):
    """Five slices of one matrix in lockstep with the interleaved groups
    capped at two slices (PEVSL_B200_IL_MAXS=2: groups of 2, 2 and 1, each
    group's whole filter application before the next, as for matrices whose
    wider groups would not stay in L2): every slice gets the bits of solving
    it alone and the exact count."""
    monkeypatch.setenv("PEVSL_B200_IL_MAXS", "2")
    grid = (41, 41, 41)
    M, intvs, fl = _lap_slices(grid, 0.3, 0.38, 5)
    v = np.cos(np.arange(M.n) * 0.37)
    with pv.Instance(M) as ev:
        r, batch = pv.cheblannr_batch(ev, intvs, [200] * 5, 1e-8, v, fl)
    assert r == 0
    monkeypatch.delenv("PEVSL_B200_IL_MAXS")
    for iv, f, b in zip(intvs, fl, batch):
        with pv.Instance(M) as ev:
            r, (one,) = pv.cheblannr_batch(ev, [iv], [200], 1e-8, v, [f])
        assert r == 0
        assert one["nev"] == b["nev"] and one["its"] == b["its"]
        assert np.array_equal(one["lam"], b["lam"]) and np.array_equal(one["res"], b["res"])
        ex = exact_eig_lap(*grid, iv[0], iv[1])
        assert b["nev"] == len(ex)


def test_interleaved_filter_plain_entries_bit_identical(gpu):
    """The interleaved kernel on a matrix without packed entries (random
    edge coefficients: 270 641 distinct values), filters of degrees 225,
    282 and 276 (the filter sum updated every third degree, slices past
    their own degree adding zeros): every slice gets the bits of solving it
    alone, and the counts of the reference build's ChebLanNr on the same
    inputs (run on the CPU: nev 6, 9, 6), residuals <= 1e-8.  The degrees
    are the reference's (findpol_cases.json holds these slices)."""
    from pevsl_b200.problems import random_coef_laplacian
    n, ia, ja, a = random_coef_laplacian(41, 41, 41, seed=3)
    M = pv.Matrix.from_csr(n, ia, ja, a)
    edges = [0.10, 0.123, 0.143, 0.165]
    intvs = [[edges[i], edges[i + 1], 0.0, 24.0] for i in range(3)]  # Gershgorin: 22.8
    fl = [pv.findpol(iv)[1] for iv in intvs]
    assert [f.deg for f in fl] == [225, 282, 276]
    v = np.cos(np.arange(n) * 0.37)
    with pv.Instance(M) as ev:
        r, batch = pv.cheblannr_batch(ev, intvs, [300] * 3, 1e-8, v, fl)
    assert r == 0
    for iv, f, b, cnt in zip(intvs, fl, batch, [6, 9, 6]):
        with pv.Instance(M) as ev:
            r, (one,) = pv.cheblannr_batch(ev, [iv], [300], 1e-8, v, [f])
        assert r == 0
        assert one["nev"] == b["nev"] == cnt and one["its"] == b["its"]
        assert np.array_equal(one["lam"], b["lam"]) and np.array_equal(one["res"], b["res"])
        assert np.all(b["res"] < 1e-8) and np.all(b["res"] / np.abs(b["lam"]) <= 1e-8)
    M.free()


def _banded_heavy_matrix(n, seed):
    """Symmetric packed-eligible matrix: 6 random off-diagonals per row within
    +-30000 columns, values from a set of 64, and heavy rows of 1500
    entries: one alone and four adjacent ones."""
    rng = np.random.default_rng(seed)
    vals = np.round(rng.standard_normal(64), 3)
    r, c = [], []
    for _ in range(3):
        off = rng.integers(1, 30000, size=n)
        rows = np.arange(n)
        keep = rows + off < n
        r.append(rows[keep])
        c.append(rows[keep] + off[keep])
    h0 = n // 2 - (n // 2) % 4
    for h in (n // 5, h0, h0 + 1, h0 + 2, h0 + 3):
        cols = np.unique(rng.integers(max(0, h - 30000), min(n, h + 30000), size=1600))
        cols = cols[cols != h][:1500]
        r.append(np.full(len(cols), h))
        c.append(cols)
    r, c = np.concatenate(r), np.concatenate(c)
    key = np.unique(np.minimum(r, c) * n + np.maximum(r, c))
    r, c = key // n, key % n
    v = vals[rng.integers(0, 64, size=len(r))]
    rows = np.concatenate([r, c, np.arange(n)])
    cols = np.concatenate([c, r, np.arange(n)])
    vv = np.concatenate([v, v, np.full(n, 40.0)])
    order = np.lexsort((cols, rows))
    rows, cols, vv = rows[order], cols[order], vv[order]
    ia = np.zeros(n + 1, np.int32)
    np.add.at(ia, rows + 1, 1)
    ia = np.cumsum(ia).astype(np.int32)
    return Csr(n, ia, cols.astype(np.int32), vv.astype(np.float64))


def test_interleaved_filter_heavy_rows_bit_identical(gpu):
    """The interleaved filter on a scattered matrix with heavy rows (the
    lanes of a row walk up to 1500 entries while their neighbours walk 7):
    three slices in lockstep give every slice the bits of solving it alone
    with the one-vector kernel, after 40 Lanczos steps of degree-60
    filters."""
    A = _banded_heavy_matrix(70001, 5)
    M = dev_matrix(A)
    rows = np.repeat(np.arange(A.n), np.diff(A.ia))
    rad = np.bincount(rows, weights=np.abs(A.a), minlength=A.n) - 40.0
    lmin, lmax = 40.0 - rad.max() - 1.0, 40.0 + rad.max() + 1.0
    edges = np.linspace(39.0, 41.0, 4)
    intvs = [[edges[i], edges[i + 1], lmin, lmax] for i in range(3)]
    fl = [pv.findpol(iv, deg_in=61)[1] for iv in intvs]
    v = np.cos(np.arange(A.n) * 0.37)
    with pv.Instance(M) as ev:
        r, batch = pv.cheblannr_batch(ev, intvs, [40] * 3, 1e-8, v, fl)
    for iv, f, b in zip(intvs, fl, batch):
        with pv.Instance(M) as ev:
            r1, (one,) = pv.cheblannr_batch(ev, [iv], [40], 1e-8, v, [f])
        assert one["status"] == b["status"] and one["nev"] == b["nev"] and one["its"] == b["its"]
        if b["status"] == 0:
            assert np.array_equal(one["lam"], b["lam"]) and np.array_equal(one["res"], b["res"])
    M.free()


def test_multi_problem_with_interleaved_group(gpu):
    """A lockstep group that mixes a problem above 2^16 rows (interleaved)
    with small problems (grid-interleaved batch kernel) gives every slice
    the bits of solving its problem alone."""
    specs = [((41, 41, 41), 0.3, 0.34, 2), ((11, 10, 9), 0.6, 1.4, 3)]
    probs, sep, insts = [], [], []
    for grid, a, b, ns in specs:
        M, intvs, fl = _lap_slices(grid, a, b, ns)
        v = np.sin(np.arange(M.n) * 0.11 + ns)
        ev = pv.Instance(M)
        insts.append((ev, M))
        r, o = pv.cheblannr_batch(ev, intvs, [200] * ns, 1e-8, v, fl)
        assert r == 0
        sep.append(o)
        probs.append((ev, intvs, [200] * ns, 1e-8, v, fl))
    r, multi = pv.cheblannr_multi(probs)
    assert r == 0
    for o1, o2 in zip(sep, multi):
        for a, b in zip(o1, o2):
            assert a["nev"] == b["nev"] and a["its"] == b["its"]
            assert np.array_equal(a["lam"], b["lam"])
    for ev, M in insts:
        ev.close()


def test_kpm_groups_sum_to_one_group(gpu):
    """pEVSL_Kpmdos with the vectors split over two groups (SRC/kpmdos.c:
    97-102): in the counter-based Gaussian stream each group draws exactly
    its share of one process's vectors, so the groups' moments and counts
    (left unsummed by a no-op reduction) add up to the one-group result."""
    from pevsl_b200.distributed import REDUCE_FN
    lib = pv.load()
    A = dev_matrix(laplacian(20, 20, 20))
    intv = [0.6, 1.2, 0.0, 12.0]
    noop = REDUCE_FN(lambda buf, n, ctx: None)
    with pv.Instance(A) as ev:
        pv.set_rng(pv.RNG_GAUSS, 3)
        r, mu, ec = ev.kpmdos(100, 1, 30, intv)
        assert r == 0
        lib.pEVSL_B200_SetGroupReduce(ev.p, C.cast(noop, C.c_void_p), None)
        parts = []
        for g in range(2):
            pv.set_rng(pv.RNG_GAUSS, 3)
            r, mu_g, ec_g = ev.kpmdos(100, 1, 30, intv, ngroups=2, groupid=g)
            assert r == 0
            parts.append((mu_g, ec_g))
        lib.pEVSL_B200_SetGroupReduce(ev.p, None, None)
    assert rel(parts[0][0] + parts[1][0], mu) <= 1e-13
    assert abs(parts[0][1] + parts[1][1] - ec) <= 1e-12 * abs(ec)
