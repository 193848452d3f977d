"""Generalized problem A x = lambda B x on the GPU.

* B-solvers: the least-squares polynomials (pEVSL_LSPolSol) and Chebyshev
  iterations (pEVSL_ChebIterSolv1/2) against the reference build's outputs
  for the same B and right-hand side (tests/golden/gen_bsolve.json), to
  1e-13 relative (same recurrences; the fused kernels may round a multiply
  and add together where the reference's BLAS does not);
* the reference's own generalized driver (TESTS/Gen_Lap/LapPLanN.c, built by
  tests/dropin/Makefile with the Chebyshev B-solver of tests/dropin/shim in
  place of MUMPS) against the same driver on the reference build
  (tests/golden/genlap8.json): bounds to 1e-10, slices to 1e-12, filter
  degrees and per-slice counts identical, eigenvalues to 1e-10;
* a whole interval through the Python API against the dense generalized
  eigenvalues of scipy (A 2D Laplacian, B 1D Laplacian): every eigenvalue
  found, to 1e-10, residuals ||A x - lam B x|| <= 1e-8.
"""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import pevsl_b200 as pv
from conftest import golden
from test_gpu_dropin import binary

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def csr_of(nx, ny, nz):
    from checkers import laplacian
    L = laplacian(nx, ny, nz)
    return pv.Matrix.from_csr(L.n, L.ia, L.ja, L.a), L


@pytest.fixture(scope="module")
def B512(gpu):
    M, L = csr_of(512, 1, 1)
    yield M
    M.free()


def rhs(n):
    return np.cos(0.1 * np.arange(n, dtype=np.float64)) + 0.5


@pytest.mark.parametrize("case", range(4))
def test_lspol_solve_matches_reference(B512, case):
    g = golden("gen_bsolve.json")["lspol"][case]
    S = pv.BSolver(B512, "lsrec" if g["kind"] == 0 else "lssqrt", g["lmin"], g["lmax"],
                   g["max_deg"], g["tol"])
    try:
        assert S.degree == g["deg"]
        np.testing.assert_array_equal(S.coefficients(), np.array(g["mu"]))
        x = S.solve(rhs(512))
        assert rel(x, g["x"]) <= 1e-13
    finally:
        S.free()


@pytest.mark.parametrize("case", range(5))
def test_chebiter_solve_matches_reference(B512, case):
    g = golden("gen_bsolve.json")["chebiter"][case]
    S = pv.BSolver(B512, "cheb%d" % g["kind"], g["lmin"], g["lmax"], g["deg"])
    try:
        x = S.solve(rhs(512))
        assert rel(x, g["x"]) <= 1e-13, rel(x, g["x"])
    finally:
        S.free()


def test_chebiter_degree_40_solves_to_rounding(B512):
    """the driver shim's B-solver: B x = b to rounding level"""
    from checkers import laplacian
    L = laplacian(512, 1, 1)
    S = pv.BSolver(B512, "cheb2", 2.0, 6.0, 40)
    try:
        b = rhs(512)
        x = S.solve(b)
        Bx = np.zeros(512)
        for i in range(512):
            Bx[i] = np.dot(L.a[L.ia[i]:L.ia[i + 1]], x[L.ja[L.ia[i]:L.ia[i + 1]]])
        assert np.linalg.norm(Bx - b) <= 1e-14 * np.linalg.norm(b)
    finally:
        S.free()


def _report(out):
    bounds = [float(x) for x in re.findall(r"Eigenvalue bound s for B\^\{-1\}\*A: \[([-\d.e+]+), ([-\d.e+]+)\]", out)[0]] \
        if "bound s" in out else None
    sl = [tuple(float(x) for x in m) for m in
          re.findall(r"^\s*\d+: \[\s*([-\d.e+]+)\s*,\s*([-\d.e+]+)\]", out, re.M)]
    degs = [int(x) for x in re.findall(r"polynomial \[type \d\] deg (\d+)", out)]
    counts = [int(x) for x in re.findall(r"number of eigenvalues found: (\d+)", out)]
    lams = [float(x) for x in re.findall(r"^\s*(-?\d\.\d{15}e[-+]\d+)\s+\d\.\de[-+]\d+\s*$", out, re.M)]
    return bounds, sl, degs, counts, lams


@pytest.mark.parametrize("name", ["kpm", "landos"])
def test_reference_generalized_driver(gpu, tmp_path, name):
    g = golden("genlap8.json")[name]
    exe = binary("GenLapPLanN")
    os.makedirs(tmp_path / "OUT")
    r = subprocess.run([exe] + g["args"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr
    got = _report((tmp_path / "OUT" / "LapPLanN_G0.out").read_text())
    ref = _report(g["out"])
    assert rel(got[0], ref[0]) <= 1e-10
    assert len(got[1]) == len(ref[1]) > 0
    assert rel(np.array(got[1]), np.array(ref[1])) <= 1e-12
    assert got[2] == ref[2]
    assert got[3] == ref[3] and sum(got[3]) == 205
    assert len(got[4]) == len(ref[4]) > 0
    assert np.max(np.abs(np.array(got[4]) - ref[4]) / np.abs(ref[4])) <= 1e-10
    est = re.findall(r"estimated eig count in interval: ([\d.]+)", r.stdout)
    assert est == re.findall(r"estimated eig count in interval: ([\d.]+)", g["stdout"])


def test_generalized_interval_against_dense(gpu):
    """A = 2D Laplacian 20 x 20, B = 1D Laplacian (diagonal 4) of the same
    size; [0.4, 0.9] of B^{-1} A in 2 slices, B-solve by the second-kind
    Chebyshev iteration, L^{-T} by the least-squares 1/sqrt(x)."""
    import scipy.linalg as sl
    from checkers import laplacian
    lib = pv.load()
    A, LA = csr_of(20, 20, 1)
    B, LB = csr_of(400, 1, 1)
    Ad, Bd = np.zeros((400, 400)), np.zeros((400, 400))
    for M, L in ((Ad, LA), (Bd, LB)):
        for i in range(400):
            M[i, L.ja[L.ia[i]:L.ia[i + 1]]] = L.a[L.ia[i]:L.ia[i + 1]]
    w, X = sl.eigh(Ad, Bd)
    a, b = 0.4, 0.9
    exact = w[(w >= a) & (w <= b)]
    bs = pv.BSolver(B, "cheb2", 2.0, 6.0, 40)
    lt = pv.BSolver(B, "lssqrt", 2.0, 6.0, 50, 1e-6)
    pv.set_rng(pv.RNG_GAUSS, 5)
    with pv.Instance(A) as ev:
        ev.set_generalized(B, bs, lt)
        vinit = pv.Vector(400)
        lib.pEVSL_ParvecRand(C.byref(vinit.pv))
        lo, hi = C.c_double(), C.c_double()
        r = lib.pEVSL_LanTrbounds(ev.p, 50, 200, 1e-8, C.byref(vinit.pv), 1, C.byref(lo),
                                  C.byref(hi), None)
        assert r == 0
        assert abs(lo.value - w[0]) <= 1e-6 * w[-1] and abs(hi.value - w[-1]) <= 1e-6 * w[-1]
        intv = [a, b, lo.value, hi.value]
        r, mu, ecount = ev.kpmdos(40, 1, 30, intv)
        assert r == 0 and abs(ecount - len(exact)) <= 0.25 * len(exact) + 3
        r, sli = pv.spslicer_kpm(mu, 40, intv, 2, int(10 * ecount))
        assert r == 0
        filters, intvs = [], []
        for s in range(2):
            iv = [sli[s], sli[s + 1], lo.value, hi.value]
            r, f = pv.findpol(iv, 3000, 2, 0.6, 0.15)
            assert r == 0
            filters.append(f)
            intvs.append(iv)
        r, outs = pv.cheblannr_batch(ev, intvs, [400, 400], 1e-8, vinit, filters)
        assert r == 0
        lam = np.sort(np.concatenate([o["lam"] for o in outs]))
        res = np.concatenate([o["res"] for o in outs])
        vinit.free()
    bs.free()
    lt.free()
    assert len(lam) == len(exact), (len(lam), len(exact))
    assert np.max(np.abs(lam - exact) / np.abs(exact)) <= 1e-10
    assert np.max(res) <= 1e-8


def test_generalized_filter_against_dense(gpu):
    """pEVSL_B200_ChebAvGen: y = p(A B^{-1}) v with the exact B^{-1}"""
    from checkers import laplacian
    A, LA = csr_of(8, 8, 8)
    B, LB = csr_of(512, 1, 1)
    Ad, Bd = np.zeros((512, 512)), np.zeros((512, 512))
    for M, L in ((Ad, LA), (Bd, LB)):
        for i in range(512):
            M[i, L.ja[L.ia[i]:L.ia[i + 1]]] = L.a[L.ia[i]:L.ia[i + 1]]
    r, f = pv.findpol([1.5, 1.8, 0.17, 3.92], 3000, 2, 0.6, 0.15)
    assert r == 0
    bs = pv.BSolver(B, "cheb2", 2.0, 6.0, 40)
    v = np.sin(np.arange(512.0))
    with pv.Instance(A) as ev:
        ev.set_generalized(B, bs)
        pol, keep = pv._polparams(f)
        vv, yv = pv.Vector(512, v), pv.Vector(512)
        assert ev.lib.pEVSL_B200_ChebAvGen(ev.p, C.byref(pol), vv.pv.data, yv.pv.data) == 0
        y = yv.get()
        vv.free()
        yv.free()
    bs.free()
    M = Ad @ np.linalg.inv(Bd)
    T = (M - f.cc * np.eye(512)) / f.dd
    tk, tkm1 = v.copy(), None
    yref = f.mu[0] * v
    for k in range(1, f.deg + 1):
        tn = (2.0 if k > 1 else 1.0) * (T @ tk) - (tkm1 if tkm1 is not None else 0.0)
        yref = yref + f.mu[k] * tn
        tkm1, tk = tk, tn
    assert rel(y, yref) <= 1e-10


def test_generalized_lockstep_equals_one_by_one(gpu, monkeypatch):
    """Slices of one generalized problem with the least-squares B-solve run
    in lockstep (one interleaved filter application per step for all of
    them); each slice gets the bits of solving it alone, and every
    eigenvalue of the dense pencil in the interval (A 2D Laplacian 24 x 24,
    B 1D Laplacian of the same size)."""
    import scipy.linalg as sl
    A, LA = csr_of(24, 24, 1)
    B, LB = csr_of(576, 1, 1)
    Ad, Bd = np.zeros((576, 576)), np.zeros((576, 576))
    for M, L in ((Ad, LA), (Bd, LB)):
        for i in range(576):
            M[i, L.ja[L.ia[i]:L.ia[i + 1]]] = L.a[L.ia[i]:L.ia[i + 1]]
    w = sl.eigh(Ad, Bd, eigvals_only=True)
    lmin, lmax = w[0] - 1e-6, w[-1] + 1e-6
    edges = np.linspace(0.4, 0.7, 4)
    intvs = [[edges[i], edges[i + 1], lmin, lmax] for i in range(3)]
    fl = [pv.findpol(iv, 3000, 2, 0.6, 0.15)[1] for iv in intvs]
    v = np.cos(np.arange(576) * 0.3)
    bs = pv.BSolver(B, "lsrec", 2.0, 6.0, 80, 1e-10)
    outs = {}
    for mode in ("lockstep", "one_by_one"):
        if mode == "one_by_one":
            monkeypatch.setenv("PEVSL_B200_GEN_LOCKSTEP_OFF", "1")
        with pv.Instance(A) as ev:
            ev.set_generalized(B, bs)
            r, o = pv.cheblannr_batch(ev, intvs, [400] * 3, 1e-8, v, fl)
        assert r == 0
        outs[mode] = o
    bs.free()
    for iv, a, b in zip(intvs, outs["lockstep"], outs["one_by_one"]):
        assert a["nev"] == b["nev"] and a["its"] == b["its"]
        assert np.array_equal(a["lam"], b["lam"]) and np.array_equal(a["res"], b["res"])
        ex = w[(w >= iv[0]) & (w <= iv[1])]
        assert a["nev"] == len(ex)
        assert np.max(np.abs(a["lam"] - ex) / np.abs(ex)) <= 1e-10
        assert np.max(a["res"]) <= 1e-8
