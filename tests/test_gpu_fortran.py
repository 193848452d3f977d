"""The Fortran binding (include/pevsl_f90.h, FORTRAN/pevsl_f90.c of the
reference) called the way a Fortran program calls it: every argument by
reference, objects as uintptr_t handles, host arrays.

* standard problem: parcsr from C-indexed CSR, bounds, filter, ChebLanNr,
  pevsl_get_nev / pevsl_copy_result -> the analytic Laplacian eigenvalues
  to 1e-10 and eigenvector residuals <= 1e-8; pevsl_parcsrmatvec against
  numpy; KPM count estimate near the exact count;
* generalized problem: B parcsr, Chebyshev-iteration B-solve and
  least-squares L^{-T} installed through the binding, eigenvalues against
  scipy's dense generalized eigenvalues to 1e-10; the staged B-solvers
  (pevsl_chebiter, pevsl_lspolsol) against the reference build's outputs
  (tests/golden/gen_bsolve.json).
"""
import ctypes as C

import numpy as np
import pytest

import pevsl_b200 as pv
from checkers import exact_eig_lap, laplacian
from conftest import golden

pytestmark = pytest.mark.gpu

U = C.c_uint64  # uintptr_t on this host


def ref(x, t):
    return C.byref(t(x)) if not isinstance(x, C._SimpleCData) else C.byref(x)


def dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def parcsr(lib, L):
    n = L.n
    starts = np.array([0, n], dtype=np.int32)
    h = U()
    lib.pevsl_parcsrcreate_f90_(ref(n, C.c_int), ref(n, C.c_int), ip(starts), ip(starts),
                                ip(L.ia), ip(L.ja), dp(L.a), ref(1, C.c_int), C.byref(h))
    assert h.value
    return h


def dense(L):
    M = np.zeros((L.n, L.n))
    for i in range(L.n):
        M[i, L.ja[L.ia[i]:L.ia[i + 1]]] = L.a[L.ia[i]:L.ia[i + 1]]
    return M


def test_fortran_standard_problem(gpu):
    lib = pv.load()
    L = laplacian(12, 12, 12)
    n = L.n
    A = parcsr(lib, L)
    x = np.sin(np.arange(n, dtype=np.float64))
    y = np.zeros(n)
    lib.pevsl_parcsrmatvec_f90_(dp(x), dp(y), C.byref(A))
    assert np.max(np.abs(y - dense(L) @ x)) <= 1e-12
    h = U()
    lib.pevsl_start_f90_(ref(1, C.c_int), C.byref(h))
    lib.pevsl_seta_parcsr_f90_(C.byref(h), C.byref(A))
    lmin, lmax = C.c_double(), C.c_double()
    lib.pevsl_lanbounds_f90_(C.byref(h), ref(50, C.c_int), ref(200, C.c_int),
                             ref(1e-8, C.c_double), C.byref(lmin), C.byref(lmax))
    assert lmin.value <= 0.19 and 11.8 <= lmax.value <= 12.0 + 1e-6
    a, b = 1.0, 1.6
    intv = np.array([a, b, lmin.value, lmax.value])
    mu = np.zeros(81)
    ecnt = C.c_double()
    lib.pevsl_kpmdos_ecnt_f90_(C.byref(h), ref(80, C.c_int), ref(1, C.c_int), ref(30, C.c_int),
                               dp(intv), dp(mu), C.byref(ecnt))
    exact = exact_eig_lap(12, 12, 12, a, b)
    assert abs(ecnt.value - len(exact)) <= 0.2 * len(exact)
    pol = U()
    lib.pevsl_findpol_f90_(dp(intv), ref(0.8, C.c_double), ref(0.2, C.c_double), C.byref(pol))
    assert pol.value
    lib.pevsl_cheblannr_f90_(C.byref(h), dp(intv), ref(min(n, 600), C.c_int),
                             ref(1e-8, C.c_double), C.byref(pol))
    nev = C.c_int()
    lib.pevsl_get_nev_f90_(C.byref(h), C.byref(nev))
    assert nev.value == len(exact)
    ld = n + 3
    val = np.zeros(nev.value)
    vec = np.zeros(ld * nev.value)
    lib.pevsl_copy_result_f90_(C.byref(h), dp(val), dp(vec), ref(ld, C.c_int))
    lib.pevsl_get_nev_f90_(C.byref(h), C.byref(nev))
    assert nev.value == 0  # released by copy_result
    order = np.argsort(val)
    assert np.max(np.abs(val[order] - exact) / exact) <= 1e-10
    Ad = dense(L)
    for j in range(len(val)):
        u = vec[j * ld:j * ld + n]
        assert abs(np.linalg.norm(u) - 1.0) <= 1e-10
        assert np.linalg.norm(Ad @ u - val[j] * u) <= 1e-8
    lib.pevsl_freepol_f90_(C.byref(pol))
    lib.pevsl_finish_f90_(C.byref(h))
    lib.pevsl_parcsr_free_f90_(C.byref(A))
    assert A.value == 0


def test_fortran_bsolvers_staged(gpu):
    lib = pv.load()
    g = golden("gen_bsolve.json")
    B = parcsr(lib, laplacian(512, 1, 1))
    b = np.cos(0.1 * np.arange(512, dtype=np.float64)) + 0.5
    for c in g["chebiter"]:
        ch = U()
        lib.pevsl_setup_chebiter_f90_(ref(c["lmin"], C.c_double), ref(c["lmax"], C.c_double),
                                      ref(c["deg"], C.c_int), C.byref(B), C.byref(ch))
        x = np.zeros(512)
        lib.pevsl_chebiter_f90_(ref(c["kind"], C.c_int), dp(b.copy()), dp(x), C.byref(ch))
        assert np.max(np.abs(x - c["x"])) <= 1e-13 * max(np.max(np.abs(c["x"])), 1e-300)
        lib.pevsl_free_chebiterb_f90_(C.byref(ch))
    c = g["lspol"][1]  # 1/sqrt(x), max_deg 50, tol 1e-6
    ls = U()
    lib.pevsl_setup_lspolsqrt_f90_(ref(c["lmin"], C.c_double), ref(c["lmax"], C.c_double),
                                   ref(c["max_deg"], C.c_int), ref(c["tol"], C.c_double),
                                   C.byref(B), C.byref(ls))
    x = np.zeros(512)
    lib.pevsl_lspolsol_f90_(dp(b.copy()), dp(x), C.byref(ls))
    assert np.max(np.abs(x - c["x"])) <= 1e-13 * np.max(np.abs(c["x"]))
    lib.pevsl_free_lspol_f90_(C.byref(ls))
    lib.pevsl_parcsr_free_f90_(C.byref(B))


def test_fortran_generalized_problem(gpu):
    import scipy.linalg as sl
    lib = pv.load()
    LA, LB = laplacian(20, 20, 1), laplacian(400, 1, 1)
    w = sl.eigh(dense(LA), dense(LB), eigvals_only=True)
    a, b = 0.4, 0.7
    exact = w[(w >= a) & (w <= b)]
    A, B = parcsr(lib, LA), parcsr(lib, LB)
    h = U()
    lib.pevsl_start_f90_(ref(1, C.c_int), C.byref(h))
    lib.pevsl_seta_parcsr_f90_(C.byref(h), C.byref(A))
    lib.pevsl_setb_parcsr_f90_(C.byref(h), C.byref(B))
    ch, ls = U(), U()
    lib.pevsl_setup_chebiter_f90_(ref(2.0, C.c_double), ref(6.0, C.c_double), ref(40, C.c_int),
                                  C.byref(B), C.byref(ch))
    lib.pevsl_setbsol_chebiter_f90_(C.byref(h), ref(2, C.c_int), C.byref(ch))
    lib.pevsl_setup_lspolsqrt_f90_(ref(2.0, C.c_double), ref(6.0, C.c_double), ref(50, C.c_int),
                                   ref(1e-6, C.c_double), C.byref(B), C.byref(ls))
    lib.pevsl_setltsol_lspol_f90_(C.byref(h), C.byref(ls))
    lib.pevsl_set_geneig_f90_(C.byref(h))
    x = np.cos(np.arange(400.0))
    y, z = np.zeros(400), np.zeros(400)
    lib.pevsl_bsv_f90_(C.byref(h), dp(x), dp(y))
    assert np.linalg.norm(dense(LB) @ y - x) <= 1e-13 * np.linalg.norm(x)
    lmin, lmax = C.c_double(), C.c_double()
    lib.pevsl_lanbounds_f90_(C.byref(h), ref(50, C.c_int), ref(200, C.c_int),
                             ref(1e-8, C.c_double), C.byref(lmin), C.byref(lmax))
    assert abs(lmin.value - w[0]) <= 1e-6 * w[-1] and abs(lmax.value - w[-1]) <= 1e-6 * w[-1]
    intv = np.array([a, b, lmin.value, lmax.value])
    pol = U()
    lib.pevsl_findpol_f90_(dp(intv), ref(0.6, C.c_double), ref(0.15, C.c_double), C.byref(pol))
    lib.pevsl_cheblannr_f90_(C.byref(h), dp(intv), ref(400, C.c_int), ref(1e-8, C.c_double),
                             C.byref(pol))
    nev = C.c_int()
    lib.pevsl_get_nev_f90_(C.byref(h), C.byref(nev))
    assert nev.value == len(exact)
    val, vec = np.zeros(nev.value), np.zeros(400 * nev.value)
    lib.pevsl_copy_result_f90_(C.byref(h), dp(val), dp(vec), ref(400, C.c_int))
    assert np.max(np.abs(np.sort(val) - exact) / exact) <= 1e-10
    lib.pevsl_freepol_f90_(C.byref(pol))
    lib.pevsl_free_chebiterb_f90_(C.byref(ch))
    lib.pevsl_free_lspol_f90_(C.byref(ls))
    lib.pevsl_finish_f90_(C.byref(h))
    lib.pevsl_parcsr_free_f90_(C.byref(A))
    lib.pevsl_parcsr_free_f90_(C.byref(B))
