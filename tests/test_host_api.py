"""CPU tests of the product library's host code and C-ABI (no GPU needed).

* every function declared in include/*.h is exported by libpevsl_b200.so;
* the host-side parts of the path — filter design (pEVSL_FindPol), the KPM
  and Lanczos slicers, partition/sort helpers — reproduce the reference's
  golden outputs.  These run on the host in the product as in the
  reference, so they are tested here without a GPU.  Tolerance: filter
  degree/type and return codes exact, gam/bar/coefficients/endpoints 1e-12.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

import pevsl_b200 as pv
from conftest import ROOT, golden


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def declared_functions():
    names = set()
    for h in ("pevsl.h", "pevsl_b200.h", "pevsl_itsol.h", "pevsl_f90.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        kept, cont = [], False
        for line in text.splitlines():
            if cont or line.lstrip().startswith("#"):
                cont = line.rstrip().endswith("\\")
                continue
            kept.append(line)
        text = "\n".join(kept)
        text = re.sub(r"typedef[^;]*;", "", text)
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{}]*\)\s*;", text):
            name = m.group(1)
            if name not in ("if", "while", "for", "return", "sizeof", "typedef"):
                names.add(name)
    # typedef'd callback types are not functions
    return sorted(n for n in names if n not in ("SVFuncC", "SVFunc", "MVFunc"))


def test_library_exports_every_declared_symbol(lib):
    out = os.popen("nm -D --defined-only " + pv.LIB_PATH).read()
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    assert len(declared_functions()) > 60


def test_binding_signatures_resolve(lib):
    for name, _, _ in pv.SIGNATURES:
        assert hasattr(lib, name), name


def test_findpol_matches_reference_golden(lib):
    for c in golden("findpol_cases.json")["cases"]:
        r, f = pv.findpol(c["intv"], **c["kw"])
        assert r == c["status"], c
        if r == 0:
            assert (f.type, f.deg) == (c["type"], c["deg"]), c
            assert abs(f.gam - c["gam"]) <= 1e-12 and abs(f.bar - c["bar"]) <= 1e-12, c
            assert rel(f.mu, c["mu"]) <= 1e-12
            assert f.cc == c["cc"] and f.dd == c["dd"]


def test_findpol_many_equals_one_at_a_time(lib):
    """The solve driver designs every slice's filter on host threads: each
    result is bit-for-bit the one a lone call gives, in slice order, with
    the error codes of the slices that fail."""
    e = np.linspace(0.8, 0.82, 5)
    ivs = [[e[i], e[i + 1], 0.0, 12.0] for i in range(4)]
    ivs.append([0.5, 0.50001, 0.0, 12.0])  # searched up to max_deg
    ivs.append([0.3, 0.2, 0.0, 12.0])  # invalid interval
    many = pv.findpol_many(ivs)
    for iv, (r, f) in zip(ivs, many):
        r1, f1 = pv.findpol(iv)
        assert r == r1
        if r == 0:
            assert (f.type, f.deg, f.gam, f.bar, f.cc, f.dd) == \
                (f1.type, f1.deg, f1.gam, f1.bar, f1.cc, f1.dd)
            assert np.array_equal(f.mu, f1.mu)
    assert [r for r, _ in many] == [0, 0, 0, 0, 0, -1]  # -1: check_intv


def test_host_eigensolvers_same_bits_on_concurrent_threads(lib):
    """A lockstep group solves its slices' tridiagonal eigenproblems (the
    convergence tests and the Ritz vectors) on concurrent host threads:
    pevsl_tridiag_eig and pevsl_tridiag_eig_sel keep no shared state, so
    each result is bit-for-bit the one a lone call gives."""
    from concurrent.futures import ThreadPoolExecutor
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
    rng = np.random.default_rng(7)
    cases = []
    for n in (64, 151, 200, 257, 300, 331, 400, 531):
        d = rng.uniform(-1.0, 1.0, n)
        e = rng.uniform(0.05, 0.5, n)
        cases.append((n, d, e, np.arange(n - n // 5, n, dtype=np.int32)))

    def solve(c):
        n, d, e, sel = c
        w, w2 = np.zeros(n), np.zeros(n)
        Z = np.zeros(n * len(sel))
        r1 = lib.pevsl_tridiag_eig(n, d.ctypes.data_as(dp), e.ctypes.data_as(dp),
                                   w.ctypes.data_as(dp), None)
        r2 = lib.pevsl_tridiag_eig_sel(n, d.ctypes.data_as(dp), e.ctypes.data_as(dp),
                                       w2.ctypes.data_as(dp), len(sel), sel.ctypes.data_as(ip),
                                       Z.ctypes.data_as(dp))
        return r1, r2, w, w2, Z

    lone = [solve(c) for c in cases]
    with ThreadPoolExecutor(8) as ex:
        together = list(ex.map(solve, cases * 3))
    for i, t in enumerate(together):
        a = lone[i % len(cases)]
        assert t[0] == a[0] == 0 and t[1] == a[1] == 0
        for x, y in zip(t[2:], a[2:]):
            assert np.array_equal(x, y)


@pytest.mark.parametrize("mode", ["glibc", "gauss"])
def test_slicer_and_filters_on_reference_moments(lib, mode):
    g = golden("lap20_kpm.json")
    case = g["cases"][mode]
    r, sli = pv.spslicer_kpm(case["mu"], g["Mdeg"], g["intv"], 5, case["npts"])
    assert r == case["slicer_status"]
    assert rel(sli, case["sli"]) <= 1e-12
    for p in case["pols"]:
        r, f = pv.findpol(p["intv"])
        assert r == 0 and f.deg == p["deg"] and f.type == p["type"]
        assert abs(f.gam - p["gam"]) <= 1e-12 and abs(f.bar - p["bar"]) <= 1e-12
        assert rel(f.mu, p["mu"]) <= 1e-12


def test_slicer_edge_cases(lib):
    g = golden("spslicer_cases.json")
    for c in g["cases"]:
        iv = c.get("intv", g["intv"])
        r, sli = pv.spslicer_kpm(g["mu"], g["Mdeg"], iv, c["n_int"], c["npts"])
        assert r == c["status"], c
        if "sli" in c:
            assert rel(sli, c["sli"]) <= 1e-12


def test_lanczos_slicer_on_reference_dos(lib):
    d = golden("lanczos_cases.json")["landos"]
    sli = pv.spslicer_lan(d["xdos"], d["ydos"], 4)
    assert rel(sli, d["sli4"]) <= 1e-12


def test_part1d_and_sort(lib):
    # SRC/utils.c:124-127: 9 -> [3,2,2,2], 10 -> [3,3,2,2], 11 -> [3,3,3,2]
    for length, sizes in ((9, [3, 2, 2, 2]), (10, [3, 3, 2, 2]), (11, [3, 3, 3, 2])):
        got = []
        for p in range(4):
            idx, j1, j2 = C.c_int(p), C.c_int(), C.c_int()
            lib.pEVSL_Part1d(length, 4, C.byref(idx), C.byref(j1), C.byref(j2), 1)
            got.append(j2.value - j1.value)
        assert got == sizes
        start = 0
        for p, sz in enumerate(sizes):
            for item in range(start, start + sz):
                idx, j1, j2 = C.c_int(), C.c_int(item), C.c_int()
                lib.pEVSL_Part1d(length, 4, C.byref(idx), C.byref(j1), C.byref(j2), 2)
                assert idx.value == p and j2.value == sz
            start += sz
    v = np.array([3.0, -1.0, 2.0, 2.0, 0.5])
    ind = np.zeros(5, np.int32)
    lib.sort_double(5, v.ctypes.data_as(C.POINTER(C.c_double)), ind.ctypes.data_as(C.POINTER(C.c_int)))
    assert list(v) == [-1.0, 0.5, 2.0, 2.0, 3.0] and ind[0] == 1 and ind[4] == 0
    x = np.zeros(7)
    lib.linspace(0.25, 1.75, 7, x.ctypes.data_as(C.POINTER(C.c_double)))
    assert x[0] == 0.25 and x[-1] == 1.75 and abs(x[3] - 1.0) < 1e-16


def test_findpol_needs_room_to_search(lib):
    """The degree search runs from 2 up to max_deg (or the forced degree):
    a limit of 2 or less leaves nothing to search and is PEVSL_ERR_ARG (the
    reference divides by an unset scale there).  Narrow slices are no error:
    their degrees are pinned to the reference in findpol_cases.json."""
    import pevsl_b200 as pv
    iv = [3.0, 3.5, 0.0, 12.0]
    assert pv.findpol(iv, max_deg=2)[0] == pv.ERR_ARG
    assert pv.findpol(iv, deg_in=2)[0] == pv.ERR_ARG
    r, f = pv.findpol(iv, deg_in=3)
    assert r == 0 and f.deg == 2


def test_copy_eigenvectors_rejects_bad_arguments(lib):
    """pEVSL_B200_CopyEigenvectors checks its arguments before touching the
    GPU: more vectors than the Parvecs holds, or a leading dimension below
    the vector length, is PEVSL_ERR_ARG; zero vectors is a no-op."""
    import ctypes as C
    import pevsl_b200 as pv
    W = pv.Parvecs()
    W.n_vecs, W.n_local, W.ld = 2, 10, 16
    out = np.zeros(64)
    p = out.ctypes.data_as(C.POINTER(C.c_double))
    f = pv.load().pEVSL_B200_CopyEigenvectors
    assert f(C.byref(W), 3, p, 10) == pv.ERR_ARG
    assert f(C.byref(W), 2, p, 9) == pv.ERR_ARG
    assert f(C.byref(W), -1, p, 10) == pv.ERR_ARG
    assert f(C.byref(W), 0, p, 10) == 0


# ------------------------------------------------------- randomized, against the reference build
def _random_filter_requests(count, seed):
    rng = np.random.default_rng(seed)
    for _ in range(count):
        lmin = rng.uniform(-2.0, 1.0)
        lmax = lmin + rng.uniform(1.0, 20.0)
        w = (lmax - lmin) * 10 ** rng.uniform(-3.5, -0.3)
        a = rng.uniform(lmin, lmax - 0.5 * w)
        kw = dict(max_deg=int(rng.choice([200, 1000, 3000])), damping=int(rng.integers(0, 3)),
                  thresh_int=float(rng.choice([0.6, 0.8, 0.9])), thresh_ext=0.2)
        yield [a, a + w, lmin, lmax], kw


def test_findpol_random_against_reference(lib, reference):
    """300 random filter requests (middle and end intervals, widths from
    3e-4 to 0.5 of the spectrum, every damping, three thresholds): status,
    type and degree equal to the reference build's, values to 1e-15."""
    for iv, kw in _random_filter_requests(300, 11):
        r1, p = reference.findpol(iv, **kw)
        r2, f = pv.findpol(iv, **kw)
        assert r1 == r2, (iv, kw)
        if r1 == 0:
            assert (f.type, f.deg) == (p["type"], p["deg"]), (iv, kw)
            assert abs(f.gam - p["gam"]) <= 1e-15 and abs(f.bar - p["bar"]) <= 1e-15
            assert np.max(np.abs(f.mu - p["mu"])) <= 1e-15 * np.max(np.abs(p["mu"]))


def test_spslicer_random_against_reference(lib, reference):
    """200 random KPM slicing requests on moments of a genuine density
    (Jackson-damped sums over random eigenvalues): status and every slice
    end bit for bit as the reference build's."""
    rng = np.random.default_rng(5)
    for _ in range(200):
        Mdeg = int(rng.integers(10, 400))
        lam = np.cos(rng.uniform(0.0, np.pi, int(rng.integers(5, 500))))
        k = np.arange(Mdeg + 1)
        th = np.pi / (Mdeg + 2)
        jac = ((1 - k / (Mdeg + 2)) * np.sin(th) * np.cos(k * th)
               + np.cos(th) * np.sin(k * th) / (Mdeg + 2)) / np.sin(th)
        mu = np.cos(np.outer(k, np.arccos(lam))).sum(axis=1) * jac * 2 / np.pi
        mu[0] /= 2
        lmin = rng.uniform(-3.0, 0.0)
        lmax = lmin + rng.uniform(1.0, 20.0)
        a = rng.uniform(lmin - 0.5, lmax)
        iv = [a, a + rng.uniform(0.001, lmax - lmin), lmin, lmax]
        n_int = int(rng.integers(1, 12))
        npts = int(rng.integers(2 * n_int - 1, 3000))
        r1, s1 = reference.spslicer_kpm(mu, Mdeg, iv, n_int, npts)
        r2, s2 = pv.spslicer_kpm(mu, Mdeg, iv, n_int, npts)
        assert r1 == r2
        if r1 >= 0:
            assert np.array_equal(np.asarray(s1), np.asarray(s2))


def test_spslicer_lan_random_against_reference(lib, reference):
    """200 random sampled densities (3 to 600 points, 1 to 14 slices): the
    Lanczos-DOS slice ends bit for bit as the reference build's."""
    rng = np.random.default_rng(9)
    for _ in range(200):
        npts, n_int = int(rng.integers(3, 600)), int(rng.integers(1, 15))
        x = np.sort(rng.uniform(-2.0, 5.0, npts))
        y = np.abs(rng.standard_normal(npts)) * rng.uniform(0.1, 10.0)
        s1 = reference.spslicer_lan(x, y, n_int)
        s2 = pv.spslicer_lan(x, y.copy(), n_int)
        assert np.array_equal(np.asarray(s1), np.asarray(s2))


def test_coo_to_csr_and_host_matvec_against_reference(lib, reference):
    """pEVSL_CooToCsr (0- and 1-based input, duplicates, empty rows) and the
    host pEVSL_Matvec on its result: arrays and products bit for bit as the
    reference build's (SRC/spmat.c), on 300 random matrices."""
    class Coo(C.Structure):
        _fields_ = [("nrows", C.c_int), ("ncols", C.c_int), ("nnz", C.c_int),
                    ("ir", C.POINTER(C.c_int)), ("jc", C.POINTER(C.c_int)),
                    ("vv", C.POINTER(C.c_double))]

    ip, dp = C.POINTER(C.c_int), C.POINTER(C.c_double)
    rlib = reference.lib
    rng = np.random.default_rng(1)
    for _ in range(300):
        nr, nc, nnz = int(rng.integers(1, 60)), int(rng.integers(1, 60)), int(rng.integers(0, 300))
        base = int(rng.integers(0, 2))
        ir = (rng.integers(0, nr, nnz) + base).astype(np.int32)
        jc = (rng.integers(0, nc, nnz) + base).astype(np.int32)
        vv = rng.standard_normal(nnz)
        x = rng.standard_normal(nc)
        outs = []
        for L in (rlib, lib):
            coo = Coo(nr, nc, nnz, ir.ctypes.data_as(ip), jc.ctypes.data_as(ip),
                      vv.ctypes.data_as(dp))
            csr = pv.Csr()
            r = L.pEVSL_CooToCsr(base, C.byref(coo), C.byref(csr))
            ia = np.ctypeslib.as_array(csr.ia, shape=(nr + 1,)).copy()
            m = int(ia[-1])
            ja = np.ctypeslib.as_array(csr.ja, shape=(m,)).copy() if m else np.zeros(0, np.int32)
            a = np.ctypeslib.as_array(csr.a, shape=(m,)).copy() if m else np.zeros(0)
            y = np.zeros(nr)
            L.pEVSL_Matvec(C.byref(csr), x.ctypes.data_as(dp), y.ctypes.data_as(dp))
            L.pEVSL_FreeCsr(C.byref(csr))
            outs.append((r, ia, ja, a, y))
        for u, w in zip(*outs):
            assert np.array_equal(np.asarray(u), np.asarray(w))


def test_findpol_end_intervals_random_against_reference(lib, reference):
    """200 random end-interval filters (SRC/chebpol.c:166-255; the slice at
    or beyond either end of the spectrum bounds, forced degrees among them):
    type, degree and values as the reference build's."""
    rng = np.random.default_rng(21)
    for t in range(200):
        lmin = rng.uniform(-2.0, 1.0)
        lmax = lmin + rng.uniform(1.0, 20.0)
        w = (lmax - lmin) * 10 ** rng.uniform(-3.0, -0.2)
        if t % 2 == 0:
            iv = [lmin - rng.uniform(0.0, 1.0) * (t % 4 == 0), lmin + w, lmin, lmax]
        else:
            iv = [lmax - w, lmax + rng.uniform(0.0, 1.0) * (t % 4 == 1), lmin, lmax]
        kw = dict(max_deg=int(rng.choice([200, 1000, 3000])), damping=int(rng.integers(0, 3)),
                  thresh_ext=float(rng.choice([0.1, 0.2, 0.3])),
                  deg_in=int(rng.choice([0, 0, 0, 50])))
        r1, p = reference.findpol(iv, **kw)
        r2, f = pv.findpol(iv, **kw)
        assert r1 == r2 == 0
        assert (f.type, f.deg) == (p["type"], p["deg"]) and f.type == (1 if t % 2 == 0 else 2)
        assert abs(f.gam - p["gam"]) <= 1e-15 and abs(f.bar - p["bar"]) <= 1e-15 * max(1, abs(p["bar"]))
        assert np.max(np.abs(f.mu - p["mu"])) <= 1e-14 * np.max(np.abs(p["mu"]))
