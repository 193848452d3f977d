"""ctypes access to the two CPU checkers (test infrastructure).

* ``ref``    -- oracle/_ref/libpevsl_ref.so: the pEVSL reference compiled from
               its own sources (oracle/Makefile), driven through its public
               API by oracle/ref_glue.c.
* ``oracle`` -- oracle/_build/liboracle.so: the plain-C restatement
               (oracle/pevsl_oracle.c).

Both expose the same flat entry points with prefixes ``oref_`` / ``orc_`` and
the same ``orc_spec`` / ``orc_out`` run description (oracle/pipeline.h), so a
test can run one case through either and compare.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
REF_SO = os.path.join(ORACLE_DIR, "_ref", "libpevsl_ref.so")
ORC_SO = os.path.join(ORACLE_DIR, "_build", "liboracle.so")
# the reference source tree (read only); one variable for every recipe,
# script and test that builds or reads the reference
REFERENCE_TREE = os.environ.get("PEVSL_REFDIR", "/root/reference")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def build_oracle() -> None:
    """Build liboracle.so (and libpevsl_ref.so when the reference tree exists)."""
    targets = ["oracle"]
    if os.path.isdir(REFERENCE_TREE) and not os.path.exists(REF_SO):
        targets.append("ref")
    if not os.path.exists(ORC_SO) or "ref" in targets:
        subprocess.run(["make", "-s", "-C", ORACLE_DIR, f"REFDIR={REFERENCE_TREE}"] + targets,
                       check=True)


class OrcSpec(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("ia", C.c_void_p), ("ja", C.c_void_p), ("a", C.c_void_p),
        ("a_lo", C.c_double), ("b_hi", C.c_double), ("nslices", C.c_int),
        ("bounds_mode", C.c_int), ("lmin", C.c_double), ("lmax", C.c_double),
        ("lan_lanm", C.c_int), ("lan_maxit", C.c_int), ("lan_bndtype", C.c_int),
        ("lan_tol", C.c_double),
        ("dos_type", C.c_int), ("Mdeg", C.c_int), ("kpm_damping", C.c_int), ("nvec", C.c_int),
        ("landos_msteps", C.c_int), ("landos_npts", C.c_int),
        ("pol_damping", C.c_int), ("pol_max_deg", C.c_int),
        ("thresh_int", C.c_double), ("thresh_ext", C.c_double),
        ("tol", C.c_double), ("mlan_min", C.c_int),
        ("rng_mode", C.c_int), ("seed", C.c_uint64),
    ]


class OrcOut(C.Structure):
    _fields_ = [
        ("cap", C.c_int), ("mu", C.c_void_p), ("sli", C.c_void_p), ("deg", C.c_void_p),
        ("ptype", C.c_void_p), ("gam", C.c_void_p), ("bar", C.c_void_p), ("nev", C.c_void_p),
        ("its", C.c_void_p), ("lam", C.c_void_p), ("res", C.c_void_p),
        ("lmin", C.c_double), ("lmax", C.c_double), ("ecount", C.c_double), ("npts", C.c_int),
        ("status", C.c_int),
        ("t_bounds", C.c_double), ("t_dos", C.c_double), ("t_slicer", C.c_double),
        ("t_slices", C.c_double), ("t_total", C.c_double),
    ]


@dataclass
class Csr:
    n: int
    ia: np.ndarray
    ja: np.ndarray
    a: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.ia[-1])


@dataclass
class RunSpec:
    """One spectrum-slicing run (fields as in oracle/pipeline.h)."""
    a_lo: float
    b_hi: float
    nslices: int
    bounds_mode: int = 0
    lmin: float = 0.0
    lmax: float = 12.0
    lan_lanm: int = 50
    lan_maxit: int = 200
    lan_bndtype: int = 1
    lan_tol: float = 1e-8
    dos_type: int = 0
    Mdeg: int = 300
    kpm_damping: int = 1
    nvec: int = 60
    landos_msteps: int = 40
    landos_npts: int = 200
    pol_damping: int = 2
    pol_max_deg: int = 3000
    thresh_int: float = 0.8
    thresh_ext: float = 0.2
    tol: float = 1e-8
    mlan_min: int = 300
    rng_mode: int = 0
    seed: int = 0


@dataclass
class RunResult:
    lmin: float
    lmax: float
    ecount: float
    npts: int
    status: int
    mu: np.ndarray
    sli: np.ndarray
    deg: np.ndarray
    ptype: np.ndarray
    gam: np.ndarray
    bar: np.ndarray
    nev: np.ndarray
    its: np.ndarray
    lam: list = field(default_factory=list)
    res: list = field(default_factory=list)
    times: dict = field(default_factory=dict)


class Checker:
    """Uniform wrapper over the reference build (prefix oref_) or the
    restatement (prefix orc_)."""

    def __init__(self, which: str):
        build_oracle()
        self.which = which
        path = REF_SO if which == "ref" else ORC_SO
        self.lib = C.CDLL(path)
        self.p = "oref_" if which == "ref" else "orc_"

    def f(self, name):
        return getattr(self.lib, self.p + name)

    # -- random stream -------------------------------------------------
    def set_rng(self, mode: int, seed: int) -> None:
        """Stream used by the next pipeline / unit call."""
        if self.which == "ref":
            self.lib.oref_set_unit_rng(C.c_int(mode), C.c_uint64(seed))
        self.f("set_rng")(C.c_int(mode), C.c_uint64(seed))

    # -- kernels of the path -------------------------------------------
    def matvec(self, A: Csr, x: np.ndarray) -> np.ndarray:
        y = np.zeros(A.n)
        self.f("matvec")(A.n, _ptr(A.ia), _ptr(A.ja), _ptr(A.a), _ptr(x), _ptr(y))
        return y

    def kpmdos(self, A: Csr, Mdeg, damping, nvec, intv):
        mu = np.zeros(Mdeg + 1)
        ec = C.c_double()
        iv = np.asarray(intv, dtype=np.float64)
        r = self.f("kpmdos")(A.n, _ptr(A.ia), _ptr(A.ja), _ptr(A.a), Mdeg, damping, nvec,
                             _ptr(iv), _ptr(mu), C.byref(ec))
        return r, mu, ec.value

    def spslicer_kpm(self, mu, Mdeg, intv, n_int, npts):
        sli = np.zeros(n_int + 1)
        iv = np.asarray(intv, dtype=np.float64)
        mu = np.ascontiguousarray(mu, dtype=np.float64)
        r = self.f("spslicer_kpm")(_ptr(sli), _ptr(mu), Mdeg, _ptr(iv), n_int, npts)
        return r, sli

    def findpol(self, intv, max_deg=3000, damping=2, thresh_int=0.8, thresh_ext=0.2, deg_in=0):
        iv = np.asarray(intv, dtype=np.float64)
        mu = np.zeros(max_deg + 1)
        t, d = C.c_int(), C.c_int()
        gam, bar, cc, dd = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        r = self.f("findpol")(_ptr(iv), max_deg, damping, C.c_double(thresh_int),
                              C.c_double(thresh_ext), deg_in, C.byref(t), C.byref(d),
                              C.byref(gam), C.byref(bar), C.byref(cc), C.byref(dd), _ptr(mu))
        if r:
            return r, None
        return r, dict(type=t.value, deg=d.value, gam=gam.value, bar=bar.value, cc=cc.value,
                       dd=dd.value, mu=mu[: d.value + 1].copy())

    def chebav(self, A: Csr, pol: dict, v: np.ndarray) -> np.ndarray:
        y = np.zeros(A.n)
        mu = np.ascontiguousarray(pol["mu"])
        self.f("chebav")(A.n, _ptr(A.ia), _ptr(A.ja), _ptr(A.a), pol["deg"],
                         C.c_double(pol["cc"]), C.c_double(pol["dd"]), _ptr(mu), _ptr(v), _ptr(y))
        return y

    # -- B-solvers of the generalized problem (reference build only) ----
    def lspol(self, kind, max_deg, tol, lmin, lmax, B: Csr, b):
        """pEVSL_SetupLSPolRec (kind 0) / Sqrt (kind 1) on B: the degree,
        coefficients mu[0..deg], cc, dd, and pEVSL_LSPolSol(b)."""
        mu, x = np.zeros(max_deg), np.zeros(B.n)
        deg, cc, dd = C.c_int(), C.c_double(), C.c_double()
        bb = np.ascontiguousarray(b, dtype=np.float64)
        self.f("lspol")(kind, max_deg, C.c_double(tol), C.c_double(lmin), C.c_double(lmax), B.n,
                        _ptr(B.ia), _ptr(B.ja), _ptr(B.a), _ptr(mu), C.byref(deg), C.byref(cc),
                        C.byref(dd), _ptr(bb), _ptr(x))
        return deg.value, mu[:deg.value + 1].copy(), cc.value, dd.value, x

    def chebiter(self, kind, lmin, lmax, deg, B: Csr, b):
        """pEVSL_ChebIterSolv1 (kind 1) / Solv2 (kind 2) of b on B"""
        x = np.zeros(B.n)
        bb = np.ascontiguousarray(b, dtype=np.float64)
        self.f("chebiter")(kind, C.c_double(lmin), C.c_double(lmax), deg, B.n, _ptr(B.ia),
                           _ptr(B.ja), _ptr(B.a), _ptr(bb), _ptr(x))
        return x

    def lantrbounds(self, A: Csr, lanm, maxit, tol, vinit, bndtype=1):
        lo, hi = C.c_double(), C.c_double()
        v = np.ascontiguousarray(vinit, dtype=np.float64)
        r = self.f("lantrbounds")(A.n, _ptr(A.ia), _ptr(A.ja), _ptr(A.a), lanm, maxit,
                                  C.c_double(tol), _ptr(v), bndtype, C.byref(lo), C.byref(hi))
        return r, lo.value, hi.value

    def landos(self, A: Csr, nvec, msteps, npts, intv):
        xd, yd = np.zeros(npts), np.zeros(npts)
        ne = C.c_double()
        iv = np.asarray(intv, dtype=np.float64)
        r = self.f("landos")(A.n, _ptr(A.ia), _ptr(A.ja), _ptr(A.a), nvec, msteps, npts,
                             _ptr(xd), _ptr(yd), C.byref(ne), _ptr(iv))
        return r, xd, yd, ne.value

    def spslicer_lan(self, xi, yi, n_int):
        xi = np.ascontiguousarray(xi, dtype=np.float64)
        yi = np.ascontiguousarray(yi, dtype=np.float64).copy()
        sli = np.zeros(n_int + 1)
        self.f("spslicer_lan")(_ptr(xi), _ptr(yi), n_int, len(xi), _ptr(sli))
        return sli

    def cheblannr(self, A: Csr, intv, maxit, tol, vinit, pol: dict, cap=2000, want_vectors=False):
        iv = np.asarray(intv, dtype=np.float64)
        lam, res = np.zeros(cap), np.zeros(cap)
        W = np.zeros((cap, A.n)) if want_vectors else None
        nev, its = C.c_int(), C.c_int()
        mu = np.ascontiguousarray(pol["mu"])
        v = np.ascontiguousarray(vinit, dtype=np.float64)
        r = self.f("cheblannr")(A.n, _ptr(A.ia), _ptr(A.ja), _ptr(A.a), _ptr(iv), maxit,
                                C.c_double(tol), _ptr(v), pol["deg"], pol["type"],
                                C.c_double(pol["gam"]), C.c_double(pol["bar"]),
                                C.c_double(pol["cc"]), C.c_double(pol["dd"]), _ptr(mu),
                                C.byref(nev), C.byref(its), _ptr(lam), _ptr(res), _ptr(W), cap)
        m = min(nev.value, cap)
        out = dict(status=r, nev=nev.value, its=its.value, lam=lam[:m].copy(), res=res[:m].copy())
        if want_vectors:
            out["W"] = W[:m].copy()
        return out

    def pipeline(self, A: Csr, s: RunSpec, cap: int = 4000, slices=None) -> RunResult:
        """The whole run; with slices=(lo, hi) (reference build only) bounds,
        DOS and slicing run in full and ChebLanNr only on slices lo..hi-1."""
        spec = OrcSpec()
        spec.n = A.n
        spec.ia, spec.ja, spec.a = _ptr(A.ia), _ptr(A.ja), _ptr(A.a)
        for k, v in s.__dict__.items():
            setattr(spec, k, v)
        ns = s.nslices
        mu = np.zeros(s.Mdeg + 1)
        sli = np.zeros(ns + 1)
        deg, ptype, nev, its = (np.zeros(ns, dtype=np.int32) for _ in range(4))
        gam, bar = np.zeros(ns), np.zeros(ns)
        lam, res = np.zeros(ns * cap), np.zeros(ns * cap)
        out = OrcOut()
        out.cap = cap
        for name, arr in (("mu", mu), ("sli", sli), ("deg", deg), ("ptype", ptype), ("gam", gam),
                          ("bar", bar), ("nev", nev), ("its", its), ("lam", lam), ("res", res)):
            setattr(out, name, _ptr(arr))
        if slices is None:
            self.f("pipeline")(C.byref(spec), C.byref(out))
        else:
            self.f("pipeline_slices")(C.byref(spec), C.byref(out), int(slices[0]), int(slices[1]))
        rr = RunResult(out.lmin, out.lmax, out.ecount, out.npts, out.status, mu, sli, deg, ptype,
                       gam, bar, nev, its)
        for sl in range(ns):
            m = min(int(nev[sl]), cap)
            rr.lam.append(lam[sl * cap: sl * cap + m].copy())
            rr.res.append(res[sl * cap: sl * cap + m].copy())
        rr.times = dict(bounds=out.t_bounds, dos=out.t_dos, slicer=out.t_slicer,
                        slices=out.t_slices, total=out.t_total)
        return rr


def laplacian(nx: int, ny: int, nz: int) -> Csr:
    """Dirichlet Laplacian in the row/column order of LocalLapGen
    (TESTS/COMMON/lapl.c:4-70), vectorised with numpy."""
    n = nx * ny * nz
    idx = np.arange(n)
    k = idx // (nx * ny)
    i = (idx - k * nx * ny) // nx
    j = idx - k * nx * ny - i * nx
    d = 6.0 if nz > 1 else 4.0
    offs = [(-nx * ny, k > 0), (-nx, i > 0), (-1, j > 0), (0, np.ones(n, bool)),
            (1, j < nx - 1), (nx, i < ny - 1), (nx * ny, k < nz - 1)]
    if nz == 1:
        offs = [o for o in offs if abs(o[0]) != nx * ny or nx * ny == 1]
    cols = np.stack([idx + o for o, _ in offs], axis=1)
    mask = np.stack([m for _, m in offs], axis=1)
    vals = np.where(np.array([o for o, _ in offs])[None, :] == 0, d, -1.0)
    vals = np.broadcast_to(vals, cols.shape)
    counts = mask.sum(axis=1)
    ia = np.zeros(n + 1, dtype=np.int32)
    ia[1:] = np.cumsum(counts)
    ja = cols[mask].astype(np.int32)
    a = vals[mask].astype(np.float64)
    return Csr(n, ia, ja, np.ascontiguousarray(a))


def exact_eig_lap(nx: int, ny: int, nz: int, a: float, b: float) -> np.ndarray:
    """Analytic eigenvalues in [a-eps, b+eps]: ExactEigLap3
    (TESTS/COMMON/lapl.c:139-169)."""
    eps = np.finfo(np.float64).eps
    tx = np.sin(np.arange(1, nx + 1) * 0.5 * np.pi / (nx + 1.0))
    ty = np.sin(np.arange(1, ny + 1) * 0.5 * np.pi / (ny + 1.0))
    tz = np.sin(np.arange(1, nz + 1) * 0.5 * np.pi / (nz + 1.0)) if nz > 1 else np.zeros(1)
    ev = 4 * (tx[:, None, None] ** 2 + ty[None, :, None] ** 2 + tz[None, None, :] ** 2)
    ev = ev.ravel()
    return np.sort(ev[(ev >= a - eps) & (ev <= b + eps)])
