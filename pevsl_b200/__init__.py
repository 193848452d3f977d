"""pevsl_b200 — pEVSL's spectrum-slicing eigensolver on one NVIDIA B200.

The product is the C-ABI library ``libpevsl_b200.so`` (built in-tree by
``pevsl_b200.build``) that exports the pEVSL C API (include/pevsl.h) plus the
extensions of include/pevsl_b200.h.  This module binds it with ctypes and
mirrors the reference's driver-level interface (TESTS/Lap/LapPLanN.c,
TESTS/MM/MMPLanN.c) so tests and benchmarks read like the reference drivers:

    lib = pevsl_b200.load()
    A = pevsl_b200.Matrix.from_csr(n, ia, ja, a)
    with pevsl_b200.Instance(A) as ev:
        mu, ecnt = ev.kpmdos(Mdeg=300, damping=1, nvec=60, intv=[a, b, lmin, lmax])
        ...

There is no CPU fallback: ``load()`` raises if the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpevsl_b200.so")

RNG_GLIBC = 0
RNG_GAUSS = 1
PREC_FP64 = 0
PREC_MIXED = 1

# error codes of include/pevsl.h
PEVSL_NOT_IMPLEMENT = 11
ERR_CUDA = -1001
ERR_NOMEM = -1002
ERR_ARG = -1003
ERR_NOMATVEC = -1004
ERR_NONFINITE = -1005
ERR_EIG = -1006


class PevslError(RuntimeError):
    pass


# ---------------------------------------------------------------- structs
class Csr(C.Structure):
    _fields_ = [("nrows", C.c_int), ("ncols", C.c_int), ("ia", C.POINTER(C.c_int)),
                ("ja", C.POINTER(C.c_int)), ("a", C.POINTER(C.c_double))]


class Parcsr(C.Structure):
    _fields_ = [("comm", C.c_int), ("comm_handle", C.c_void_p),
                ("nrow_global", C.c_int), ("ncol_global", C.c_int),
                ("nrow_local", C.c_int), ("ncol_local", C.c_int),
                ("row_starts", C.POINTER(C.c_int)), ("col_starts", C.POINTER(C.c_int)),
                ("first_row", C.c_int), ("first_col", C.c_int),
                ("diag", C.POINTER(Csr)), ("offd", C.POINTER(Csr)),
                ("col_map_offd", C.POINTER(C.c_int))]


class Parvec(C.Structure):
    _fields_ = [("comm", C.c_int), ("n_global", C.c_int), ("n_local", C.c_int),
                ("n_first", C.c_int), ("data", C.c_void_p)]


class Parvecs(C.Structure):
    _fields_ = [("comm", C.c_int), ("n_global", C.c_int), ("n_local", C.c_int),
                ("n_first", C.c_int), ("n_vecs", C.c_int), ("ld", C.c_int),
                ("data", C.c_void_p)]


class Polparams(C.Structure):
    _fields_ = [("max_deg", C.c_int), ("min_deg", C.c_int), ("damping", C.c_int),
                ("thresh_ext", C.c_double), ("thresh_int", C.c_double),
                ("intvtol", C.c_double), ("type", C.c_int), ("mu", C.POINTER(C.c_double)),
                ("cc", C.c_double), ("dd", C.c_double), ("gam", C.c_double),
                ("bar", C.c_double), ("deg", C.c_int)]


class PevslData(C.Structure):
    _fields_ = [("comm", C.c_int), ("N", C.c_int), ("n", C.c_int), ("nfirst", C.c_int),
                ("ifGenEv", C.c_int), ("Amv", C.c_void_p), ("Bmv", C.c_void_p),
                ("Bsol", C.c_void_p), ("LTsol", C.c_void_p), ("stats", C.c_void_p),
                ("nev_computed", C.c_int), ("eval_computed", C.POINTER(C.c_double)),
                ("evec_computed", C.c_void_p), ("sigma_mult", C.c_double)]


MVFUNC = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p, C.c_void_p)

_lib = None
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p
_D = C.c_double
_I = C.c_int

# (name, restype, argtypes) of every exported symbol the binding uses; the
# CPU test suite checks that each one exists in the library.
SIGNATURES = [
    ("pEVSL_Start", _I, [_I, C.POINTER(C.POINTER(PevslData))]),
    ("pEVSL_Finish", _I, [C.POINTER(PevslData)]),
    ("pEVSL_SetAParcsr", _I, [C.POINTER(PevslData), C.POINTER(Parcsr)]),
    ("pEVSL_SetAMatvec", _I, [C.POINTER(PevslData), MVFUNC, _vp]),
    ("pEVSL_SetProbSizes", _I, [C.POINTER(PevslData), _I, _I, _I]),
    ("pEVSL_SetStdEig", _I, [C.POINTER(PevslData)]),
    ("pEVSL_SetGenEig", _I, [C.POINTER(PevslData)]),
    ("pEVSL_SetSigmaMult", _I, [C.POINTER(PevslData), _D]),
    ("pEVSL_ParcsrCreate", _I, [_I, _I, _ip, _ip, C.POINTER(Parcsr), _I]),
    ("pEVSL_ParcsrSetup", _I, [C.POINTER(Csr), C.POINTER(Parcsr)]),
    ("pEVSL_ParcsrFree", None, [C.POINTER(Parcsr)]),
    ("pEVSL_ParcsrMatvec", None, [C.POINTER(Parcsr), C.POINTER(Parvec), C.POINTER(Parvec)]),
    ("pEVSL_ParcsrMatvec0", None, [_vp, _vp, _vp]),
    ("pEVSL_ParcsrNnz", _I, [C.POINTER(Parcsr)]),
    ("pEVSL_ParcsrGetLocalMat", _I, [C.POINTER(Parcsr), _I, _vp, C.POINTER(Csr), C.c_char]),
    ("pEVSL_ParvecCreate", None, [_I, _I, _I, _I, C.POINTER(Parvec)]),
    ("pEVSL_ParvecFree", None, [C.POINTER(Parvec)]),
    ("pEVSL_ParvecRand", None, [C.POINTER(Parvec)]),
    ("pEVSL_ParvecDot", None, [C.POINTER(Parvec), C.POINTER(Parvec), _dp]),
    ("pEVSL_ParvecNrm2", None, [C.POINTER(Parvec), _dp]),
    ("pEVSL_ParvecSum", None, [C.POINTER(Parvec), _dp]),
    ("pEVSL_ParvecCopy", None, [C.POINTER(Parvec), C.POINTER(Parvec)]),
    ("pEVSL_ParvecScal", None, [C.POINTER(Parvec), _D]),
    ("pEVSL_ParvecAxpy", None, [_D, C.POINTER(Parvec), C.POINTER(Parvec)]),
    ("pEVSL_ParvecSetZero", None, [C.POINTER(Parvec)]),
    ("pEVSL_ParvecSetScalar", None, [C.POINTER(Parvec), _D]),
    ("pEVSL_ParvecsCreate", None, [_I, _I, _I, _I, _I, _I, C.POINTER(Parvecs)]),
    ("pEVSL_ParvecsFree", None, [C.POINTER(Parvecs)]),
    ("pEVSL_ParvecsGemv", None, [_D, C.POINTER(Parvecs), _I, _dp, _D, C.POINTER(Parvec)]),
    ("pEVSL_ParvecsGemtv", None, [_D, C.POINTER(Parvecs), _I, C.POINTER(Parvec), _D, _dp]),
    ("pEVSL_SetPolDef", None, [C.POINTER(Polparams)]),
    ("pEVSL_FindPol", _I, [_dp, C.POINTER(Polparams)]),
    ("pEVSL_FreePol", None, [C.POINTER(Polparams)]),
    ("pEVSL_Kpmdos", _I, [C.POINTER(PevslData), _I, _I, _I, _dp, _I, _I, _I, _dp, _dp]),
    ("pEVSL_SpslicerKpm", _I, [_dp, _dp, _I, _dp, _I, _I]),
    ("pEVSL_LanDosG", _I, [C.POINTER(PevslData), _I, _I, _I, _dp, _dp, _dp, _dp, _I, _I, _I]),
    ("pEVSL_SpslicerLan", None, [_dp, _dp, _I, _I, _dp]),
    ("pEVSL_LanTrbounds", _I, [C.POINTER(PevslData), _I, _I, _D, C.POINTER(Parvec), _I, _dp,
                               _dp, _vp]),
    ("pEVSL_ChebLanNr", _I, [C.POINTER(PevslData), _dp, _I, _D, C.POINTER(Parvec),
                             C.POINTER(Polparams), _ip, C.POINTER(_dp),
                             C.POINTER(C.POINTER(Parvecs)), C.POINTER(_dp), _vp]),
    ("pEVSL_StatsReset", None, [C.POINTER(PevslData)]),
    ("pEVSL_Part1d", None, [_I, _I, _ip, _ip, _ip, _I]),
    ("sort_double", None, [_I, _dp, _ip]),
    ("linspace", None, [_D, _D, _I, _dp]),
    ("pEVSL_B200_SetRng", _I, [_I, C.c_uint64]),
    ("pEVSL_B200_RngDraws", C.c_uint64, []),
    ("pEVSL_B200_LastIterations", _I, [C.POINTER(PevslData)]),
    ("pEVSL_B200_LastNconv", _I, [C.POINTER(PevslData)]),
    ("pEVSL_B200_LaunchCount", C.c_uint64, []),
    ("pEVSL_B200_PhaseMs", _D, [C.POINTER(PevslData), _I]),
    ("pEVSL_B200_Memcpy", _I, [_vp, _vp, C.c_size_t]),
    ("pEVSL_B200_Sync", _I, []),
    ("pEVSL_B200_LastError", _I, []),
    ("pEVSL_B200_ChebAv", _I, [C.POINTER(PevslData), C.POINTER(Polparams), _vp, _vp]),
    ("pEVSL_B200_ChebAvGen", _I, [C.POINTER(PevslData), C.POINTER(Polparams), _vp, _vp]),
    ("pEVSL_SetBParcsr", _I, [C.POINTER(PevslData), C.POINTER(Parcsr)]),
    ("pEVSL_B200_GenCounters", None, [C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), _dp, _dp]),
    ("pEVSL_B200_ResetGenCounters", None, []),
    ("pEVSL_B200_FlushL2", _I, [C.c_size_t]),
    ("pEVSL_SetBSol", _I, [C.POINTER(PevslData), _vp, _vp]),
    ("pEVSL_SetLTSol", _I, [C.POINTER(PevslData), _vp, _vp]),
    ("pEVSL_SetupLSPolRec", None, [_I, _D, _D, _D, C.POINTER(Parcsr), C.POINTER(_vp)]),
    ("pEVSL_SetupLSPolSqrt", None, [_I, _D, _D, _D, C.POINTER(Parcsr), C.POINTER(_vp)]),
    ("pEVSL_LSPolSol", None, [_vp, _vp, _vp]),
    ("pEVSL_LSPolFree", None, [_vp]),
    ("pEVSL_B200_LSPolCoefs", _I, [_I, _I, _D, _D, _D, _dp, _ip, _dp, _dp]),
    ("pEVSL_B200_LSPolDegree", _I, [_vp, _dp, _I]),
    ("pEVSL_ChebIterSetup", _I, [_D, _D, _I, C.POINTER(Parcsr), C.POINTER(_vp)]),
    ("pEVSL_ChebIterSolv1", None, [_vp, _vp, _vp]),
    ("pEVSL_ChebIterSolv2", None, [_vp, _vp, _vp]),
    ("pEVSL_ChebIterFree", None, [_vp]),
    ("pEVSL_ChebIterGetRes", _dp, [_vp]),
    ("pEVSL_ChebIterStatsPrint", None, [_vp, _vp]),
    ("pEVSL_B200_ReleaseWorkspace", None, []),
    ("pEVSL_B200_Info", _I, [C.c_char_p, _I]),
    ("pEVSL_B200_SetDevice", _I, [_I]),
    ("pEVSL_B200_EventRecord", _I, [_I]),
    ("pEVSL_B200_EventElapsedMs", _D, [_I, _I]),
    ("pEVSL_B200_HostAlloc", _vp, [C.c_size_t]),
    ("pEVSL_B200_HostFree", None, [_vp]),
    ("pEVSL_B200_ManagedAlloc", _vp, [C.c_size_t]),
    ("pEVSL_B200_ManagedFree", None, [_vp]),
    ("pEVSL_B200_MlpCreate", _I, [C.POINTER(_vp), _I, _I, _I, _I]),
    ("pEVSL_B200_MlpFree", None, [_vp]),
    ("pEVSL_B200_MlpParamCount", C.c_long, [_vp]),
    ("pEVSL_B200_MlpLayout", _I, [_vp, _ip, _ip, C.POINTER(C.c_long), C.POINTER(C.c_long)]),
    ("pEVSL_B200_MlpSetParams", _I, [_vp, C.POINTER(C.c_float)]),
    ("pEVSL_B200_MlpGetParams", _I, [_vp, C.POINTER(C.c_float)]),
    ("pEVSL_B200_MlpForward", _I, [_vp, _vp, _vp, _I]),
    ("pEVSL_B200_MlpGradients", _I, [_vp, _vp, _vp, _I, C.POINTER(C.c_float),
                                     C.POINTER(C.c_float)]),
    ("pEVSL_B200_MlpTrainStep", _I, [_vp, _vp, _vp, _I, C.c_float, C.POINTER(C.c_float)]),
    ("pEVSL_B200_FilterCounters", None, [C.POINTER(C.c_uint64), _dp, _dp]),
    ("pEVSL_B200_ResetFilterCounters", None, []),
    ("pEVSL_B200_SetPrecision", _I, [C.POINTER(PevslData), _I]),
    ("pEVSL_B200_LastFallbacks", _I, []),
    ("pEVSL_B200_SetFilterForm", _I, [_I]),
    ("pEVSL_B200_CopyEigenvectors", _I, [C.POINTER(Parvecs), _I, _dp, C.c_long]),
    ("pEVSL_B200_SetGroupReduce", _I, [C.POINTER(PevslData), _vp, _vp]),
    ("pEVSL_B200_ChebLanNrBatch", _I, [C.POINTER(PevslData), _I, _dp, _ip, _D,
                                       C.POINTER(Parvec), C.POINTER(Polparams), _ip,
                                       C.POINTER(_dp), C.POINTER(C.POINTER(Parvecs)),
                                       C.POINTER(_dp), _ip, _ip, _vp]),
    ("pEVSL_B200_ChebLanNrMulti", _I, [_I, C.POINTER(C.POINTER(PevslData)), _ip, _dp, _ip, _D,
                                       C.POINTER(C.POINTER(Parvec)), C.POINTER(Polparams), _ip,
                                       C.POINTER(_dp), C.POINTER(C.POINTER(Parvecs)),
                                       C.POINTER(_dp), _ip, _ip, _vp]),
]


def load(path: str = LIB_PATH):
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise PevslError(f"{path} is missing: build it with `python -m pevsl_b200.build`")
    lib = C.CDLL(path)
    for name, res, args in SIGNATURES:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _check(code, what):
    if code != 0:
        raise PevslError(f"{what} returned {code}")


def _ptr(a: np.ndarray, t=_dp):
    return a.ctypes.data_as(t)


def set_rng(mode: int, seed: int) -> None:
    """Choose the random stream: RNG_GLIBC (the reference's rand()) or
    RNG_GAUSS (Philox Gaussian on the GPU); restarts the draw counter."""
    _check(load().pEVSL_B200_SetRng(mode, seed), "pEVSL_B200_SetRng")


def launch_count() -> int:
    return int(load().pEVSL_B200_LaunchCount())


def filter_counters():
    """(launches, algorithmic bytes, device ms) of the fused filter kernel."""
    n, b, m = C.c_uint64(), C.c_double(), C.c_double()
    load().pEVSL_B200_FilterCounters(C.byref(n), C.byref(b), C.byref(m))
    return int(n.value), b.value, m.value


def pinned_empty(count: int, dtype) -> tuple:
    """A numpy array in page-locked host memory and its raw pointer (free
    with free_pinned)."""
    dt = np.dtype(dtype)
    p = load().pEVSL_B200_HostAlloc(max(1, count) * dt.itemsize)
    if not p:
        raise PevslError("pEVSL_B200_HostAlloc failed")
    buf = (C.c_char * (max(1, count) * dt.itemsize)).from_address(p)
    return np.frombuffer(buf, dtype=dt, count=count), p


def free_pinned(p) -> None:
    load().pEVSL_B200_HostFree(p)


def info() -> str:
    buf = C.create_string_buffer(512)
    load().pEVSL_B200_Info(buf, 512)
    return buf.value.decode()


# ---------------------------------------------------------------- vectors
class Vector:
    """A pevsl_Parvec owned by the library (managed memory)."""

    def __init__(self, n: int, values: np.ndarray | None = None):
        self.lib = load()
        self.pv = Parvec()
        self.lib.pEVSL_ParvecCreate(n, n, 0, 1, C.byref(self.pv))
        if not self.pv.data:
            raise PevslError("pEVSL_ParvecCreate failed")
        self.n = n
        if values is not None:
            self.set(values)

    def set(self, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        assert v.size == self.n
        _check(self.lib.pEVSL_B200_Memcpy(self.pv.data, v.ctypes.data, 8 * self.n), "memcpy")

    def get(self) -> np.ndarray:
        out = np.empty(self.n)
        _check(self.lib.pEVSL_B200_Memcpy(out.ctypes.data, self.pv.data, 8 * self.n), "memcpy")
        return out

    def free(self) -> None:
        if self.pv.data:
            self.lib.pEVSL_ParvecFree(C.byref(self.pv))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# ---------------------------------------------------------------- matrix
class Matrix:
    """A pevsl_Parcsr set up from a host CSR (one device CSR on the GPU)."""

    def __init__(self):
        self.lib = load()
        self.A = Parcsr()
        self.n = 0
        self.nnz = 0
        self._alive = False

    @classmethod
    def from_csr(cls, n: int, ia: np.ndarray, ja: np.ndarray, a: np.ndarray) -> "Matrix":
        m = cls()
        ia = np.ascontiguousarray(ia, dtype=np.int32)
        ja = np.ascontiguousarray(ja, dtype=np.int32)
        a = np.ascontiguousarray(a, dtype=np.float64)
        csr = Csr(n, n, _ptr(ia, _ip), _ptr(ja, _ip), _ptr(a))
        _check(m.lib.pEVSL_ParcsrCreate(n, n, None, None, C.byref(m.A), 1), "ParcsrCreate")
        _check(m.lib.pEVSL_ParcsrSetup(C.byref(csr), C.byref(m.A)), "ParcsrSetup")
        m.n, m.nnz, m._alive = n, int(ia[-1]), True
        return m

    def matvec(self, x: np.ndarray) -> np.ndarray:
        xv, yv = Vector(self.n, x), Vector(self.n)
        self.lib.pEVSL_ParcsrMatvec(C.byref(self.A), C.byref(xv.pv), C.byref(yv.pv))
        _check(self.lib.pEVSL_B200_LastError(), "ParcsrMatvec")
        return yv.get()

    def free(self) -> None:
        if self._alive:
            self.lib.pEVSL_ParcsrFree(C.byref(self.A))
            self._alive = False

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# ---------------------------------------------------------------- filters
@dataclass
class Filter:
    type: int
    deg: int
    gam: float
    bar: float
    cc: float
    dd: float
    mu: np.ndarray


def findpol(intv, max_deg=3000, damping=2, thresh_int=0.8, thresh_ext=0.2, deg_in=0):
    """pEVSL_SetPolDef + the driver overrides + pEVSL_FindPol
    (TESTS/Lap/LapPLanN.c:214-226).  Returns (code, Filter or None)."""
    lib = load()
    pol = Polparams()
    lib.pEVSL_SetPolDef(C.byref(pol))
    pol.damping, pol.thresh_int, pol.thresh_ext = damping, thresh_int, thresh_ext
    pol.max_deg, pol.deg = max_deg, deg_in
    iv = np.asarray(intv, dtype=np.float64)
    r = lib.pEVSL_FindPol(_ptr(iv), C.byref(pol))
    if r:
        return r, None
    mu = np.ctypeslib.as_array(pol.mu, shape=(pol.deg + 1,)).copy()
    f = Filter(pol.type, pol.deg, pol.gam, pol.bar, pol.cc, pol.dd, mu)
    lib.pEVSL_FreePol(C.byref(pol))
    return 0, f


def findpol_many(intvs, max_deg=3000, damping=2, thresh_int=0.8, thresh_ext=0.2):
    """findpol for every slice, the slices on concurrent host threads
    (pEVSL_FindPol keeps no shared state and ctypes releases the GIL, so
    each result is the one a lone call gives).  Returns [(code, Filter or
    None)] in slice order."""
    from concurrent.futures import ThreadPoolExecutor
    load()  # once, before the threads
    intvs = list(intvs)
    if len(intvs) <= 1:
        return [findpol(iv, max_deg, damping, thresh_int, thresh_ext) for iv in intvs]
    workers = min(len(intvs), os.cpu_count() or 1)
    with ThreadPoolExecutor(max_workers=workers) as ex:
        return list(ex.map(lambda iv: findpol(iv, max_deg, damping, thresh_int, thresh_ext),
                           intvs))


def _polparams(f: Filter):
    pol = Polparams()
    load().pEVSL_SetPolDef(C.byref(pol))
    mu = np.ascontiguousarray(f.mu, dtype=np.float64)
    pol.type, pol.deg, pol.gam, pol.bar, pol.cc, pol.dd = f.type, f.deg, f.gam, f.bar, f.cc, f.dd
    pol.mu = _ptr(mu)
    return pol, mu


def spslicer_kpm(mu, Mdeg, intv, n_int, npts):
    sli = np.zeros(n_int + 1)
    mu = np.ascontiguousarray(mu, dtype=np.float64)
    iv = np.asarray(intv, dtype=np.float64)
    r = load().pEVSL_SpslicerKpm(_ptr(sli), _ptr(mu), Mdeg, _ptr(iv), n_int, npts)
    return r, sli


def spslicer_lan(xi, yi, n_int):
    xi = np.ascontiguousarray(xi, dtype=np.float64)
    yi = np.ascontiguousarray(yi, dtype=np.float64).copy()
    sli = np.zeros(n_int + 1)
    load().pEVSL_SpslicerLan(_ptr(xi), _ptr(yi), n_int, len(xi), _ptr(sli))
    return sli


# ---------------------------------------------------------------- instance
class BSolver:
    """A B-solver of the library on a parcsr B, usable as the B-solve or
    L^{-T}-solve of a generalized instance: kind "lsrec" (least-squares
    polynomial for 1/x, pEVSL_SetupLSPolRec), "lssqrt" (1/sqrt(x),
    pEVSL_SetupLSPolSqrt), "cheb1" / "cheb2" (Chebyshev iteration of the
    first / second kind, pEVSL_ChebIterSetup) on the spectrum enclosure
    [lmin, lmax] of B; `deg` is max_deg for the polynomials, the number of
    iterations for the Chebyshev iterations."""

    def __init__(self, B: Matrix, kind: str, lmin: float, lmax: float, deg: int, tol: float = 1e-6):
        self.lib, self.B, self.kind = load(), B, kind
        self.h = C.c_void_p()
        if kind in ("lsrec", "lssqrt"):
            f = self.lib.pEVSL_SetupLSPolRec if kind == "lsrec" else self.lib.pEVSL_SetupLSPolSqrt
            f(deg, tol, lmin, lmax, C.byref(B.A), C.byref(self.h))
            if not self.h.value:
                raise PevslError(f"pEVSL_SetupLSPol ({kind}) failed")
            self.func = C.cast(self.lib.pEVSL_LSPolSol, C.c_void_p)
        elif kind in ("cheb1", "cheb2"):
            _check(self.lib.pEVSL_ChebIterSetup(lmin, lmax, deg, C.byref(B.A), C.byref(self.h)),
                   "ChebIterSetup")
            self.func = C.cast(self.lib.pEVSL_ChebIterSolv1 if kind == "cheb1"
                               else self.lib.pEVSL_ChebIterSolv2, C.c_void_p)
        else:
            raise ValueError(kind)

    @property
    def degree(self) -> int:
        """degree of a least-squares polynomial"""
        return self.lib.pEVSL_B200_LSPolDegree(self.h, None, 0)

    def coefficients(self) -> np.ndarray:
        d = self.degree
        mu = np.zeros(d + 1)
        self.lib.pEVSL_B200_LSPolDegree(self.h, _ptr(mu), d + 1)
        return mu

    def solve(self, b: np.ndarray) -> np.ndarray:
        """x = the solver applied to b (called as a user would call it)"""
        bv, xv = Vector(self.B.n, b), Vector(self.B.n)
        fn = C.CFUNCTYPE(None, _vp, _vp, _vp)(self.func.value)
        fn(bv.pv.data, xv.pv.data, self.h)
        _check(self.lib.pEVSL_B200_LastError(), "B-solve")
        x = xv.get()
        bv.free()
        xv.free()
        return x

    def free(self):
        if self.h.value:
            if self.kind.startswith("ls"):
                self.lib.pEVSL_LSPolFree(self.h)
            else:
                self.lib.pEVSL_ChebIterFree(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def lspol_coefs(kind: int, max_deg: int, tol: float, lmin: float, lmax: float):
    """Host-only least-squares coefficients of 1/x (kind 0) or 1/sqrt(x)
    (kind 1) on [lmin, lmax]: (deg, mu[0..deg], cc, dd)."""
    mu = np.zeros(max_deg)
    deg, cc, dd = C.c_int(), C.c_double(), C.c_double()
    _check(load().pEVSL_B200_LSPolCoefs(kind, max_deg, tol, lmin, lmax, _ptr(mu), C.byref(deg),
                                        C.byref(cc), C.byref(dd)), "LSPolCoefs")
    return deg.value, mu[:deg.value + 1].copy(), cc.value, dd.value


class Instance:
    """One pEVSL instance (pEVSL_Start ... pEVSL_Finish) bound to a matrix."""

    def __init__(self, A: Matrix | None = None):
        self.lib = load()
        self.p = C.POINTER(PevslData)()
        _check(self.lib.pEVSL_Start(1, C.byref(self.p)), "pEVSL_Start")
        self.A = A
        if A is not None:
            _check(self.lib.pEVSL_SetAParcsr(self.p, C.byref(A.A)), "SetAParcsr")

    @property
    def n(self) -> int:
        return self.p.contents.n

    def set_generalized(self, B: Matrix, bsol: BSolver, ltsol: BSolver | None = None) -> None:
        """A x = lambda B x: B as the parcsr B matvec, bsol as the B-solve,
        ltsol (B^{-1/2} or another L^{-T}) for the DOS start vectors."""
        _check(self.lib.pEVSL_SetBParcsr(self.p, C.byref(B.A)), "SetBParcsr")
        _check(self.lib.pEVSL_SetBSol(self.p, bsol.func, bsol.h), "SetBSol")
        if ltsol is not None:
            _check(self.lib.pEVSL_SetLTSol(self.p, ltsol.func, ltsol.h), "SetLTSol")
        _check(self.lib.pEVSL_SetGenEig(self.p), "SetGenEig")
        self._gen = (B, bsol, ltsol)

    def set_precision(self, precision: int) -> None:
        """PREC_FP64 (default) or PREC_MIXED (FP32 filter and KPM moments,
        FP64 Lanczos basis / reorthogonalisation / refinement)."""
        _check(self.lib.pEVSL_B200_SetPrecision(self.p, precision), "SetPrecision")

    def close(self):
        if self.p:
            self.lib.pEVSL_Finish(self.p)
            self.p = C.POINTER(PevslData)()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def kpmdos(self, Mdeg, damping, nvec, intv, ngroups=1, groupid=0):
        """pEVSL_Kpmdos; with ngroups > 1 this instance computes group
        `groupid`'s share of the vectors and the sum over the groups goes
        through the reduction installed by pEVSL_B200_SetGroupReduce."""
        mu = np.zeros(Mdeg + 1)
        ec = C.c_double()
        iv = np.asarray(intv, dtype=np.float64)
        r = self.lib.pEVSL_Kpmdos(self.p, Mdeg, damping, nvec, _ptr(iv), ngroups, groupid, 0,
                                  _ptr(mu), C.byref(ec))
        return r, mu, ec.value

    def landos(self, nvec, msteps, npts, intv):
        xd, yd = np.zeros(npts), np.zeros(npts)
        ne = C.c_double()
        iv = np.asarray(intv, dtype=np.float64)
        r = self.lib.pEVSL_LanDosG(self.p, nvec, msteps, npts, _ptr(xd), _ptr(yd), C.byref(ne),
                                   _ptr(iv), 1, 0, 0)
        return r, xd, yd, ne.value

    def lantrbounds(self, lanm, maxit, tol, vinit: np.ndarray, bndtype=1):
        v = Vector(self.n, vinit)
        lo, hi = C.c_double(), C.c_double()
        r = self.lib.pEVSL_LanTrbounds(self.p, lanm, maxit, tol, C.byref(v.pv), bndtype,
                                       C.byref(lo), C.byref(hi), None)
        return r, lo.value, hi.value

    def chebav(self, f: Filter, v: np.ndarray) -> np.ndarray:
        pol, _keep = _polparams(f)
        vv, yv = Vector(self.n, v), Vector(self.n)
        _check(self.lib.pEVSL_B200_ChebAv(self.p, C.byref(pol), vv.pv.data, yv.pv.data), "ChebAv")
        return yv.get()

    def cheblannr(self, intv, maxit, tol, vinit, f: Filter, want_vectors=False):
        """pEVSL_ChebLanNr; pairs sorted ascending as the drivers do."""
        pol, _keep = _polparams(f)
        v = vinit if isinstance(vinit, Vector) else Vector(self.n, vinit)
        iv = np.asarray(intv, dtype=np.float64)
        nev = C.c_int()
        lam, res = _dp(), _dp()
        W = C.POINTER(Parvecs)()
        r = self.lib.pEVSL_ChebLanNr(self.p, _ptr(iv), maxit, tol, C.byref(v.pv), C.byref(pol),
                                     C.byref(nev), C.byref(lam), C.byref(W), C.byref(res), None)
        out = dict(status=r, nev=nev.value, its=self.lib.pEVSL_B200_LastIterations(self.p),
                   nconv=self.lib.pEVSL_B200_LastNconv(self.p))
        m = nev.value
        libc = C.CDLL(None)
        libc.free.argtypes = [_vp]
        if r == 0:
            lam_a = np.ctypeslib.as_array(lam, shape=(m,)).copy() if m else np.zeros(0)
            res_a = np.ctypeslib.as_array(res, shape=(m,)).copy() if m else np.zeros(0)
            order = np.argsort(lam_a, kind="stable")
            out["lam"], out["res"] = lam_a[order], res_a[order]
            if want_vectors and m:
                Wh = np.empty((m, self.n))
                _check(self.lib.pEVSL_B200_CopyEigenvectors(W, m, _ptr(Wh), self.n),
                       "CopyEigenvectors")
                out["W"] = Wh[order].copy()
            if lam:
                libc.free(C.cast(lam, _vp))
            if res:
                libc.free(C.cast(res, _vp))
            if W:
                self.lib.pEVSL_ParvecsFree(W)
                libc.free(C.cast(W, _vp))
        for k, ph in (("t_iter_ms", 2), ("t_pol_ms", 3), ("t_reorth_ms", 4), ("t_ritz_ms", 5)):
            out[k] = self.lib.pEVSL_B200_PhaseMs(self.p, ph)
        return out


def _free_outputs(lib, lam, res, W):
    libc = C.CDLL(None)
    libc.free.argtypes = [_vp]
    if lam:
        libc.free(C.cast(lam, _vp))
    if res:
        libc.free(C.cast(res, _vp))
    if W:
        lib.pEVSL_ParvecsFree(W)
        libc.free(C.cast(W, _vp))


def cheblannr_batch(ev: "Instance", intvs, maxits, tol, vinit, filters, fstats=None):
    """pEVSL_B200_ChebLanNrBatch: all slices in lockstep; a list of per-slice
    dicts like Instance.cheblannr (without vectors).  fstats: a C FILE*
    (e.g. from open_log) that receives the solver's log, as the reference's
    fstats argument does (SRC/cheblanNr.c:298: one line per convergence
    test with the trace of the Ritz values above the bar)."""
    lib = ev.lib
    ns = len(filters)
    pols = (Polparams * max(ns, 1))()
    keep = []
    for i, f in enumerate(filters):
        p, mu = _polparams(f)
        pols[i] = p
        keep.append(mu)
    v = vinit if isinstance(vinit, Vector) else Vector(ev.n, vinit)
    iv = np.ascontiguousarray(np.asarray(intvs, dtype=np.float64).reshape(-1))
    mx = np.ascontiguousarray(maxits, dtype=np.int32)
    nev = np.zeros(ns, np.int32)
    its = np.zeros(ns, np.int32)
    status = np.zeros(ns, np.int32)
    lam = (_dp * max(ns, 1))()
    res = (_dp * max(ns, 1))()
    W = (C.POINTER(Parvecs) * max(ns, 1))()
    r = lib.pEVSL_B200_ChebLanNrBatch(ev.p, ns, _ptr(iv), _ptr(mx, _ip), tol, C.byref(v.pv),
                                      pols, _ptr(nev, _ip), lam, W, res, _ptr(its, _ip),
                                      _ptr(status, _ip), fstats)
    outs = []
    for i in range(ns):
        m = int(nev[i])
        o = dict(status=int(status[i]), nev=m, its=int(its[i]))
        if status[i] == 0:
            la = np.ctypeslib.as_array(lam[i], shape=(m,)).copy() if m else np.zeros(0)
            rs = np.ctypeslib.as_array(res[i], shape=(m,)).copy() if m else np.zeros(0)
            order = np.argsort(la, kind="stable")
            o["lam"], o["res"] = la[order], rs[order]
        _free_outputs(lib, lam[i], res[i], W[i])
        outs.append(o)
    return r, outs


def cheblannr_multi(problems):
    """pEVSL_B200_ChebLanNrMulti: several problems, all their slices in
    lockstep.  problems is a list of (Instance, intvs, maxits, tol, vinit,
    filters); tol is taken from the first.  Returns (code, list per problem of
    per-slice dicts like cheblannr_batch)."""
    if not problems:
        return 0, []
    lib = problems[0][0].lib
    tol = problems[0][3]
    nprob = len(problems)
    ns = [len(p[5]) for p in problems]
    tot = sum(ns)
    pevs = (C.POINTER(PevslData) * nprob)(*[p[0].p for p in problems])
    vecs, keep = [], []
    for p in problems:
        v = p[4] if isinstance(p[4], Vector) else Vector(p[0].n, p[4])
        keep.append(v)
        vecs.append(C.pointer(v.pv))
    vin = (C.POINTER(Parvec) * nprob)(*vecs)
    pols = (Polparams * max(tot, 1))()
    iv = np.zeros(4 * max(tot, 1))
    mx = np.zeros(max(tot, 1), np.int32)
    o = 0
    for p in problems:
        for k, f in enumerate(p[5]):
            pp, mu = _polparams(f)
            pols[o] = pp
            keep.append(mu)
            iv[4 * o:4 * o + 4] = p[1][k]
            mx[o] = p[2][k]
            o += 1
    nsl = np.ascontiguousarray(ns, np.int32)
    nev = np.zeros(max(tot, 1), np.int32)
    its = np.zeros(max(tot, 1), np.int32)
    status = np.zeros(max(tot, 1), np.int32)
    lam = (_dp * max(tot, 1))()
    res = (_dp * max(tot, 1))()
    W = (C.POINTER(Parvecs) * max(tot, 1))()
    r = lib.pEVSL_B200_ChebLanNrMulti(nprob, pevs, _ptr(nsl, _ip), _ptr(iv), _ptr(mx, _ip), tol,
                                      vin, pols, _ptr(nev, _ip), lam, W, res, _ptr(its, _ip),
                                      _ptr(status, _ip), None)
    outs, o = [], 0
    for p in problems:
        per = []
        for _ in p[5]:
            m = int(nev[o])
            d = dict(status=int(status[o]), nev=m, its=int(its[o]))
            if status[o] == 0:
                la = np.ctypeslib.as_array(lam[o], shape=(m,)).copy() if m else np.zeros(0)
                rs = np.ctypeslib.as_array(res[o], shape=(m,)).copy() if m else np.zeros(0)
                order = np.argsort(la, kind="stable")
                d["lam"], d["res"] = la[order], rs[order]
            _free_outputs(lib, lam[o], res[o], W[o])
            per.append(d)
            o += 1
        outs.append(per)
    for v, p in zip(keep[:nprob], problems):
        if v is not p[4]:
            v.free()
    return r, outs


class ManagedArray:
    """A CUDA managed-memory array (pEVSL_B200_ManagedAlloc) with a numpy view."""

    def __init__(self, shape, dtype=np.float32):
        self.lib = load()
        self.dtype = np.dtype(dtype)
        self.shape = tuple(shape) if hasattr(shape, "__len__") else (int(shape),)
        nbytes = int(np.prod(self.shape)) * self.dtype.itemsize
        self.ptr = self.lib.pEVSL_B200_ManagedAlloc(nbytes)
        if not self.ptr:
            raise PevslError("pEVSL_B200_ManagedAlloc failed")
        buf = (C.c_char * nbytes).from_address(self.ptr)
        self.a = np.frombuffer(buf, dtype=self.dtype).reshape(self.shape)

    def set(self, x):
        self.lib.pEVSL_B200_Sync()
        self.a[...] = x
        return self

    def get(self):
        self.lib.pEVSL_B200_Sync()
        return self.a.copy()

    def free(self):
        if self.ptr:
            self.a = None
            self.lib.pEVSL_B200_ManagedFree(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Mlp:
    """The learned-DOS network (pEVSL_B200_Mlp*): nin -> width -> ... -> nout,
    GELU between the `layers` linear maps, BF16 weights, FP32 accumulation."""

    def __init__(self, nin, width, nout, layers):
        self.lib = load()
        self.p = _vp()
        _check(self.lib.pEVSL_B200_MlpCreate(C.byref(self.p), nin, width, nout, layers), "MlpCreate")
        self.nin, self.width, self.nout, self.layers = nin, width, nout, layers
        self.np = int(self.lib.pEVSL_B200_MlpParamCount(self.p))

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.np
        _check(self.lib.pEVSL_B200_MlpSetParams(self.p, p.ctypes.data_as(C.POINTER(C.c_float))),
               "MlpSetParams")

    def get_params(self):
        p = np.zeros(self.np, np.float32)
        _check(self.lib.pEVSL_B200_MlpGetParams(self.p, p.ctypes.data_as(C.POINTER(C.c_float))),
               "MlpGetParams")
        return p

    def forward(self, X: ManagedArray, Y: ManagedArray, B):
        _check(self.lib.pEVSL_B200_MlpForward(self.p, X.ptr, Y.ptr, B), "MlpForward")

    def gradients(self, X: ManagedArray, T: ManagedArray, B):
        loss = C.c_float()
        g = np.zeros(self.np, np.float32)
        _check(self.lib.pEVSL_B200_MlpGradients(self.p, X.ptr, T.ptr, B, C.byref(loss),
                                                g.ctypes.data_as(C.POINTER(C.c_float))),
               "MlpGradients")
        return float(loss.value), g

    def train_step(self, X: ManagedArray, T: ManagedArray, B, lr, want_loss=False):
        loss = C.c_float()
        _check(self.lib.pEVSL_B200_MlpTrainStep(self.p, X.ptr, T.ptr, B, lr,
                                                C.byref(loss) if want_loss else None),
               "MlpTrainStep")
        return float(loss.value) if want_loss else None

    def close(self):
        if self.p:
            self.lib.pEVSL_B200_MlpFree(self.p)
            self.p = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- whole run
@dataclass
class SliceRun:
    """Inputs of one spectrum-slicing run (the driver sequence of
    TESTS/Lap/LapPLanN.c with the bounds step of TESTS/MM/MMPLanN.c)."""
    a_lo: float
    b_hi: float
    nslices: int
    bounds_mode: int = 0          # 0: lmin/lmax given, 1: pEVSL_LanTrbounds
    lmin: float = 0.0
    lmax: float = 12.0
    lan_lanm: int = 50
    lan_maxit: int = 200
    lan_bndtype: int = 1
    lan_tol: float = 1e-8
    dos_type: int = 0             # 0: KPM, 1: Lanczos DOS
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
    rng_mode: int = RNG_GLIBC
    seed: int = 0


@dataclass
class SliceResult:
    lmin: float
    lmax: float
    ecount: float
    npts: int
    status: int
    mu: np.ndarray
    sli: np.ndarray
    deg: list = field(default_factory=list)
    ptype: list = field(default_factory=list)
    gam: list = field(default_factory=list)
    bar: list = field(default_factory=list)
    nev: list = field(default_factory=list)
    its: list = field(default_factory=list)
    lam: list = field(default_factory=list)
    res: list = field(default_factory=list)
    times: dict = field(default_factory=dict)
    fallbacks: int = 0            # mixed form: slices solved again in FP64


def gen_counters():
    """(filters, degrees, bytes, ms) of the generalized filter since the
    last reset (pEVSL_B200_GenCounters)."""
    f, d = C.c_uint64(), C.c_uint64()
    b, ms = C.c_double(), C.c_double()
    load().pEVSL_B200_GenCounters(C.byref(f), C.byref(d), C.byref(b), C.byref(ms))
    return f.value, d.value, b.value, ms.value


def open_log(path: str):
    """A C FILE* opened for writing (libc fopen), for the solvers' fstats
    argument; close it with close_log."""
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    f = libc.fopen(path.encode(), b"w")
    if not f:
        raise PevslError(f"cannot open {path}")
    return C.c_void_p(f)


def close_log(f) -> None:
    libc = C.CDLL(None)
    libc.fclose.argtypes = [C.c_void_p]
    libc.fclose(f)


def solve_interval(A: Matrix, s: SliceRun, batched: bool = False,
                   precision: int = PREC_FP64, setup=None, fstats=None) -> SliceResult:
    """Run the whole slicing path through the C API, in the reference
    drivers' order: start vector, bounds, DOS, slicer, then each slice
    (one pEVSL_ChebLanNr per slice, or all slices in lockstep through
    pEVSL_B200_ChebLanNrBatch when batched).  setup(instance), if given,
    runs right after pEVSL_Start (e.g. Instance.set_generalized)."""
    import time
    lib = load()
    t_all = time.perf_counter()
    set_rng(s.rng_mode, s.seed)
    with Instance(A) as ev:
        # pEVSL_Start reseeds rand() with srand(0); restart the chosen stream
        set_rng(s.rng_mode, s.seed)
        ev.set_precision(precision)
        if setup is not None:
            setup(ev)
        vinit = Vector(A.n)
        lib.pEVSL_ParvecRand(C.byref(vinit.pv))
        times = {}
        t = time.perf_counter()
        if s.bounds_mode == 1:
            lo, hi = C.c_double(), C.c_double()
            r = lib.pEVSL_LanTrbounds(ev.p, s.lan_lanm, s.lan_maxit, s.lan_tol, C.byref(vinit.pv),
                                      s.lan_bndtype, C.byref(lo), C.byref(hi), None)
            _check(r, "LanTrbounds")
            lmin, lmax = lo.value, hi.value
        else:
            lmin, lmax = s.lmin, s.lmax
        times["bounds"] = time.perf_counter() - t
        intv = [s.a_lo, s.b_hi, lmin, lmax]
        status = 0
        t = time.perf_counter()
        mu = np.zeros(s.Mdeg + 1)
        if s.dos_type == 0:
            r, mu, ecount = ev.kpmdos(s.Mdeg, s.kpm_damping, s.nvec, intv)
            if r:
                status = 100 + r
            npts = int(10 * ecount)
            times["dos"] = time.perf_counter() - t
            r, sli = spslicer_kpm(mu, s.Mdeg, intv, s.nslices, npts)
            if r and not status:
                status = 200 + r
        else:
            r, xd, yd, ecount = ev.landos(s.nvec, s.landos_msteps, s.landos_npts, intv)
            if r:
                status = 100 + r
            npts = s.landos_npts
            times["dos"] = time.perf_counter() - t
            sli = spslicer_lan(xd, yd, s.nslices)
        res = SliceResult(lmin, lmax, ecount, npts, status, mu, sli)
        ev_int = int(1 + ecount / float(s.nslices))
        t = time.perf_counter()
        # every slice's filter at once, on host threads (the same filters as
        # designing them one slice at a time)
        slice_ivs = [[sli[sl], sli[sl + 1], lmin, lmax] for sl in range(s.nslices)]
        designed = findpol_many(slice_ivs, s.pol_max_deg, s.pol_damping, s.thresh_int,
                                s.thresh_ext)
        if batched:
            nev = ev_int + 2
            mlan = min(max(5 * nev, s.mlan_min), A.n)
            filters, intvs = [], []
            for sl in range(s.nslices):
                r, f = designed[sl]
                if r:
                    raise PevslError(f"pEVSL_FindPol returned {r} for slice {sl}")
                filters.append(f)
                intvs.append(slice_ivs[sl])
            r, outs = cheblannr_batch(ev, intvs, [mlan] * s.nslices, s.tol, vinit, filters,
                                      fstats)
            res.fallbacks = int(lib.pEVSL_B200_LastFallbacks())
            for f, out in zip(filters, outs):
                if out["status"] and not res.status:
                    res.status = 300 + abs(out["status"])
                res.deg.append(f.deg)
                res.ptype.append(f.type)
                res.gam.append(f.gam)
                res.bar.append(f.bar)
                res.nev.append(out["nev"])
                res.its.append(out["its"])
                res.lam.append(out.get("lam", np.zeros(0)))
                res.res.append(out.get("res", np.zeros(0)))
        for sl in range(0 if not batched else s.nslices, s.nslices):
            nev = ev_int + 2
            mlan = min(max(5 * nev, s.mlan_min), A.n)
            iv = slice_ivs[sl]
            r, f = designed[sl]
            if r:
                res.status = res.status or 300 + abs(r)
                continue
            out = ev.cheblannr(iv, mlan, s.tol, vinit, f)
            res.fallbacks += int(lib.pEVSL_B200_LastFallbacks())
            if out["status"] and not res.status:
                res.status = 300 + abs(out["status"])
            res.deg.append(f.deg)
            res.ptype.append(f.type)
            res.gam.append(f.gam)
            res.bar.append(f.bar)
            res.nev.append(out["nev"])
            res.its.append(out["its"])
            res.lam.append(out.get("lam", np.zeros(0)))
            res.res.append(out.get("res", np.zeros(0)))
        times["slices"] = time.perf_counter() - t
        times["total"] = time.perf_counter() - t_all
        res.times = times
        vinit.free()
    return res
