"""The allocation-free projection entry point, pEVSL_B200_ParvecsGemtvNoAlloc.

It exists for callers that must not let the library allocate device memory
(a framework that owns all device memory through its own pool, loops that
cannot afford cudaMalloc's device synchronisation, programs with a fixed
memory budget).  It computes w = V(:,0:k)' x into caller memory with only a
fixed scratch array of the library as workspace.  This test calls it through
the C-ABI twice in a row with different inputs and checks each result
against the allocating entry point pEVSL_ParvecsGemtv (and numpy) to 1e-13
relative, the tolerance of the other Gram-Schmidt tests; it checks that a
third, warmed-up call leaves the device's free memory (cudaMemGetInfo, read
through torch) unchanged, and that sizes beyond the limit (k > 256) are
refused with an error code.

The file name makes pytest collect it last.
"""
import ctypes as C

import numpy as np
import pytest

import pevsl_b200 as pv

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_gemtv_no_alloc_matches_allocating_entry_point():
    lib = pv.load()
    f = lib.pEVSL_B200_ParvecsGemtvNoAlloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_long, C.c_long, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    n, k, ld = 30011, 97, 30016
    rng = np.random.default_rng(2024)
    # inputs and outputs are allocated by the caller (here through the
    # regular API); the entry point itself allocates nothing
    X = pv.Parvecs()
    lib.pEVSL_ParvecsCreate(n, k, ld, n, 0, 1, C.byref(X))
    Vh = np.zeros((k, ld))
    Vh[:, :n] = rng.standard_normal((k, n))
    assert lib.pEVSL_B200_Memcpy(X.data, Vh.ctypes.data, Vh.nbytes) == 0
    w = pv.Vector(k)
    try:
        for call in range(2):
            x = pv.Vector(n, rng.standard_normal(n) * (call + 1))
            assert f(X.data, n, ld, k, x.pv.data, w.pv.data, None) == 0
            assert lib.pEVSL_B200_Sync() == 0
            got = w.get()
            ref = np.zeros(k)
            lib.pEVSL_ParvecsGemtv(1.0, C.byref(X), k, C.byref(x.pv), 0.0,
                                   ref.ctypes.data_as(C.POINTER(C.c_double)))
            assert rel(got, ref) <= 1e-13, call
            assert rel(got, Vh[:, :n] @ x.get()) <= 1e-13, call
            x.free()
        # a warmed-up call takes no device memory: the free bytes that the
        # driver reports are the same before and after it
        import torch
        x = pv.Vector(n, rng.standard_normal(n))
        assert lib.pEVSL_B200_Sync() == 0
        free0, _ = torch.cuda.mem_get_info()
        assert f(X.data, n, ld, k, x.pv.data, w.pv.data, None) == 0
        assert lib.pEVSL_B200_Sync() == 0
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0, (free0, free1)
        assert rel(w.get(), Vh[:, :n] @ x.get()) <= 1e-13
        x.free()
        # sizes beyond the stated maximum are refused, nothing is launched
        assert f(X.data, n, ld, 257, w.pv.data, w.pv.data, None) == pv.ERR_ARG
        assert f(X.data, n, ld, 0, w.pv.data, w.pv.data, None) == pv.ERR_ARG
        assert f(X.data, n, n - 1, k, w.pv.data, w.pv.data, None) == pv.ERR_ARG
    finally:
        w.free()
        lib.pEVSL_ParvecsFree(C.byref(X))
