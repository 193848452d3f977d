"""Parity at the benchmark's own configuration: the 100^3 Laplacian
(n = 1e6), interval [0.80, 0.82], 4 slices, thick-restart bounds, KPM with
30 seeded Gaussian vectors, filters FindPol(damping 2, 0.8 / 0.2), ChebLanNr
tol 1e-8 -- the run bench.py times.

The fixture tests/golden/lap100_c2.json is the reference build's own run of
exactly these inputs (tests/golden/make_golden.py c2, oracle/_ref, one
process per slice).  Checked: bounds within 1e-10 relative, slice ends
within 1e-12, filter degrees and per-slice counts identical,
eigenvalues within 1e-10 relative, every residual <= 1e-8 (absolute and
relative to |lambda|), and the total equal to the analytic count of
ExactEigLap3 (TESTS/COMMON/lapl.c:139-169).  The lockstep (batched) path is
the one timed; it gives each slice the bits of solving it alone.

Lanczos steps: equal to the reference's, or a whole number of convergence-
test cycles (20 steps) apart -- at C2 slices 0, 2 and 3 stop at the
reference's step (431, 531, 431) and slice 1 at 511 against the
reference's 551.  The reference's test (SRC/cheblanNr.c:293-331) stops a slice
when the sum of its Ritz values above the bar changes by less than 2e-12
between two tests; at C2 that sum is about 5.4e7, whose ulp (7.5e-9) is
3700 times the threshold, so the test fires only when two consecutive sums
are bit-identical.  One ulp of difference in any of the ~130 summed Ritz
values -- the tridiagonal eigensolver (LAPACK DSTEV there, an implicit QR
here) and the dot products (OpenBLAS there, fixed-order GPU reductions here)
round differently -- moves the stop by a cycle or more; the eigenpairs it
returns are the converged ones either way (counts identical, eigenvalues to
1e-10, residuals <= 1e-8).
"""
import numpy as np
import pytest

import pevsl_b200 as pv
from checkers import exact_eig_lap, laplacian
from conftest import golden

pytestmark = pytest.mark.gpu


def test_c2_run_matches_reference_build(gpu):
    g = golden("lap100_c2.json")
    spec = g["spec"]
    A = laplacian(*g["grid"])
    M = pv.Matrix.from_csr(A.n, A.ia, A.ja, A.a)
    r = pv.solve_interval(M, pv.SliceRun(**spec), batched=True)
    M.free()
    assert r.status == 0 and g["status"] == 0
    assert abs(r.lmin - g["lmin"]) <= 1e-10 * abs(g["lmax"])
    assert abs(r.lmax - g["lmax"]) <= 1e-10 * abs(g["lmax"])
    assert np.max(np.abs(np.asarray(r.sli) - g["sli"])) <= 1e-12 * np.max(np.abs(g["sli"]))
    assert list(r.deg) == g["deg"]
    assert list(r.nev) == g["nev"]
    for its, ref in zip(r.its, g["its"]):
        assert (its - ref) % 20 == 0, (list(r.its), g["its"])
    assert sum(a == b for a, b in zip(r.its, g["its"])) >= 3, (list(r.its), g["its"])
    for sl in range(spec["nslices"]):
        lam, ref = np.asarray(r.lam[sl]), np.asarray(g["lam"][sl])
        assert np.max(np.abs(lam - ref)) <= 1e-10 * np.max(np.abs(ref))
        assert np.all(r.res[sl] < 1e-8) and np.all(r.res[sl] / np.abs(lam) <= 1e-8)
    exact = exact_eig_lap(*g["grid"], spec["a_lo"], spec["b_hi"])
    assert sum(r.nev) == len(exact)
