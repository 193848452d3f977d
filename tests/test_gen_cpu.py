"""CPU tests of the generalized problem's host side (no GPU needed).

The least-squares B-solver's coefficients are host arithmetic in the
product as in the reference (SRC/lspolapprox.c:62-148): degree, centre,
half-width and every coefficient must equal the reference build's
(tests/golden/gen_bsolve.json, made by make_golden.py gen) exactly.
"""
import numpy as np
import pytest

import pevsl_b200 as pv
from conftest import golden


@pytest.mark.parametrize("case", range(4))
def test_lspol_coefficients_equal_reference(lib, case):
    g = golden("gen_bsolve.json")["lspol"][case]
    deg, mu, cc, dd = pv.lspol_coefs(g["kind"], g["max_deg"], g["tol"], g["lmin"], g["lmax"])
    assert deg == g["deg"]
    assert cc == g["cc"] and dd == g["dd"]
    np.testing.assert_array_equal(mu, np.array(g["mu"]))


def test_lspol_degree_cap_and_arguments(lib):
    # the tolerance is never met: the degree is max_deg - 1 (the last case
    # of the golden file), as the reference's loop without a break
    g = golden("gen_bsolve.json")["lspol"][3]
    assert g["deg"] == g["max_deg"] - 1
    with pytest.raises(pv.PevslError):
        pv.lspol_coefs(2, 10, 1e-6, 2.0, 6.0)
    with pytest.raises(pv.PevslError):
        pv.lspol_coefs(0, 10, 1e-6, 6.0, 2.0)
    with pytest.raises(pv.PevslError):
        pv.lspol_coefs(0, 0, 1e-6, 2.0, 6.0)


def test_lspol_approximates_the_function(lib):
    """The polynomial is what it claims: 1/x and 1/sqrt(x) on [2, 6]."""
    x = np.linspace(2.0, 6.0, 101)
    for kind, f in ((0, 1.0 / x), (1, 1.0 / np.sqrt(x))):
        deg, mu, cc, dd = pv.lspol_coefs(kind, 80, 1e-10, 2.0, 6.0)
        p = np.polynomial.chebyshev.chebval((x - cc) / dd, mu)
        assert np.max(np.abs(p - f) / f) < 1e-11, (kind, deg)


# ---------------------------------------------------------------- B-solvers
# numpy restatements of the reference's B-solvers, checked against the
# reference build's outputs (the fixture's x): the least-squares series
# (SRC/lspolapprox.c:245-288) and both Chebyshev iterations
# (EXTERNAL/ITERSOL/chebiter.c:121-198, 204-270).

def _B512():
    import scipy.sparse as sp
    from checkers import laplacian
    L = laplacian(512, 1, 1)
    return sp.csr_matrix((L.a, L.ja, L.ia), shape=(512, 512))


def _b():
    return np.cos(0.1 * np.arange(512, dtype=np.float64)) + 0.5


def lspol_apply(B, mu, cc, dd, b):
    """y = sum_k mu_k T_k((B - cc)/dd) b by the three-term recurrence"""
    vkm1, vk = None, b.copy()
    y = mu[0] * vk
    for k in range(1, len(mu)):
        t = (1.0 if k == 1 else 2.0) / dd
        w = (B @ vk - cc * vk) * t
        if vkm1 is not None:
            w = w - vkm1
        y = y + mu[k] * w
        vkm1, vk = vk, w
    return y


def chebiter1(B, lb, ub, deg, b):
    d, c = (ub + lb) * 0.5, (ub - lb) * 0.5
    if deg < 1:
        return np.zeros_like(b)
    alp = 2.0 / d
    p = b.copy()
    x = alp * p
    r = b - B @ x
    for _ in range(1, deg):
        t = c * alp * 0.5
        bet = t * t
        alp = 1.0 / (d - bet)
        p = bet * p + r
        x = x + alp * p
        r = b - B @ x
    return x


def chebiter2(B, lb, ub, deg, b):
    theta, delta = (ub + lb) * 0.5, (ub - lb) * 0.5
    sigma = theta / delta
    rho = 1.0 / sigma
    x = np.zeros_like(b)
    r = b.copy()
    d = r / theta
    for _ in range(deg):
        x = x + d
        r = r - B @ d
        rho1 = 1.0 / (2.0 * sigma - rho)
        d = rho1 * rho * d + 2.0 * rho1 / delta * r
        rho = rho1
    return x


@pytest.mark.parametrize("case", range(4))
def test_lspol_restatement_matches_reference_solve(case):
    g = golden("gen_bsolve.json")["lspol"][case]
    x = lspol_apply(_B512(), np.array(g["mu"]), g["cc"], g["dd"], _b())
    assert np.max(np.abs(x - g["x"])) <= 1e-13 * np.max(np.abs(g["x"]))


@pytest.mark.parametrize("case", range(5))
def test_chebiter_restatement_matches_reference_solve(case):
    g = golden("gen_bsolve.json")["chebiter"][case]
    f = chebiter1 if g["kind"] == 1 else chebiter2
    x = f(_B512(), g["lmin"], g["lmax"], g["deg"], _b())
    assert np.max(np.abs(x - np.array(g["x"]))) <= 1e-13 * max(np.max(np.abs(g["x"])), 1e-300)


def test_lspol_random_against_reference(lib, reference):
    """120 random least-squares requests (1/x and 1/sqrt(x), max_deg 5 to
    200, tolerances 1e-12 to 1e-2, intervals with ratios 1.5 to 400):
    degree, cc, dd and every coefficient bit for bit as the reference
    build's."""
    from checkers import laplacian
    B, b = laplacian(64, 1, 1), np.ones(64)
    rng = np.random.default_rng(2)
    for _ in range(120):
        kind, md = int(rng.integers(0, 2)), int(rng.integers(5, 200))
        tol = 10 ** rng.uniform(-12, -2)
        lo = rng.uniform(0.01, 3.0)
        hi = lo * rng.uniform(1.5, 400.0)
        d1, mu1, cc1, dd1, _ = reference.lspol(kind, md, tol, lo, hi, B, b)
        d2, mu2, cc2, dd2 = pv.lspol_coefs(kind, md, tol, lo, hi)
        assert (d1, cc1, dd1) == (d2, cc2, dd2)
        assert np.array_equal(mu1, np.asarray(mu2)[: d1 + 1])
