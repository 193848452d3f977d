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
