"""The ELL filter kernels built for a fixed row width (5, the 2D five-point
stencil; 7, the 3D seven-point stencil) against the build for any width.

Both builds add every row's products in entry order with the same
operations, so a lockstep run (two-slice groups, k_cheb_il2_e) and a
one-slice run (one-vector degree, k_cheb_il_e<1>) must give the same bits
whichever build runs, and the exact eigenvalue counts.  The forms are chosen
once per process (PEVSL_B200_ELL, PEVSL_B200_ELL_W), so each run is a child
process with the ELL forms forced on (no set-up timing picks another form).
"""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

CHILD = r"""
import json, sys
sys.path.insert(0, sys.argv[1])
import numpy as np
import pevsl_b200 as pv
from checkers import exact_eig_lap, laplacian
grid = tuple(json.loads(sys.argv[2]))
a, b, ns = json.loads(sys.argv[3])
L = laplacian(*grid)
ev = exact_eig_lap(*grid, 0.0, 100.0)
lmin, lmax = ev[0] - 1e-6, ev[-1] + 1e-6
edges = np.linspace(a, b, ns + 1)
intvs = [[edges[i], edges[i + 1], lmin, lmax] for i in range(ns)]
fl = [pv.findpol(iv)[1] for iv in intvs]
M = pv.Matrix.from_csr(L.n, L.ia, L.ja, L.a)
v = np.cos(np.arange(M.n) * 0.37)
out = {"n": M.n, "batch": [], "one": None, "exact": []}
with pv.Instance(M) as e:
    r, batch = pv.cheblannr_batch(e, intvs, [200] * ns, 1e-8, v, fl)
assert r == 0, r
for s in batch:
    out["batch"].append({"nev": int(s["nev"]), "its": int(s["its"]),
                         "lam": [float(x).hex() for x in s["lam"]],
                         "res": [float(x).hex() for x in s["res"]]})
with pv.Instance(M) as e:
    r, (one,) = pv.cheblannr_batch(e, [intvs[0]], [200], 1e-8, v, [fl[0]])
assert r == 0, r
out["one"] = {"nev": int(one["nev"]), "its": int(one["its"]),
              "lam": [float(x).hex() for x in one["lam"]],
              "res": [float(x).hex() for x in one["res"]]}
for iv in intvs:
    out["exact"].append([float(x) for x in exact_eig_lap(*grid, iv[0], iv[1])])
M.free()
print("RESULT " + json.dumps(out))
"""


def _run(grid, spec, fixed_width):
    env = dict(os.environ, PEVSL_B200_ELL="1", PEVSL_B200_ELL_W=str(fixed_width))
    p = subprocess.run([sys.executable, "-c", CHILD, HERE, json.dumps(grid), json.dumps(spec)],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    line = [x for x in p.stdout.splitlines() if x.startswith("RESULT ")]
    assert line, p.stdout[-2000:]
    return json.loads(line[-1][len("RESULT "):])


@pytest.mark.parametrize("grid,spec", [
    ((299, 301, 1), [2.300, 2.304, 2]),   # 89 999 rows, width 5
    ((41, 41, 41), [0.30, 0.33, 2]),      # 68 921 rows, width 7
])
def test_fixed_width_ell_kernels_match_any_width(gpu, grid, spec):
    fixed = _run(grid, spec, 1)
    anyw = _run(grid, spec, 0)
    assert fixed["n"] >= 65536
    # the same bits from both builds, batched and alone
    assert fixed["batch"] == anyw["batch"]
    assert fixed["one"] == anyw["one"]
    # a slice in lockstep gets the bits of solving it alone
    assert fixed["one"] == fixed["batch"][0]
    # and the exact counts and eigenvalues
    for s, ex in zip(fixed["batch"], fixed["exact"]):
        assert s["nev"] == len(ex) and len(ex) > 0
        lam = [float.fromhex(x) for x in s["lam"]]
        assert max(abs(x - y) for x, y in zip(lam, ex)) <= 1e-10 * max(abs(y) for y in ex)
        assert all(float.fromhex(x) < 1e-8 for x in s["res"])
