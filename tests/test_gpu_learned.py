"""The learned-DOS network's GPU kernels against the CPU oracle
(oracle/mlp_oracle.py, which mirrors their BF16 rounding points).

Tolerances: the loss to 1e-4 relative; gradients and outputs per layer to
1e-2 in relative 2-norm (FP32 sums in a different order can move an
activation across a BF16 rounding boundary, which changes it by 2^-8
relative).
"""
import os
import sys

import numpy as np
import pytest

import pevsl_b200 as pv

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import mlp_oracle as mo  # noqa: E402

pytestmark = pytest.mark.gpu


def relnorm(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def _net(nin, width, nout, layers, seed):
    lay = mo.Layout(nin, width, nout, layers)
    p = lay.init(seed)
    rng = np.random.default_rng(seed + 1)
    Ws, bs = lay.unpack(p)
    for l in range(layers):
        bs[l][:lay.nr[l]] = rng.normal(0, 0.05, lay.nr[l])
    net = pv.Mlp(nin, width, nout, layers)
    assert net.np == lay.np
    net.set_params(p)
    return lay, p, net


@pytest.mark.parametrize("dims", [(37, 48, 29, 3, 21), (300, 256, 300, 4, 64), (5, 16, 3, 1, 7)])
def test_mlp_gradients_and_outputs_match_oracle(gpu, dims):
    nin, width, nout, layers, B = dims
    lay, p, net = _net(nin, width, nout, layers, 11)
    rng = np.random.default_rng(2)
    X = rng.normal(size=(B, nin)).astype(np.float32)
    T = rng.normal(size=(B, nout)).astype(np.float32)
    Xm, Tm, Ym = pv.ManagedArray((B, nin)).set(X), pv.ManagedArray((B, nout)).set(T), \
        pv.ManagedArray((B, nout))
    net.forward(Xm, Ym, B)
    y_o, _, _ = mo.forward(lay, p, X)
    assert relnorm(Ym.get(), y_o) <= 1e-2
    loss, g = net.gradients(Xm, Tm, B)
    loss_o, g_o = mo.loss_grad(lay, p, X, T)
    assert abs(loss - loss_o) <= 1e-4 * loss_o
    for l in range(layers):
        w = slice(lay.woff[l], lay.woff[l] + lay.k[l] * lay.n[l])
        b = slice(lay.boff[l], lay.boff[l] + lay.n[l])
        assert relnorm(g[w], g_o[w]) <= 1e-2, ("W", l)
        assert relnorm(g[b], g_o[b]) <= 1e-2, ("b", l)
    # padding carries no gradient
    Ws, _ = lay.unpack(g)
    assert np.all(Ws[0][:, nin:] == 0)
    net.close()


def test_mlp_training_fits_a_linear_map(gpu):
    """Adam steps on the GPU bring the loss of a learnable map down by 20x."""
    nin, nout, B = 24, 16, 256
    lay, p, net = _net(nin, 64, nout, 3, 5)
    rng = np.random.default_rng(9)
    X = rng.normal(size=(B, nin)).astype(np.float32)
    M = rng.normal(size=(nin, nout)).astype(np.float32) / np.sqrt(nin)
    T = (X @ M).astype(np.float32)
    Xm, Tm = pv.ManagedArray((B, nin)).set(X), pv.ManagedArray((B, nout)).set(T)
    l0 = net.train_step(Xm, Tm, B, 3e-3, want_loss=True)
    for _ in range(400):
        net.train_step(Xm, Tm, B, 3e-3)
    l1 = net.train_step(Xm, Tm, B, 3e-3, want_loss=True)
    assert l1 < l0 / 20, (l0, l1)
    # the weights changed only on the real entries
    q = net.get_params()
    Ws, _ = lay.unpack(q)
    assert np.all(Ws[0][:, nin:] == 0) and np.all(Ws[2][nout:, :] == 0)
    net.close()


def test_learned_dos_denoises_few_vector_moments(gpu):
    """Trained on moment pairs of 200 matrices of the families (4 draws of
    8-vector moments against 256-vector moments, all from the library's
    KPM), the network brings held-out 8-vector moments closer to the
    256-vector moments than they were, and its slices go through the
    plain-KPM check."""
    from pevsl_b200 import learned as ld
    specs = ld.training_specs(200, seed=1, sizes="small")
    X, T = ld.moment_pairs(specs, seed=1, draws=4)
    model = ld.LearnedDos(seed=0)
    hist = model.fit(X, T, epochs=60, batch=64, lr=1e-3, seed=0)
    assert hist[-1] < hist[0]
    held = ld.training_specs(12, seed=999, sizes="small")
    Xh, Th = ld.moment_pairs(held, seed=77)
    P = model.predict(Xh)
    err_plain = np.linalg.norm(Xh[:, 1:] - Th[:, 1:], axis=1)
    err_learned = np.linalg.norm(P[:, 1:] - Th[:, 1:], axis=1)
    assert np.mean(err_learned) < np.mean(err_plain), (err_learned, err_plain)
    assert np.mean(err_learned < err_plain) >= 0.75, (err_learned, err_plain)
    # the slicing path with its plain-KPM check runs end to end
    kind, s, size = held[0]
    n, ia, ja, a = ld.family_matrix(kind, s, size)
    M = pv.Matrix.from_csr(n, ia, ja, a)
    with pv.Instance(M) as ev:
        lmin, lmax = ld.spectrum_bounds(ev)
        sli, info = ld.learned_slices(ev, [lmin + 0.2 * (lmax - lmin), lmin + 0.4 * (lmax - lmin),
                                           lmin, lmax], 4, model, seed=5)
        assert info["used"] in ("learned", "kpm") and len(sli) == 5 and np.all(np.diff(sli) > 0)
    M.free()
    model.close()
