"""CPU checks of the learned-DOS pieces that need no GPU: the MLP oracle's
backward pass against finite differences (FP64 form), its bfloat16 rounding,
and the parameter layout the library uses."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import mlp_oracle as mo  # noqa: E402


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -7, 1.0 + 3 * 2 ** -8, -2.5, 0.0, 3.1415926],
                 np.float32)
    r = mo.bf16(x)
    # 1 + 2^-8 is halfway between 1 and 1 + 2^-7: ties to even -> 1
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0 + 2 ** -7)
    # 1 + 3*2^-8 is halfway between 1 + 2^-7 and 1 + 2^-6: ties to even -> 1 + 2^-6
    assert r[3] == np.float32(1.0 + 2 ** -6)
    assert r[4] == -2.5 and r[5] == 0.0 and abs(r[6] - 3.140625) < 1e-7


def test_layout_padding():
    lay = mo.Layout(300, 256, 300, 4)
    assert lay.k == [304, 256, 256, 256] and lay.n == [256, 256, 256, 304]
    assert lay.np == 304 * 256 + 256 + 2 * (256 * 256 + 256) + 256 * 304 + 304
    p = lay.init(1)
    Ws, bs = lay.unpack(p)
    assert np.all(Ws[0][:, 300:] == 0) and np.all(Ws[3][300:, :] == 0)
    assert all(np.all(b == 0) for b in bs)


def test_oracle_gradient_matches_finite_differences():
    lay = mo.Layout(7, 12, 5, 3)
    rng = np.random.default_rng(3)
    p = lay.init(5).astype(np.float64)
    Ws, bs = lay.unpack(p)
    for b in bs:
        b[:] = rng.normal(0, 0.1, b.shape) * (np.arange(b.size) < b.size)
    X = rng.normal(size=(6, 7))
    T = rng.normal(size=(6, 5))
    loss, g = mo.loss_grad(lay, p, X, T, bf=False)
    # central differences on the real (unpadded) parameters
    idx = []
    for l in range(lay.layers):
        for n in range(lay.nr[l]):
            idx.append(lay.woff[l] + n * lay.k[l] + (n % lay.kr[l]))
            idx.append(lay.boff[l] + n)
    h = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += h
        lp, _ = mo.loss_grad(lay, q, X, T, bf=False)
        q[i] -= 2 * h
        lm, _ = mo.loss_grad(lay, q, X, T, bf=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])
