"""CPU oracle of the learned-DOS MLP (test infrastructure only).

The reference has no learned part; this is the checker for the library's
BF16 training kernels (pevsl_b200/csrc/gpu_mlp.cu): the same network, the
same padded parameter layout, and the same rounding points --

  forward   a_0 = bf16(x);  z_l = a_l W_l^T + b_l (W_l in bf16, sums in
            FP32 or FP64);  a_{l+1} = bf16(gelu(z_l)) between layers; the
            last z is the output;
  loss      mean of (y - t)^2 over the batch and the real outputs;
  backward  dz_L = 2 (y - t) / (B nout);  dW_l = bf16(dz_l)^T a_l;
            db_l = column sums of dz_l;  dz_{l-1} = (bf16(dz_l) W_l) *
            gelu'(z_{l-1});
            gelu(z) = z Phi(z), gelu'(z) = Phi(z) + z phi(z).

With bf16=False every rounding point is skipped and the arithmetic is FP64:
that form is checked against finite differences in tests/test_learned_cpu.py.
"""
import math

import numpy as np

_erf = np.vectorize(math.erf)


def bf16(x):
    """Round FP32 values to bfloat16 (round to nearest even), returned as FP32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(x.shape)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    cdf = 0.5 * (1.0 + _erf(z / math.sqrt(2.0)))
    pdf = np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)
    return cdf + z * pdf


def pad16(x):
    return (x + 15) // 16 * 16


class Layout:
    """Padded parameter layout: per layer l, W_l (N_l x K_l row-major) then
    b_l (N_l), K/N padded to multiples of 16."""

    def __init__(self, nin, width, nout, layers):
        self.nin, self.width, self.nout, self.layers = nin, width, nout, layers
        self.k, self.n, self.woff, self.boff, self.kr, self.nr = [], [], [], [], [], []
        off = 0
        for l in range(layers):
            kr = nin if l == 0 else width
            nr = nout if l + 1 == layers else width
            k, n = pad16(kr), pad16(nr)
            self.k.append(k)
            self.n.append(n)
            self.kr.append(kr)
            self.nr.append(nr)
            self.woff.append(off)
            off += k * n
            self.boff.append(off)
            off += n
        self.np = off

    def unpack(self, p):
        Ws, bs = [], []
        for l in range(self.layers):
            Ws.append(p[self.woff[l]:self.woff[l] + self.k[l] * self.n[l]].reshape(self.n[l], self.k[l]))
            bs.append(p[self.boff[l]:self.boff[l] + self.n[l]])
        return Ws, bs

    def init(self, seed):
        """Uniform(-1/sqrt(K), 1/sqrt(K)) weights, zero biases, zero padding."""
        rng = np.random.default_rng(seed)
        p = np.zeros(self.np, np.float32)
        Ws, _ = self.unpack(p)
        for l in range(self.layers):
            lim = 1.0 / math.sqrt(self.kr[l])
            Ws[l][:self.nr[l], :self.kr[l]] = rng.uniform(-lim, lim, (self.nr[l], self.kr[l]))
        return p


def forward(lay, p, X, bf=True):
    """Returns (y [B][nout], zs, acts) for X [B][nin]."""
    dt = np.float32 if bf else np.float64
    rnd = bf16 if bf else (lambda v: np.asarray(v, np.float64))
    Ws, bs = lay.unpack(np.asarray(p, dt))
    B = X.shape[0]
    a = np.zeros((B, lay.k[0]), dt)
    a[:, :lay.nin] = X
    a = rnd(a)
    acts, zs = [a], []
    for l in range(lay.layers):
        W = rnd(Ws[l])
        z = (a.astype(np.float64) @ W.astype(np.float64).T + bs[l]).astype(dt)
        zs.append(z)
        if l + 1 < lay.layers:
            a = rnd(gelu(z.astype(np.float64)).astype(dt))
            acts.append(a)
    return zs[-1][:, :lay.nout], zs, acts


def loss_grad(lay, p, X, T, bf=True):
    """(loss, gradient in the parameter layout)."""
    dt = np.float32 if bf else np.float64
    rnd = bf16 if bf else (lambda v: np.asarray(v, np.float64))
    y, zs, acts = forward(lay, p, X, bf)
    B = X.shape[0]
    L = lay.layers
    d = (y.astype(np.float64) - T)
    loss = float(np.sum(d * d) / (B * lay.nout))
    dz = np.zeros((B, lay.n[L - 1]), dt)
    dz[:, :lay.nout] = (2.0 / (B * lay.nout)) * d
    g = np.zeros(lay.np, np.float64)
    Ws, _ = lay.unpack(np.asarray(p, dt))
    for l in range(L - 1, -1, -1):
        dzr = rnd(dz).astype(np.float64)
        gW = dzr.T @ acts[l].astype(np.float64)
        g[lay.woff[l]:lay.woff[l] + lay.k[l] * lay.n[l]] = gW.ravel()
        g[lay.boff[l]:lay.boff[l] + lay.n[l]] = np.sum(dz.astype(np.float64), axis=0)
        if l == 0:
            break
        da = dzr @ rnd(Ws[l]).astype(np.float64)
        dz = (da * gelu_grad(zs[l - 1].astype(np.float64))).astype(dt)
    return loss, g
