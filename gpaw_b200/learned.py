"""Learned multigrid-like preconditioner (north star pattern 4).

A small linear 3-level 3-D convolution network stands in for the multigrid
V-cycle M(R) of gpaw/preconditioner.py inside RMM-DIIS:

    x  = R / s                         s = RMS(R) per band
    r1 = Restrict(x)                   level 1   (our transformer kernel, nn=1)
    a1 = conv_a(r1)        1 -> 16     level 1
    r2 = Restrict(a1)                  level 2   (16 channels per band)
    a2 = conv_b(r2)       16 -> 16     level 2
    u1 = Interp(a2) + a1               level 1
    b1 = conv_c(u1)       16 -> 1      level 1
    y  = Interp(b1) + conv_0(x)  1->1  level 0
    out = s * y

Convolutions are 3x3x3 with BF16 weights and FP32 accumulation
(gb_conv3d_forward); training uses the hand-written backward kernels:
conv backward-data = conv with flipped, transposed weights;
conv backward-weight = gb_conv3d_backward_weight; and the adjoints of the
nn=1 transfer operators, Interp^T = 8 Restrict and Restrict^T = Interp / 8
(exact for the linear-interpolation / full-weighting pair).  The network is
linear and homogeneous of degree one in R, like M.  The loss is the mean
over bands of ||out - M(R)||^2 / ||M(R)||^2 on (residual, multigrid
correction) pairs that RMM-DIIS produces.

At run time the multigrid preconditioner is both the fallback and the judge:
every call compares the network with M on a few bands; if the relative
deviation exceeds `tolerance`, that call returns M(R) instead.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from gpaw_b200 import _native as nat
from gpaw_b200.transformers import Transformer

SHAPES = {'w0': (1, 1, 27), 'wa': (16, 1, 27), 'wb': (16, 16, 27), 'wc': (1, 16, 27)}


def flip_transpose(w):
    """w[co][ci][k] -> w'[ci][co][26 - k] (weights of the adjoint conv)."""
    return w.transpose(0, 1).flip(-1).contiguous()


class ConvNet:
    def __init__(self, gd0, seed=0, device=None):
        self.gd0 = gd0
        self.gd1 = gd0.coarsen()
        self.gd2 = self.gd1.coarsen()
        self.device = device or gd0.device
        self.pbc = (ctypes.c_int * 3)(*[int(p) for p in gd0.pbc_c])
        self.r01 = Transformer(self.gd0, self.gd1, 1)
        self.r12 = Transformer(self.gd1, self.gd2, 1)
        self.i21 = Transformer(self.gd2, self.gd1, 1)
        self.i10 = Transformer(self.gd1, self.gd0, 1)
        g = torch.Generator().manual_seed(seed)
        self.params = {}
        for k, shp in SHAPES.items():
            fan_in = shp[1] * 27
            self.params[k] = (torch.randn(shp, generator=g, dtype=torch.float64) /
                              np.sqrt(fan_in)).to(torch.float32).to(self.device)
        # start close to "identity-ish" smoothing: level-0 centre weight
        self.params['w0'][0, 0, 13] = 0.5

    # -------------------------------------------------------------- kernels
    def _n(self, gd):
        return nat.i64(gd.n_c)

    def conv(self, x, w32, gd, out=None, accumulate=False):
        """x: (nb, cin, n...) FP32 -> (nb, cout, n...)."""
        cout, cin, _ = w32.shape
        nb = x.shape[0]
        wb = w32.to(torch.bfloat16).contiguous()
        if out is None:
            out = torch.empty((nb, cout) + tuple(gd.n_c), dtype=torch.float32, device=x.device)
        nat.check(nat.lib().gb_conv3d_forward(
            nat.ptr(x), nat.ptr(wb), nat.ptr(out), nb, cin, cout, self._n(gd),
            (ctypes.c_int * 3)(*[int(p) for p in gd.pbc_c]), int(accumulate),
            nat.stream_of(x)), 'gb_conv3d_forward')
        return out

    def conv_bwd_w(self, x, dy, w32, gd):
        cout, cin, _ = w32.shape
        dw = torch.zeros_like(w32)
        nat.check(nat.lib().gb_conv3d_backward_weight(
            nat.ptr(x), nat.ptr(dy), nat.ptr(dw), x.shape[0], cin, cout, self._n(gd),
            (ctypes.c_int * 3)(*[int(p) for p in gd.pbc_c]), nat.stream_of(x)),
            'gb_conv3d_backward_weight')
        return dw

    @staticmethod
    def _flat(t):
        return t.reshape((-1,) + tuple(t.shape[-3:]))

    def transfer(self, t, T):
        lead = tuple(t.shape[:-3])
        out = T.apply(self._flat(t))
        return out.reshape(lead + tuple(out.shape[-3:]))

    # -------------------------------------------------------------- network
    def forward(self, R, keep=False):
        """R: (nb, n0, n1, n2) any float dtype -> (nb, n0, n1, n2) FP32."""
        p = self.params
        nb = R.shape[0]
        x = R.to(torch.float32)
        s = x.reshape(nb, -1).pow(2).mean(1).sqrt().clamp_min(1e-30)
        x = (x / s.reshape(-1, 1, 1, 1))[:, None].contiguous()        # (nb, 1, n0)
        r1 = self.transfer(x, self.r01)                                  # (nb, 1, n1)
        a1 = self.conv(r1, p['wa'], self.gd1)                            # (nb, 16, n1)
        r2 = self.transfer(a1, self.r12)                                 # (nb, 16, n2)
        a2 = self.conv(r2, p['wb'], self.gd2)                            # (nb, 16, n2)
        u1 = self.transfer(a2, self.i21) + a1                            # (nb, 16, n1)
        b1 = self.conv(u1, p['wc'], self.gd1)                            # (nb, 1, n1)
        y = self.transfer(b1, self.i10)                                  # (nb, 1, n0)
        self.conv(x, p['w0'], self.gd0, out=y, accumulate=True)
        out = y[:, 0] * s.reshape(-1, 1, 1, 1)
        if keep:
            self._cache = dict(x=x, s=s, r1=r1, r2=r2, u1=u1)
        return out

    def backward(self, g_out):
        """Gradients of the loss w.r.t. the four weight tensors, given
        dL/d(out) (nb, n0, n1, n2) FP32 (uses the cache of forward(keep=True))."""
        c = self._cache
        p = self.params
        nb = g_out.shape[0]
        gy = (g_out * c['s'].reshape(-1, 1, 1, 1))[:, None].contiguous()   # (nb, 1, n0)
        grads = {'w0': self.conv_bwd_w(c['x'], gy, p['w0'], self.gd0)}
        gb1 = 8.0 * self.transfer(gy, self.r01)                             # Interp^T
        grads['wc'] = self.conv_bwd_w(c['u1'], gb1, p['wc'], self.gd1)
        gu1 = self.conv(gb1, flip_transpose(p['wc']), self.gd1)            # (nb, 16, n1)
        ga2 = 8.0 * self.transfer(gu1, self.r12)                            # Interp^T
        grads['wb'] = self.conv_bwd_w(c['r2'], ga2, p['wb'], self.gd2)
        gr2 = self.conv(ga2, flip_transpose(p['wb']), self.gd2)            # (nb, 16, n2)
        ga1 = gu1 + self.transfer(gr2, self.i21) / 8.0                      # Restrict^T
        grads['wa'] = self.conv_bwd_w(c['r1'], ga1, p['wa'], self.gd1)
        return grads

    @staticmethod
    def loss_and_grad(out, target):
        """mean_b ||out_b - t_b||^2 / ||t_b||^2 and its gradient."""
        nb = out.shape[0]
        t = target.to(torch.float32)
        d = out - t
        den = t.reshape(nb, -1).pow(2).sum(1).clamp_min(1e-30)
        loss = (d.reshape(nb, -1).pow(2).sum(1) / den).mean()
        g = 2.0 * d / (den.reshape(-1, 1, 1, 1) * nb)
        return float(loss), g

    # -------------------------------------------------------------- training
    def train(self, pairs, steps=300, lr=3e-3, batch=16, seed=0, log_every=50):
        """Adam on (R, M(R)) pairs (lists of (nb, n...) tensors)."""
        m = {k: torch.zeros_like(v) for k, v in self.params.items()}
        v2 = {k: torch.zeros_like(v) for k, v in self.params.items()}
        b1, b2, eps = 0.9, 0.999, 1e-8
        rng = np.random.default_rng(seed)
        R_all = torch.cat([r for r, _ in pairs])
        M_all = torch.cat([t for _, t in pairs])
        hist = []
        for it in range(1, steps + 1):
            idx = torch.as_tensor(rng.choice(len(R_all), size=min(batch, len(R_all)),
                                             replace=False), device=R_all.device)
            R = R_all[idx].contiguous()
            T = M_all[idx].contiguous()
            out = self.forward(R, keep=True)
            loss, g = self.loss_and_grad(out, T)
            grads = self.backward(g)
            for k in self.params:
                m[k] = b1 * m[k] + (1 - b1) * grads[k]
                v2[k] = b2 * v2[k] + (1 - b2) * grads[k]**2
                mh = m[k] / (1 - b1**it)
                vh = v2[k] / (1 - b2**it)
                self.params[k] -= lr * mh / (vh.sqrt() + eps)
            hist.append(loss)
            if log_every and it % log_every == 0:
                print(f'  train step {it}: loss {np.mean(hist[-log_every:]):.4e}', flush=True)
        return hist

    def relative_error(self, R, target):
        out = self.forward(R)
        nb = R.shape[0]
        t = target.to(torch.float32)
        return ((out - t).reshape(nb, -1).norm(dim=1) / t.reshape(nb, -1).norm(dim=1)).cpu().numpy()


class LearnedPreconditioner:
    """Drop-in for Preconditioner.__call__(R, kpt) with the multigrid as
    fallback and judge."""

    def __init__(self, net: ConvNet, multigrid, tolerance=0.5, nprobe=2):
        self.net = net
        self.multigrid = multigrid
        self.tolerance = tolerance
        self.nprobe = nprobe
        self.calls = 0
        self.fallbacks = 0

    def __call__(self, R, kpt=None, ekin=None, out=None):
        if R.ndim == 3:
            return self(R[None], kpt)[0]
        self.calls += 1
        y = self.net.forward(R).to(R.dtype)
        k = min(self.nprobe, R.shape[0])
        probe = self.multigrid(R[:k].contiguous(), kpt)
        dev = ((y[:k] - probe).reshape(k, -1).norm(dim=1) /
               probe.reshape(k, -1).norm(dim=1).clamp_min(1e-30)).max().item()
        if not np.isfinite(dev) or dev > self.tolerance:
            self.fallbacks += 1
            y = self.multigrid(R, kpt)
        if out is not None:
            out.copy_(y)
            return out
        return y
