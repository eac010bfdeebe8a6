"""ORACLE (test infrastructure): FP64 numpy restatement of the learned
preconditioner network of gpaw_b200/learned.py (forward and manual
backward), built from oracle/fd.py's restriction / interpolation (which are
pinned to the reference's transformers) and a direct 3x3x3 convolution.
Used to check the GPU forward/backward kernels; its own gradient is checked
against central finite differences in tests/test_learned_oracle.py."""
from __future__ import annotations

import numpy as np

from oracle import fd

OFFS = [(k // 9 - 1, (k // 3) % 3 - 1, k % 3 - 1) for k in range(27)]


def shift(x, o, pbc):
    """x[..., p + o] with zero padding or periodic wrap per axis."""
    out = x
    for c in range(3):
        if o[c] == 0:
            continue
        ax = x.ndim - 3 + c
        out = np.roll(out, -o[c], axis=ax)
        if not pbc[c]:
            idx = [slice(None)] * x.ndim
            idx[ax] = slice(-o[c], None) if o[c] > 0 else slice(0, -o[c])
            out[tuple(idx)] = 0.0
    return out


def conv(x, w, pbc):
    """x (nb, cin, n...), w (cout, cin, 27) -> (nb, cout, n...)."""
    nb, cin = x.shape[:2]
    cout = w.shape[0]
    y = np.zeros((nb, cout, int(np.prod(x.shape[2:]))))
    for k, o in enumerate(OFFS):
        xs = shift(x, o, pbc).reshape(nb, cin, -1)
        y += np.einsum('oi,bip->bop', w[:, :, k], xs)
    return y.reshape((nb, cout) + x.shape[2:])


def conv_bwd_w(x, dy, pbc):
    nb, cout, cin = dy.shape[0], dy.shape[1], x.shape[1]
    dw = np.zeros((cout, cin, 27))
    d = dy.reshape(nb, cout, -1)
    for k, o in enumerate(OFFS):
        dw[:, :, k] = np.einsum('bop,bip->oi', d, shift(x, o, pbc).reshape(nb, cin, -1))
    return dw


def conv_bwd_x(dy, w, pbc):
    """adjoint of conv: flipped, transposed weights."""
    wt = np.transpose(w, (1, 0, 2))[:, :, ::-1]
    return conv(dy, wt, pbc)


class Net:
    def __init__(self, grid0: fd.Grid, params):
        self.g0 = grid0
        self.g1 = grid0.coarsen()
        self.g2 = self.g1.coarsen()
        self.pbc = tuple(bool(p) for p in grid0.pbc_c)
        self.p = {k: np.asarray(v, float) for k, v in params.items()}
        self.T01 = fd.Transformer(self.g0, self.g1, 1)
        self.T12 = fd.Transformer(self.g1, self.g2, 1)
        self.T21 = fd.Transformer(self.g2, self.g1, 1)
        self.T10 = fd.Transformer(self.g1, self.g0, 1)

    def forward(self, R):
        p, pbc = self.p, self.pbc
        nb = R.shape[0]
        s = np.sqrt((R.reshape(nb, -1)**2).mean(1))
        x = (R / s[:, None, None, None])[:, None]
        r1 = self.T01.apply(x)
        a1 = conv(r1, p['wa'], pbc)
        r2 = self.T12.apply(a1)
        a2 = conv(r2, p['wb'], pbc)
        u1 = self.T21.apply(a2) + a1
        b1 = conv(u1, p['wc'], pbc)
        z = self.T10.apply(b1)
        y = conv(z, p['wp'], pbc) + conv(x, p['w0'], pbc)
        self.c = dict(x=x, s=s, r1=r1, r2=r2, u1=u1, z=z)
        return y[:, 0] * s[:, None, None, None]

    def backward(self, g):
        c, p, pbc = self.c, self.p, self.pbc
        gy = (g * c['s'][:, None, None, None])[:, None]
        grads = {'w0': conv_bwd_w(c['x'], gy, pbc), 'wp': conv_bwd_w(c['z'], gy, pbc)}
        gz = conv_bwd_x(gy, p['wp'], pbc)
        gb1 = 8.0 * self.T01.apply(gz)
        grads['wc'] = conv_bwd_w(c['u1'], gb1, pbc)
        gu1 = conv_bwd_x(gb1, p['wc'], pbc)
        ga2 = 8.0 * self.T12.apply(gu1)
        grads['wb'] = conv_bwd_w(c['r2'], ga2, pbc)
        gr2 = conv_bwd_x(ga2, p['wb'], pbc)
        ga1 = gu1 + self.T21.apply(gr2) / 8.0
        grads['wa'] = conv_bwd_w(c['r1'], ga1, pbc)
        return grads


def weight(x, grid):
    """A x = (K + 1) x, K = -1/2 nabla^2 with the 7-point (nn=1) stencil of
    gpaw/fd_operators.py Laplace (the energy-norm weight of the loss)."""
    coefs, offs = fd.guc_laplace(grid.h_cv, -0.5, 1)
    return fd.fd_apply(coefs, offs, x, grid.pbc_c) + x


def loss_and_grad(out, t, grid):
    """mean_b ||A(out_b - t_b)||^2 / ||A t_b||^2 and its gradient
    2 A^T A (out - t) / (den nb); A is symmetric."""
    nb = out.shape[0]
    Ad = weight(out - t, grid)
    den = (weight(t, grid).reshape(nb, -1)**2).sum(1)
    loss = ((Ad.reshape(nb, -1)**2).sum(1) / den).mean()
    return loss, 2.0 * weight(Ad, grid) / (den[:, None, None, None] * nb)
