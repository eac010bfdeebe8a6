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
    z  = Interp(b1)                    level 0
    y  = conv_p(z) + conv_0(x)   1->1  level 0 (post- and pre-smoothing)
    out = s * y

Convolutions are 3x3x3 with BF16 weights and FP32 accumulation
(gb_conv3d_forward); training uses the hand-written backward kernels:
conv backward-data = conv with flipped, transposed weights;
conv backward-weight = gb_conv3d_backward_weight; and the adjoints of the
nn=1 transfer operators, Interp^T = 8 Restrict and Restrict^T = Interp / 8
(exact for the linear-interpolation / full-weighting pair).  The network is
linear and homogeneous of degree one in R, like M.  The loss is the mean
over bands of ||A(out - M(R)/s)||^2 / ||A M(R)/s||^2 on (residual, multigrid
correction) pairs that RMM-DIIS produces, in the energy norm A = K + 1
(K = -1/2 nabla^2): an error e in a correction reappears as (K - eps) e in
the next residual, so plain L2 would let high-frequency errors through that
RMM-DIIS's fixed trial step amplifies.  s is the multigrid step of the grid
(0.66666666 / diagonal of the kinetic stencil), which makes one set of
weights serve grids of different spacing.

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

SHAPES = {'w0': (1, 1, 27), 'wa': (16, 1, 27), 'wb': (16, 16, 27), 'wc': (1, 16, 27),
          'wp': (1, 1, 27)}


def flip_transpose(w):
    """w[co][ci][k] -> w'[ci][co][26 - k] (weights of the adjoint conv)."""
    return w.transpose(0, 1).flip(-1).contiguous()


class ConvNet:
    def __init__(self, gd0, seed=0, device=None, params=None):
        self.gd0 = gd0
        self.gd1 = gd0.coarsen()
        self.gd2 = self.gd1.coarsen()
        self.device = device or gd0.device
        self.pbc = (ctypes.c_int * 3)(*[int(p) for p in gd0.pbc_c])
        self.r01 = Transformer(self.gd0, self.gd1, 1)
        self.r12 = Transformer(self.gd1, self.gd2, 1)
        self.i21 = Transformer(self.gd2, self.gd1, 1)
        self.i10 = Transformer(self.gd1, self.gd0, 1)
        # energy-norm weight A = K + 1 (K = -1/2 nabla^2, 7-point, FP32):
        # an error e in the correction costs ~ (K - eps) e in the next
        # residual, so training and the judge measure errors through A
        from gpaw_b200.fd_operators import Laplace
        self.kin = Laplace(gd0, -0.5, 1, float)
        if params is not None:
            # the same weights on another grid (the network is translation
            # invariant; only the transfer operators depend on the grid)
            self.params = params
            return
        g = torch.Generator().manual_seed(seed)
        self.params = {}
        for k, shp in SHAPES.items():
            fan_in = shp[1] * 27
            w = torch.randn(shp, generator=g, dtype=torch.float64) / np.sqrt(fan_in)
            if k == 'w0':
                # start close to an identity-like smoother at level 0
                w[0, 0, 13] = 0.5
            if k == 'wp':
                # the post-interpolation conv starts as the identity
                w.zero_()
                w[0, 0, 13] = 1.0
            self.params[k] = w.to(torch.float32).to(self.device)

    @staticmethod
    def _stencil27(op):
        """27-entry kernel of a radius-1 FD operator (entries of larger
        offsets are dropped); index k <-> offset (k//9-1, (k//3)%3-1, k%3-1)."""
        w = torch.zeros(27, dtype=torch.float64)
        for c, o in zip(op.coef_p, np.asarray(op.offset_pc).reshape(-1, 3)):
            if np.abs(o).max() <= 1:
                w[(o[0] + 1) * 9 + (o[1] + 1) * 3 + (o[2] + 1)] += c
        return w

    def init_from_multigrid(self, mg):
        """Set the weights to the V-cycle of `mg` (gpaw/preconditioner.py,
        c/fd_preconditioner.c), in the network's normalised form T = M(R)/s:

          a1: ch0 = -(4s K1 - 1) r1,  ch1 = -r1            (r1 = Restrict(x))
          a2: ch2 = (32s - 256 s^2 K2) r2                  (r2 = Restrict(a1 ch0))
          b1 = (8s - 16 s^2 K1) u1[ch1] + (4s K1 - 1) u1[ch2]
          y  = (1/s - K0') Interp(b1) - x

        K1, K2 are the 7-point coarse Laplacians of the V-cycle; K0' is the
        radius-1 part of the fine kinetic stencil (the V-cycle's own K0 reaches
        +-3 points, which a 3x3x3 kernel cannot hold -- training corrects it).
        """
        s = float(mg.step)
        d = torch.zeros(27, dtype=torch.float64)
        d[13] = 1.0
        K1 = self._stencil27(mg.kin1)
        K2 = self._stencil27(mg.kin2)
        K0 = self._stencil27(mg.kin0)
        w = {k: torch.zeros(shp, dtype=torch.float64) for k, shp in SHAPES.items()}
        w['wa'][0, 0] = -(4 * s * K1 - d)
        w['wa'][1, 0] = -d
        w['wb'][2, 0] = 32 * s * d - 256 * s * s * K2
        w['wc'][0, 1] = 8 * s * d - 16 * s * s * K1
        w['wc'][0, 2] = 4 * s * K1 - d
        w['wp'][0, 0] = d / s - K0
        w['w0'][0, 0] = -d
        for k in SHAPES:
            self.params[k].copy_(w[k].to(self.params[k]))
        return self

    def on_grid(self, gd):
        """This network (shared weights) on another grid descriptor."""
        return ConvNet(gd, device=self.device, params=self.params)

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

    def conv_pair(self, x0, x1, w0_32, w1_32, gd):
        """conv(x0, w0) + conv(x1, w1) for single-channel FP32 inputs, one
        launch (gb_conv3d_forward_pair)."""
        wb = torch.cat([w0_32, w1_32], dim=1).to(torch.bfloat16).contiguous()   # (1, 2, 27)
        out = torch.empty_like(x0)
        nat.check(nat.lib().gb_conv3d_forward_pair(
            nat.ptr(x0), nat.ptr(x1), nat.ptr(wb), nat.ptr(out), x0.shape[0], self._n(gd),
            (ctypes.c_int * 3)(*[int(p) for p in gd.pbc_c]), nat.stream_of(x0)),
            'gb_conv3d_forward_pair')
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
    def forward(self, R, keep=False, scale=1.0):
        """R: (nb, n0, n1, n2) any float dtype -> scale * net(R), (nb, n0, n1, n2)
        FP32.  The network is linear and homogeneous, so inference runs on R
        as it is (FP32 accumulation does not care about the overall scale);
        training (keep=True) normalises every band to unit RMS first, which
        keeps the per-band loss weights independent of the residual size.
        `scale` is folded into the last convolution's weights."""
        p = self.params
        nb = R.shape[0]
        x = R.to(torch.float32)
        if keep:
            s = x.reshape(nb, -1).pow(2).mean(1).sqrt().clamp_min(1e-30)
            x = x / s.reshape(-1, 1, 1, 1)
        x = x.reshape((nb, 1) + tuple(x.shape[1:])).contiguous()          # (nb, 1, n0)
        r1 = self.transfer(x, self.r01)                                  # (nb, 1, n1)
        a1 = self.conv(r1, p['wa'], self.gd1)                            # (nb, 16, n1)
        r2 = self.transfer(a1, self.r12)                                 # (nb, 16, n2)
        a2 = self.conv(r2, p['wb'], self.gd2)                            # (nb, 16, n2)
        u1 = torch.empty_like(a1)                                        # Interp(a2) + a1
        self.i21.apply_axpy(self._flat(a2), self._flat(u1), 1.0, self._flat(a1), 1.0)
        b1 = self.conv(u1, p['wc'], self.gd1)                            # (nb, 1, n1)
        z = self.transfer(b1, self.i10)                                  # (nb, 1, n0)
        y = self.conv_pair(z, x, p['wp'] * scale, p['w0'] * scale, self.gd0)
        if keep:
            self._cache = dict(x=x, s=s, r1=r1, r2=r2, u1=u1, z=z)
            return y[:, 0] * s.reshape(-1, 1, 1, 1)
        return y[:, 0]

    def backward(self, g_out):
        """Gradients of the loss w.r.t. the four weight tensors, given
        dL/d(out) (nb, n0, n1, n2) FP32 (uses the cache of forward(keep=True))."""
        c = self._cache
        p = self.params
        nb = g_out.shape[0]
        gy = (g_out * c['s'].reshape(-1, 1, 1, 1))[:, None].contiguous()   # (nb, 1, n0)
        grads = {'w0': self.conv_bwd_w(c['x'], gy, p['w0'], self.gd0),
                 'wp': self.conv_bwd_w(c['z'], gy, p['wp'], self.gd0)}
        gz = self.conv(gy, flip_transpose(p['wp']), self.gd0)               # (nb, 1, n0)
        gb1 = 8.0 * self.transfer(gz, self.r01)                             # Interp^T
        grads['wc'] = self.conv_bwd_w(c['u1'], gb1, p['wc'], self.gd1)
        gu1 = self.conv(gb1, flip_transpose(p['wc']), self.gd1)            # (nb, 16, n1)
        ga2 = 8.0 * self.transfer(gu1, self.r12)                            # Interp^T
        grads['wb'] = self.conv_bwd_w(c['r2'], ga2, p['wb'], self.gd2)
        gr2 = self.conv(ga2, flip_transpose(p['wb']), self.gd2)            # (nb, 16, n2)
        ga1 = gu1 + self.transfer(gr2, self.i21) / 8.0                      # Restrict^T
        grads['wa'] = self.conv_bwd_w(c['r1'], ga1, p['wa'], self.gd1)
        return grads

    def weight(self, x):
        """A x = (K + 1) x for a batch (nb, n0, n1, n2) of FP32 grids."""
        y = torch.empty_like(x)
        self.kin.apply(x.contiguous(), y)
        return y.add_(x)

    def loss_and_grad(self, out, target):
        """mean_b ||A(out_b - t_b)||^2 / ||A t_b||^2 and its gradient
        2 A^T A (out - t) / (den nb) (A is symmetric)."""
        nb = out.shape[0]
        t = target.to(torch.float32)
        d = out - t
        Ad = self.weight(d)
        den = self.weight(t).reshape(nb, -1).pow(2).sum(1).clamp_min(1e-30)
        loss = (Ad.reshape(nb, -1).pow(2).sum(1) / den).mean()
        g = 2.0 * self.weight(Ad) / (den.reshape(-1, 1, 1, 1) * nb)
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
        """||net(R) - target|| / ||target|| per band (host array)."""
        return self.relative_error_t(R, target).cpu().numpy()

    def relative_error_from(self, out, target):
        """||A(out - target)|| / ||A target|| per band (device tensor)."""
        nb = out.shape[0]
        t = target.to(torch.float32)
        return (self.weight(out - t).reshape(nb, -1).norm(dim=1) /
                self.weight(t).reshape(nb, -1).norm(dim=1).clamp_min(1e-30))

    def relative_error_t(self, R, target):
        out = self.forward(R)
        nb = R.shape[0]
        t = target.to(torch.float32)
        return (self.weight(out - t).reshape(nb, -1).norm(dim=1) /
                self.weight(t).reshape(nb, -1).norm(dim=1).clamp_min(1e-30))


def train_multi(sets, steps=400, lr=3e-3, batch=16, seed=0, log_every=0):
    """Adam over several grids at once: `sets` is a list of (net, R, T)
    with nets sharing one parameter dict (ConvNet.on_grid) and (R, T) the
    (residual, scaled multigrid correction) pairs recorded on that net's
    grid.  Each step takes a batch from one set, in proportion to its size.
    Returns the loss history."""
    params = sets[0][0].params
    assert all(net.params is params for net, _, _ in sets)
    m = {k: torch.zeros_like(v) for k, v in params.items()}
    v2 = {k: torch.zeros_like(v) for k, v in params.items()}
    b1, b2, eps = 0.9, 0.999, 1e-8
    rng = np.random.default_rng(seed)
    sizes = np.array([len(R) for _, R, _ in sets], float)
    prob = sizes / sizes.sum()
    hist = []
    for it in range(1, steps + 1):
        lr_t = lr * 0.5 * (1.0 + np.cos(np.pi * (it - 1) / steps))   # cosine decay
        net, R_all, T_all = sets[rng.choice(len(sets), p=prob)]
        idx = torch.as_tensor(rng.choice(len(R_all), size=min(batch, len(R_all)),
                                         replace=False), device=R_all.device)
        out = net.forward(R_all[idx].contiguous(), keep=True)
        loss, g = net.loss_and_grad(out, T_all[idx].contiguous())
        grads = net.backward(g)
        for k in params:
            m[k] = b1 * m[k] + (1 - b1) * grads[k]
            v2[k] = b2 * v2[k] + (1 - b2) * grads[k]**2
            params[k] -= lr_t * (m[k] / (1 - b1**it)) / ((v2[k] / (1 - b2**it)).sqrt() + eps)
        hist.append(loss)
        if log_every and it % log_every == 0:
            print(f'  train step {it}: loss {np.mean(hist[-log_every:]):.4e}', flush=True)
    return hist


class PairRecorder:
    """Wraps the multigrid preconditioner during ordinary iterations and
    keeps (residual, correction / step) pairs of a few random bands per call:
    the training data that the method itself generates."""

    def __init__(self, multigrid, per_call=8, max_pairs=512, seed=0):
        self.multigrid = multigrid
        self.per_call = per_call
        self.max_pairs = max_pairs
        self.rng = np.random.default_rng(seed)
        self.R = []
        self.T = []
        self.count = 0

    def __call__(self, R, kpt=None, ekin=None, out=None):
        y = self.multigrid(R, kpt, out=out)
        if self.count < self.max_pairs and R.ndim == 4:
            k = min(self.per_call, R.shape[0], self.max_pairs - self.count)
            idx = torch.as_tensor(self.rng.choice(R.shape[0], size=k, replace=False),
                                  device=R.device)
            self.R.append(R[idx].to(torch.float32))
            self.T.append((y[idx] / self.multigrid.step).to(torch.float32))
            self.count += k
        return y

    def pairs(self):
        return torch.cat(self.R), torch.cat(self.T)


class FoldedNet:
    """Inference form of a ConvNet on a periodic grid of even sizes (all
    three levels): the linear layers folded into composite stencils
    (gb_learned_fold_stride / gb_learned_fold_fine), with the 16-channel
    level-2 convolution kept as it is.  Per forward:

        r1 = Restrict(x)                      (transformer kernel)
        r2 = Q *2 r1                          (stride-2 5^3 stencil, 1 -> 16)
        a2 = conv_b(r2)                       (16 -> 16, unchanged)
        b1 = C1 * r1 + G (x) a2               (5^3 stencil + parity stencil)
        y  = W0 * x  + H (x) b1               (3^3 stencil + parity stencil)

    instead of four transfers and five convolutions over 16-channel level-1
    tensors.  The composite weights come from applying the unfolded network
    (its own kernels and BF16 weights) to delta inputs on a small periodic
    grid, so both forms compute the same linear map up to FP32 rounding;
    every probe also checks that no weight falls outside the windows the
    kernels read."""

    PROBE_N = 32

    @staticmethod
    def applies(gd):
        """Periodic, every size divisible by 4 and the level-1 rows at least
        10 points long (the stencils' wrap-around arithmetic)."""
        n = np.asarray(gd.n_c)
        return bool(np.all(gd.pbc_c) and np.all(n % 4 == 0) and n[2] >= 20)

    def __init__(self, net: ConvNet, scale=1.0):
        gd = net.gd0
        if not self.applies(gd):
            raise ValueError('FoldedNet: needs a periodic grid, sizes divisible by 4, >= 20')
        self.net = net
        self.scale = float(scale)
        from gpaw_b200.grid_descriptor import GridDescriptor
        N = self.PROBE_N
        gdp = GridDescriptor((N, N, N), np.eye(3) * N * 0.4, True, device=net.device)
        pn = ConvNet(gdp, device=net.device, params=net.params)
        self._extract(pn)

    @staticmethod
    def _window(t, centre, lo, hi, what):
        """t (..., M, M, M) response around `centre` (3 ints): returns the
        block of offsets lo..hi per axis and checks that the rest is zero."""
        c0, c1, c2 = centre
        blk = t[..., c0 + lo:c0 + hi + 1, c1 + lo:c1 + hi + 1, c2 + lo:c2 + hi + 1].clone()
        rest = t.clone()
        rest[..., c0 + lo:c0 + hi + 1, c1 + lo:c1 + hi + 1, c2 + lo:c2 + hi + 1] = 0
        scale = blk.abs().max().clamp_min(1e-30)
        if rest.abs().max() > 1e-6 * scale:
            raise RuntimeError(f'FoldedNet: {what} reaches beyond its stencil window')
        return blk

    def _extract(self, pn):
        p = pn.params
        dev = pn.device
        N1 = pn.gd1.n_c[0]          # level-1 probe size
        c1 = N1 // 2
        # C1 = conv_c o conv_a on level 1: b1[p] = sum_d C1[d] r1[p + d]
        r1 = torch.zeros((1, 1, N1, N1, N1), dtype=torch.float32, device=dev)
        r1[0, 0, c1, c1, c1] = 1.0
        a1 = pn.conv(r1, p['wa'], pn.gd1)
        b1 = pn.conv(a1, p['wc'], pn.gd1)[0, 0]
        blk = self._window(b1, (c1, c1, c1), -2, 2, 'conv_c o conv_a')
        self.C1 = blk.flip(0, 1, 2).contiguous().reshape(-1)           # C1[d] = b1[c - d]
        # Q = Restrict o conv_a: r2[c][I] = sum_d Q[c][d] r1[2I + d]; one probe
        # per parity class of the delta position
        N2 = pn.gd2.n_c[0]
        Q = torch.zeros((16, 5, 5, 5), dtype=torch.float64, device=dev)
        seen = torch.zeros((5, 5, 5), dtype=torch.bool, device=dev)
        par = [(a, b, c) for a in (0, 1) for b in (0, 1) for c in (0, 1)]
        r1 = torch.zeros((8, 1, N1, N1, N1), dtype=torch.float32, device=dev)
        for k, (a, b, c) in enumerate(par):
            r1[k, 0, c1 + a, c1 + b, c1 + c] = 1.0
        r2 = pn.transfer(pn.conv(r1, p['wa'], pn.gd1), pn.r12)          # (8, 16, N2^3)
        I = torch.arange(N2, device=dev)
        for k, (a, b, c) in enumerate(par):
            q = torch.tensor([c1 + a, c1 + b, c1 + c], device=dev)
            d = [((q[ax] - 2 * I + N1 // 2) % N1) - N1 // 2 for ax in range(3)]   # wrapped offsets
            inside = [(dd.abs() <= 2) for dd in d]
            resp = r2[k].double()
            mask = inside[0][:, None, None] & inside[1][None, :, None] & inside[2][None, None, :]
            if resp[:, ~mask].abs().max() > 1e-6 * resp.abs().max().clamp_min(1e-30):
                raise RuntimeError('FoldedNet: restrict o conv_a reaches beyond its stencil window')
            ix = [torch.nonzero(m).flatten() for m in inside]
            sub = resp[:, ix[0]][:, :, ix[1]][:, :, :, ix[2]]
            dx, dy, dz = [(d[ax][ix[ax]] + 2) for ax in range(3)]
            Q[:, dx[:, None, None], dy[None, :, None], dz[None, None, :]] = sub
            seen[dx[:, None, None], dy[None, :, None], dz[None, None, :]] = True
        if not bool(seen.all()):
            raise RuntimeError('FoldedNet: the restriction probes did not cover every offset')
        self.Q = Q.reshape(16, 125).T.contiguous().to(torch.float32)   # [125][16]
        # G = conv_c o Interp(2 -> 1): b1[p] = sum_c G[c][p - 2J] a2[c][J]
        J0 = N2 // 2
        a2 = torch.zeros((16, 16, N2, N2, N2), dtype=torch.float32, device=dev)
        for c in range(16):
            a2[c, c, J0, J0, J0] = 1.0
        b1 = pn.conv(pn.transfer(a2, pn.i21), p['wc'], pn.gd1)[:, 0]     # (16, N1^3)
        blk = self._window(b1, (2 * J0,) * 3, -2, 3, 'conv_c o interpolation')
        self.G = blk.contiguous().reshape(16, 216)
        # H = conv_p o Interp(1 -> 0), the step folded in; W0 = step * w0
        # (BF16-rounded like the unfolded level-0 convolution)
        N0 = pn.gd0.n_c[0]
        b1 = torch.zeros((1, 1, N1, N1, N1), dtype=torch.float32, device=dev)
        b1[0, 0, c1, c1, c1] = 1.0
        y = pn.conv(pn.transfer(b1, pn.i10), p['wp'] * self.scale, pn.gd0)[0, 0]
        blk = self._window(y, (2 * c1,) * 3, -2, 3, 'conv_p o interpolation')
        self.H = blk.contiguous().reshape(216)
        self.W0 = (p['w0'] * self.scale).to(torch.bfloat16).to(torch.float32).reshape(27).contiguous()

    def forward(self, R):
        """scale * net(R) for R (nb, n0, n1, n2): FP32 out."""
        net = self.net
        x = R.to(torch.float32).contiguous()
        nb = x.shape[0]
        st = nat.stream_of(x)
        r1 = net.r01.apply(x)
        n1 = nat.i64(net.gd1.n_c)
        r2 = torch.empty((nb, 16) + tuple(net.gd2.n_c), dtype=torch.float32, device=x.device)
        nat.check(nat.lib().gb_learned_fold_stride(nat.ptr(r1), nat.ptr(self.Q), nat.ptr(r2), nb,
                                                   n1, st), 'gb_learned_fold_stride')
        a2 = net.conv(r2, net.params['wb'], net.gd2)
        b1 = torch.empty_like(r1)
        nat.check(nat.lib().gb_learned_fold_fine(nat.ptr(r1), nat.ptr(self.C1), 2, nat.ptr(a2),
                                                 nat.ptr(self.G), 16, nat.ptr(b1), nb, n1, st),
                  'gb_learned_fold_fine')
        y = torch.empty_like(x)
        nat.check(nat.lib().gb_learned_fold_fine(nat.ptr(x), nat.ptr(self.W0), 1, nat.ptr(b1),
                                                 nat.ptr(self.H), 1, nat.ptr(y), nb,
                                                 nat.i64(net.gd0.n_c), st), 'gb_learned_fold_fine')
        return y


class LearnedPreconditioner:
    """Drop-in for Preconditioner.__call__(R, kpt): the network's correction
    (scaled by the multigrid step of this grid), with the multigrid as judge
    and fallback.

    Every `probe_every`-th call (default 3: once per RMM-DIIS pass) also
    applies the multigrid to `nprobe` bands and compares; a relative
    deviation above `tolerance` (or a non-finite output) sets the device
    flag `failed`.  Nothing is read back during the call, so it runs
    inside a captured SCF step; the SCF driver reads the flag once per
    iteration with its other scalars and, when it is set, continues with the
    multigrid alone (`fallback`)."""

    def __init__(self, net: ConvNet, multigrid, tolerance=0.5, nprobe=2, probe_every=3):
        self.net = net
        self.multigrid = multigrid
        self.fallback = multigrid
        self.step = multigrid.step
        self.tolerance = tolerance
        self.nprobe = nprobe
        # judge one call in `probe_every` (3 = once per RMM-DIIS pass with its
        # default niter = 3 preconditioner calls); a captured SCF step holds
        # the same calls on every replay, so the cadence is fixed
        self.probe_every = max(1, int(probe_every))
        self._calls = 0
        self.failed = torch.zeros((), dtype=torch.bool, device=net.device)
        self.deviation = torch.zeros((), dtype=torch.float64, device=net.device)
        # periodic grids (sizes divisible by 4): the folded inference form
        self.folded = None
        if FoldedNet.applies(net.gd0):
            self.folded = FoldedNet(net, scale=self.step)
        # one call on seeded data: first launches and the stencil autotuner's
        # timing (the judge's nprobe-band shapes) happen here, not inside
        # the SCF that uses the preconditioner
        g = torch.Generator(device=net.device).manual_seed(0)
        R = torch.randn((self.nprobe + 1,) + tuple(net.gd0.n_c), generator=g,
                        device=net.device, dtype=torch.float32)
        self(R)
        self.failed.zero_()
        self.deviation.zero_()
        self._calls = 0

    def __call__(self, R, kpt=None, ekin=None, out=None):
        if R.ndim == 3:
            o = None if out is None else out[None]
            return self(R[None], kpt, out=o)[0]
        y = (self.folded.forward(R) if self.folded is not None
             else self.net.forward(R, scale=self.step))
        probe_now = self._calls % self.probe_every == 0
        self._calls += 1
        if probe_now:
            k = min(self.nprobe, R.shape[0])
            probe = self.multigrid(R[:k].contiguous(), kpt).to(torch.float32)
            dev = self.net.relative_error_from(y[:k], probe).max().to(torch.float64)
            self.deviation.copy_(torch.maximum(self.deviation, dev))
            bad = ~torch.isfinite(dev) | (dev > self.tolerance)
            self.failed.logical_or_(bad)
        y = y.to(R.dtype)
        if out is not None:
            out.copy_(y)
            return out
        return y


def collect_pairs(calc, iterations=6, per_call=8, max_pairs=512, seed=0):
    """Run `iterations` ordinary SCF iterations of `calc` (eagerly, with its
    multigrid preconditioner) and return the recorded (residual, correction /
    step) pairs as two FP32 tensors (bands, n0, n1, n2)."""
    mg = calc.preconditioner
    rec = PairRecorder(mg, per_call=per_call, max_pairs=max_pairs, seed=seed)
    calc.use_preconditioner(rec)
    try:
        calc.update_hamiltonian()
        for _ in range(iterations):
            calc.iteration()
    finally:
        calc.use_preconditioner(mg)
    return rec.pairs()
