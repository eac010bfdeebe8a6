"""CPU: the learned-preconditioner oracle's manual backward agrees with
central finite differences (FP64), and the transfer-operator adjoint
identities it relies on hold (Interp^T = 8 Restrict for nn=1)."""
import numpy as np
import pytest

from oracle import fd
from oracle import learned as ol

SHAPES = {'w0': (1, 1, 27), 'wa': (16, 1, 27), 'wb': (16, 16, 27), 'wc': (1, 16, 27),
          'wp': (1, 1, 27)}


@pytest.mark.parametrize('pbc', [(1, 1, 1), (0, 0, 0)])
def test_transfer_adjoint(pbc):
    g0 = fd.Grid((16, 12, 8), (3.0, 2.5, 2.0), pbc)
    g1 = g0.coarsen()
    R = fd.Transformer(g0, g1, 1)
    I = fd.Transformer(g1, g0, 1)
    rng = np.random.default_rng(0)
    a = rng.standard_normal(tuple(g0.n_c))
    b = rng.standard_normal(tuple(g1.n_c))
    assert abs((a * I.apply(b)).sum() - 8.0 * (R.apply(a) * b).sum()) < 1e-10 * abs((a * I.apply(b)).sum())


@pytest.mark.parametrize('pbc', [(1, 1, 1), (0, 1, 0)])
def test_oracle_gradient_vs_finite_differences(pbc):
    rng = np.random.default_rng(1)
    params = {k: rng.standard_normal(s) * 0.2 for k, s in SHAPES.items()}
    g0 = fd.Grid((8, 8, 8), (2.0, 2.0, 2.0), pbc)
    net = ol.Net(g0, params)
    R = rng.standard_normal((2,) + tuple(g0.n_c))
    T = rng.standard_normal(R.shape)
    out = net.forward(R)
    loss, g = ol.loss_and_grad(out, T, g0)
    grads = net.backward(g)
    eps = 1e-6
    for k in SHAPES:
        for idx in [(0, 0, 13), (0, 0, 0), tuple(np.array(SHAPES[k]) - 1)]:
            p = {kk: v.copy() for kk, v in params.items()}
            p[k][idx] += eps
            lp, _ = ol.loss_and_grad(ol.Net(g0, p).forward(R), T, g0)
            p[k][idx] -= 2 * eps
            lm, _ = ol.loss_and_grad(ol.Net(g0, p).forward(R), T, g0)
            fdg = (lp - lm) / (2 * eps)
            assert abs(fdg - grads[k][idx]) < 1e-6 * max(1.0, abs(fdg)), (k, idx)
