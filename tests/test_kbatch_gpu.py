"""GPU: k-point batches -- one launch over every (k-point, band) with a Bloch
phase set per k-point (gb_*_apply_k, gb_fd_precond_k, gb_lfc_add_k /
integrate_k) -- against one call per k-point with that k-point's phases
(the reference's loop over kpt_u, gpaw/eigensolvers/eigensolver.py:136-144)
and, for the stencil, against the oracle.  complex128 and complex64."""
import numpy as np
import pytest
import torch

from conftest import relerr
from oracle import fd

pytestmark = pytest.mark.gpu

K_C = np.array([[0.25, 0.25, 0.25], [0.25, -0.25, 0.25], [-0.25, 0.25, 0.25],
                [0.25, 0.25, -0.25]])


def _gd(N=(16, 20, 24), pbc=(1, 1, 1)):
    from gpaw_b200.grid_descriptor import GridDescriptor
    return GridDescriptor(N, 0.35 * np.array(N), pbc)


def _phases(gd):
    return np.array([gd.phase_factor_cd(k) for k in K_C])


def _data(gd, nb, dtype, seed=0):
    g = torch.Generator(device='cuda').manual_seed(seed)
    real = torch.float64 if dtype == torch.complex128 else torch.float32
    shape = (len(K_C) * nb,) + tuple(gd.n_c)
    return torch.complex(torch.randn(shape, generator=g, device='cuda', dtype=real),
                         torch.randn(shape, generator=g, device='cuda', dtype=real))


@pytest.mark.parametrize('dtype', [torch.complex128, torch.complex64])
@pytest.mark.parametrize('potential', [False, True])
def test_stencil_kbatch(dtype, potential):
    from gpaw_b200.fd_operators import Laplace
    gd = _gd()
    lap = Laplace(gd, -0.5, 3, complex)
    ph = _phases(gd)
    nb = 3
    x = _data(gd, nb, dtype)
    real = torch.float64 if dtype == torch.complex128 else torch.float32
    vt = torch.rand(tuple(gd.n_c), device='cuda', dtype=real) if potential else None
    y = torch.empty_like(x)
    if potential:
        lap.apply_potential(x, y, vt, ph)
    else:
        lap.apply(x, y, ph)
    for k in range(len(K_C)):
        sl = slice(k * nb, (k + 1) * nb)
        want = torch.empty_like(x[sl])
        if potential:
            lap.apply_potential(x[sl].contiguous(), want, vt, ph[k])
        else:
            lap.apply(x[sl].contiguous(), want, ph[k])
        assert torch.equal(y[sl], want), k
    if dtype == torch.complex128 and not potential:
        k = 2
        a = x[k * nb:(k + 1) * nb].cpu().numpy()
        ref = fd.fd_apply(lap.coef_p, lap.offset_pc, a, (1, 1, 1), ph[k])
        assert relerr(y[k * nb:(k + 1) * nb].cpu().numpy(), ref) < 1e-12


@pytest.mark.parametrize('dtype', [torch.complex128, torch.complex64])
def test_transformer_and_vcycle_kbatch(dtype):
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200.transformers import Transformer
    from gpaw_b200.preconditioner import Preconditioner
    gd = _gd((16, 16, 24))
    ph = _phases(gd)
    nb = 2
    x = _data(gd, nb, dtype, seed=3)

    class K:
        def __init__(self, p):
            self.phase_cd = p
    for nn in (1, 3):
        t = Transformer(gd, gd.coarsen(), nn, complex)
        y = t.apply(x, phases=ph)
        for k in range(len(K_C)):
            sl = slice(k * nb, (k + 1) * nb)
            assert torch.equal(y[sl], t.apply(x[sl].contiguous(), phases=ph[k])), (nn, k)
    P = Preconditioner(gd, Laplace(gd, -0.5, 3, complex), complex)
    d = P(x, K(ph)).clone()
    for k in range(len(K_C)):
        sl = slice(k * nb, (k + 1) * nb)
        assert torch.equal(d[sl], P(x[sl].contiguous(), K(ph[k]))), k


@pytest.mark.parametrize('dtype', [torch.complex128, torch.complex64])
def test_lfc_kbatch(dtype):
    from gpaw_b200.lfc import LFC
    from gpaw_b200.spline import Spline
    gd = _gd((16, 16, 20))

    class KD:
        ibzk_qc = K_C
        gamma = False
    r = np.linspace(0, 2.2, 41)
    f = np.exp(-(r / 0.9)**2)
    spl = [[Spline.from_data(0, 2.2, f), Spline.from_data(1, 2.2, f)],
           [Spline.from_data(2, 2.2, f)]]
    lfc = LFC(gd, spl, kd=KD(), cut=True, dtype=complex)
    lfc.set_positions(np.array([[0.05, 0.9, 0.5], [0.5, 0.3, 0.1]]))
    nb = 3
    nk = len(K_C)
    x = _data(gd, nb, dtype, seed=5)
    c = lfc.integrate(x, {}, q=range(nk))
    tol = 1e-13 if dtype == torch.complex128 else 1e-6
    for k in range(nk):
        sl = slice(k * nb, (k + 1) * nb)
        want = lfc.integrate(x[sl].contiguous(), {}, q=k)
        assert relerr(c[sl].cpu().numpy(), want.cpu().numpy()) < tol
    g = torch.Generator(device='cuda').manual_seed(9)
    real = torch.float64 if dtype == torch.complex128 else torch.float32
    cM = torch.complex(torch.randn((nk * nb, lfc.Mmax), generator=g, device='cuda', dtype=real),
                       torch.randn((nk * nb, lfc.Mmax), generator=g, device='cuda', dtype=real))
    a = torch.zeros_like(x)
    lfc.add_M(a, cM, q=range(nk))
    for k in range(nk):
        sl = slice(k * nb, (k + 1) * nb)
        want = torch.zeros_like(x[sl])
        lfc.add_M(want, cM[sl].contiguous(), q=k)
        assert torch.equal(a[sl], want), k
