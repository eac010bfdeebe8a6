"""The FP64 FFT/DST Poisson solver (gpaw/poisson.py:842-1007).

CPU: the oracle restatement (oracle/poisson.py) is pinned by the equation
it solves, applied with GPAW's own C stencil (oracle/_ref `_gpaw.Operator`
with the reference's Laplace(-1/(4 pi), 3) coefficients, or the oracle's
stencil where that build is absent) to the solution extended oddly across
zero boundaries (the sine basis): L phi = -4 pi (rho - mean rho) to 1e-12,
on the H2 fine grid (63^3, zero boundaries), a periodic and a mixed grid;
and
the charged zero-boundary branch reproduces the analytic potential of a
Gaussian charge far from it.
GPU: gpaw_b200.poisson.FastPoissonSolver against the oracle at 1e-12 on the
H2 fine grid (N = 64, zero boundaries), the Si64 fine grid (112^3,
periodic) and a charged zero-boundary case."""
from math import pi

import numpy as np
import pytest

from conftest import relerr
from oracle import fd, poisson, ref

BOHR = 0.52917721


def _apply_laplace(phi, N_c, pbc_c, cell_cv):
    """(-1/(4 pi)) L phi with the solver's boundary treatment: periodic axes
    wrap; on a zero-boundary axis the sine basis extends phi oddly about
    the boundary points (phi(0) = phi(N) = 0, phi(-j) = -phi(j)), which for
    stencils longer than one point is not the zero padding of the stencil
    operators.  The odd extension (period 2N) is applied as a periodic array
    with GPAW's own C stencil (oracle/_ref) where that build is present."""
    h_cv = np.asarray(cell_cv) / np.asarray(N_c)[:, None]
    coef, off = fd.guc_laplace(h_cv, -0.25 / pi, 3)
    ext = np.asarray(phi, float)
    for c in range(3):
        if not pbc_c[c]:
            z = np.zeros_like(np.take(ext, [0], axis=c))
            ext = np.concatenate([z, ext, z, -np.flip(ext, axis=c)], axis=c)
    ext = np.ascontiguousarray(ext)
    if ref.available():
        op = ref.operator(coef, off, ext.shape, (1, 1, 1), True)
        out = np.zeros_like(ext)
        op.apply(ext, out)
    else:
        out = fd.fd_apply(coef, off, ext[None], (1, 1, 1))[0]
    sl = tuple(slice(0, n) if p else slice(1, n + 1)
               for p, n in zip(pbc_c, phi.shape))
    return out[sl]


def _rho(n_c, seed, neutral=True):
    rng = np.random.default_rng(seed)
    rho = rng.standard_normal(tuple(n_c))
    return rho - rho.mean() if neutral else rho


@pytest.mark.parametrize('N_c,pbc,cell', [
    ((64, 64, 64), (0, 0, 0), (6.0 / BOHR, 6.0 / BOHR, 6.74 / BOHR)),
    ((24, 28, 32), (1, 1, 1), (5.0, 5.5, 6.5)),
    ((20, 24, 16), (1, 0, 1), (4.0, 4.5, 3.5)),
])
def test_oracle_solves_the_fd_equation(N_c, pbc, cell):
    N_c = np.array(N_c)
    n_c = N_c - (1 - np.array(pbc))
    cell_cv = np.diag(cell)
    rho = _rho(n_c, 1, neutral=False) + 0.01
    phi = poisson.solve(rho, N_c, pbc, cell_cv, charge=0.0)
    lhs = _apply_laplace(phi, N_c, pbc, cell_cv)
    # (-1/(4 pi)) L phi = rho - background
    assert relerr(lhs, rho - rho.mean()) < 1e-12


def test_oracle_charged_zero_boundary_far_field():
    """A Gaussian of charge Q at the centre of a zero-boundary box: the
    solution is the Gaussian branch alone (the neutral remainder vanishes),
    i.e. Q / r away from the centre."""
    N_c = np.array([48, 48, 48])
    cell_cv = np.diag([12.0, 12.0, 12.0])
    n_c = N_c - 1
    g, phi_g = poisson.gaussian(N_c, n_c, (1, 1, 1), cell_cv)
    rho = 0.7 * g / np.sqrt(4 * pi)
    phi = poisson.solve(rho, N_c, (0, 0, 0), cell_cv)
    # the remainder is the quadrature error of the Gaussian's charge
    assert relerr(phi, 0.7 * phi_g / np.sqrt(4 * pi)) < 1e-8


def _gpu_case(N_c, pbc, cell_cv, rho):
    import torch
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.poisson import FastPoissonSolver
    gd = GridDescriptor(N_c, cell_cv, pbc)
    ps = FastPoissonSolver(nn=3)
    ps.set_grid_descriptor(gd)
    phi = torch.zeros(tuple(gd.n_c), dtype=torch.float64, device='cuda')
    ps.solve(phi, torch.from_numpy(rho).cuda())
    return phi.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize('N_c,pbc,cell,neutral', [
    # H2 configuration fine grid: 6.0 x 6.0 x 6.74 A, N = 32 coarse -> 64 fine
    ((64, 64, 64), (0, 0, 0), (6.0 / BOHR, 6.0 / BOHR, 6.74 / BOHR), True),
    # Si64 fine grid: 2 x 56 = 112 points per axis of the 10.86 A cell
    ((112, 112, 112), (1, 1, 1), (10.86 / BOHR,) * 3, True),
    ((20, 24, 16), (1, 0, 1), (4.0, 4.5, 3.5), True),
    ((48, 40, 44), (0, 0, 0), (9.0, 8.0, 8.5), False),
])
def test_gpu_poisson_matches_oracle(N_c, pbc, cell, neutral):
    N_c = np.array(N_c)
    n_c = N_c - (1 - np.array(pbc))
    cell_cv = np.diag(cell)
    rho = _rho(n_c, 2, neutral) + (0.0 if neutral else 0.05)
    got = _gpu_case(N_c, pbc, cell_cv, rho)
    want = poisson.solve(rho, N_c, pbc, cell_cv)
    assert relerr(got, want) < 1e-12
