"""FP64 Poisson solver on the GPU (drop-in for gpaw.poisson.FastPoissonSolver).

Solves the finite-difference Poisson equation  L phi = -4 pi rho  exactly in
the eigenbasis of the FD Laplacian L (order 2 nn): plane waves on periodic
axes (FFT) and sine waves on zero-boundary axes (type-I DST), as
gpaw/poisson.py:842-1007 does.  The eigenvalues are
  lambda(k) = sum_p c_p (exp(i k.o_p) - 1)
for the stencil of Laplace(gd, -1/(4 pi), nn), with k = 2 pi m / N on
periodic axes and pi m / N on zero-boundary axes; the zero mode is dropped
(neutral periodic systems).  Everything stays on the device in FP64; the
transforms are cuFFT through torch.fft (a sine transform is the imaginary
part of an FFT of the odd extension).
"""
from __future__ import annotations

import numpy as np
import torch

from gpaw_b200.fd_operators import Laplace


def _dst1(x, dim):
    """Type-I DST along `dim` (unnormalised): X_k = sum_j x_j sin(pi jk/(n+1))."""
    n = x.shape[dim]
    zero = torch.zeros_like(x.narrow(dim, 0, 1))
    ext = torch.cat([zero, x, zero, -x.flip(dim)], dim=dim)
    Y = torch.fft.fft(ext, dim=dim)
    return -0.5 * Y.narrow(dim, 1, n).imag


class FastPoissonSolver:
    def __init__(self, nn=3, **kwargs):
        self.nn = nn
        self.gd = None

    def set_grid_descriptor(self, gd):
        self.gd = gd
        lap = Laplace(gd, -0.25 / np.pi, self.nn)
        if not gd.orthogonal:
            raise NotImplementedError('FastPoissonSolver needs an orthogonal cell')
        lam = np.zeros(tuple(gd.n_c))
        ks = []
        for c in range(3):
            m = np.arange(gd.n_c[c]) + gd.beg_c[c]
            k = 2 * np.pi * m / gd.N_c[c]
            if not gd.pbc_c[c]:
                k = k / 2
            ks.append(k)
        for coef, o in zip(lap.coef_p, lap.offset_pc):
            if not np.any(o):
                continue
            phase = (ks[0][:, None, None] * o[0] + ks[1][None, :, None] * o[1] +
                     ks[2][None, None, :] * o[2])
            lam += coef * (np.cos(phase) - 1.0)
        with np.errstate(divide='ignore'):
            inv = np.where(np.abs(lam) > 1e-10, 1.0 / lam, 0.0)
        self.inv_lambda = torch.from_numpy(inv).to(gd.device)
        self.description = lap.description

    def _forward(self, a):
        for c in range(3):
            dim = a.ndim - 3 + c
            if self.gd.pbc_c[c]:
                a = torch.fft.fft(a, dim=dim)
            else:
                a = _dst1(a.real, dim) + (1j * _dst1(a.imag, dim) if a.is_complex() else 0)
        return a

    def _backward(self, a):
        for c in range(3):
            dim = a.ndim - 3 + c
            if self.gd.pbc_c[c]:
                a = torch.fft.ifft(a, dim=dim)
            else:
                n = a.shape[dim]
                re = _dst1(a.real, dim) * (2.0 / (n + 1))
                im = _dst1(a.imag, dim) * (2.0 / (n + 1)) if a.is_complex() else 0
                a = re + 1j * im if a.is_complex() else re
        return a

    def solve_neutral(self, phi_g, rho_g, timer=None):
        """phi_g <- the solution of (-1/(4 pi)) L phi = rho_g, rho_g taken
        as given (gpaw/poisson.py:957-1002)."""
        if self.gd is None:
            raise RuntimeError('set_grid_descriptor first')
        assert rho_g.dtype == torch.float64, 'the Poisson solve stays FP64'
        a = rho_g.to(torch.complex128) if any(self.gd.pbc_c) else rho_g
        a = self._forward(a)
        a = a * self.inv_lambda
        a = self._backward(a)
        phi_g.copy_(a.real if a.is_complex() else a)
        return 1

    def _gaussian(self):
        """The normalised L = 0 Gaussian at the cell centre and its
        potential (gpaw/utilities/gauss.py:95-139 with a = 19; r^2 clamped
        at 1e-12, gpaw/utilities/tools.py:96-115)."""
        if getattr(self, '_gauss', None) is None:
            gd = self.gd
            icell_cv = np.linalg.inv(gd.cell_cv).T
            a = 4 * 19.0 * (icell_cv**2).sum(1).max()
            idx = np.indices(tuple(gd.n_c)).reshape(3, -1).T + gd.beg_c
            r_v = idx @ gd.h_cv - 0.5 * gd.cell_cv.sum(0)
            r2 = np.maximum((r_v**2).sum(1), 1e-12)
            r = torch.from_numpy(np.sqrt(r2))
            g = np.sqrt(4 * a**3) / np.pi * np.exp(-a * r2)
            phi = 2 * np.sqrt(np.pi) * torch.special.erf(np.sqrt(a) * r) / r
            self._gauss = (torch.from_numpy(g).reshape(tuple(gd.n_c)).to(gd.device),
                           phi.reshape(tuple(gd.n_c)).to(gd.device))
        return self._gauss

    def solve(self, phi_g, rho_g, charge=None, eps=None, maxcharge=1e-6,
              zero_initial_phi=False, timer=None):
        """phi_g <- the potential of rho_g (gpaw/poisson.py:178-279): a
        uniform background equal to the mean of rho_g is subtracted from
        neutral systems (|charge| <= maxcharge) and from periodic ones; a
        charged zero-boundary system is neutralised with a Gaussian whose
        analytic potential is added back; charged systems with mixed
        boundaries are not supported.  charge=None reads the charge from
        rho_g (one device-to-host read); a caller that knows its density
        is neutral passes charge=0 and the solve stays on the device."""
        if self.gd is None:
            raise RuntimeError('set_grid_descriptor first')
        background = rho_g.mean()
        if charge is None:
            charge = float(rho_g.sum()) * self.gd.dv
        if abs(charge) <= maxcharge or all(self.gd.pbc_c):
            return self.solve_neutral(phi_g, rho_g - background)
        if any(self.gd.pbc_c):
            raise NotImplementedError('charged system with mixed boundary conditions')
        g, phi_gauss = self._gaussian()
        q = float(rho_g.sum()) * self.gd.dv / np.sqrt(4 * np.pi)
        self.solve_neutral(phi_g, rho_g - q * g)
        phi_g.add_(q * phi_gauss)
        return 1
