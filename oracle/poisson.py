"""ORACLE (test infrastructure): the FFT/DST Poisson solver in numpy.

Restates gpaw/poisson.py:842-1007 (FastPoissonSolver: eigenvalues of the
order-2nn FD Laplacian in the plane-wave / sine basis, set_grid_descriptor
at :850-955, solve_neutral at :957-1002 with the transforms of :769-835:
numpy FFT on periodic axes, scipy type-I DST times 1/2 forward and
1/(n + 1) backward on zero-boundary axes) and the charge handling of
BasePoissonSolver.solve (gpaw/poisson.py:178-279): a uniform background is
subtracted from neutral and from periodic systems; a charged zero-boundary
system is neutralised with the normalised Gaussian of
gpaw/utilities/gauss.py:95-139 (exponent a = 4 * 19 * max_c |icell_c|^2,
centred in the cell, r^2 clamped at 1e-12 as in
gpaw/utilities/tools.py:96-115) whose analytic potential is added back.
"""
from __future__ import annotations

from math import erf, pi, sqrt

import numpy as np
from scipy.fft import dst

from oracle.fd import guc_laplace


def eigenvalues(N_c, n_c, beg_c, pbc_c, h_cv, nn):
    """lambda(k) = sum_p c_p (exp(i k . o_p) - 1) of Laplace(-1/(4 pi), nn),
    k = 2 pi m / N (periodic) or pi m / N (zero boundary), m = beg + index."""
    coef_p, offset_pc = guc_laplace(h_cv, -0.25 / pi, nn)
    ph = []
    for c in range(3):
        m = np.arange(n_c[c]) + beg_c[c]
        k = 2 * pi * m / N_c[c]
        if not pbc_c[c]:
            k = k / 2
        ph.append(np.exp(1j * k))
    lam = np.zeros(tuple(n_c), complex)
    for coef, o in zip(coef_p, offset_pc):
        if not np.any(o):
            continue
        t = (ph[0][:, None, None]**o[0] * ph[1][None, :, None]**o[1] *
             ph[2][None, None, :]**o[2])
        lam += coef * (t - 1.0)
    assert np.linalg.norm(lam.imag) < 1e-10
    lam = lam.real
    with np.errstate(divide='ignore'):
        return np.where(np.abs(lam) > 1e-10, 1.0 / lam, 0.0)


def solve_neutral(rho, inv_lambda, pbc_c):
    a = np.asarray(rho, float)
    for c in range(3):
        a = np.fft.fft(a, axis=c) if pbc_c[c] else 0.5 * dst(a, type=1, axis=c)
    a = a * inv_lambda
    for c in range(3):
        if pbc_c[c]:
            a = np.fft.ifft(a, axis=c)
        else:
            a = dst(a, type=1, axis=c) / (a.shape[c] + 1)
    return np.real(a)


def gaussian(N_c, n_c, beg_c, cell_cv):
    """(g, phi_g): the L = 0 Gaussian sqrt(4 a^3)/pi exp(-a r^2) (integral
    sqrt(4 pi)) at the centre of a zero-boundary cell and its potential
    2 sqrt(pi) erf(sqrt(a) r) / r."""
    cell_cv = np.asarray(cell_cv, float)
    icell_cv = np.linalg.inv(cell_cv).T
    a = 4 * 19.0 * (icell_cv**2).sum(1).max()
    h_cv = cell_cv / np.asarray(N_c)[:, None]
    idx = np.indices(tuple(n_c)).reshape(3, -1).T + np.asarray(beg_c)
    r_v = idx @ h_cv - 0.5 * cell_cv.sum(0)
    r2 = np.maximum((r_v**2).sum(1), 1e-12)
    r = np.sqrt(r2)
    g = sqrt(4 * a**3) / pi * np.exp(-a * r2)
    phi = 2 * sqrt(pi) * np.array([erf(sqrt(a) * x) for x in r]) / r
    return g.reshape(tuple(n_c)), phi.reshape(tuple(n_c))


def solve(rho, N_c, pbc_c, cell_cv, nn=3, charge=None, maxcharge=1e-6):
    """phi with (-1/(4 pi)) L phi = rho, L the order-2nn FD Laplacian,
    following BasePoissonSolver.solve's branches."""
    N_c = np.asarray(N_c)
    pbc_c = np.asarray(pbc_c, bool)
    beg_c = np.where(pbc_c, 0, 1)
    n_c = N_c - beg_c
    cell_cv = np.asarray(cell_cv, float)
    h_cv = cell_cv / N_c[:, None]
    dv = abs(np.linalg.det(cell_cv)) / N_c.prod()
    inv = eigenvalues(N_c, n_c, beg_c, pbc_c, h_cv, nn)
    actual = rho.sum() * dv
    background = actual / dv / n_c.prod()
    if charge is None:
        charge = actual
    if abs(charge) <= maxcharge or pbc_c.all():
        return solve_neutral(rho - background, inv, pbc_c)
    assert not pbc_c.any(), 'charged systems with mixed boundaries'
    g, phi_g = gaussian(N_c, n_c, beg_c, cell_cv)
    q = actual / sqrt(4 * pi)
    return solve_neutral(rho - q * g, inv, pbc_c) + q * phi_g
