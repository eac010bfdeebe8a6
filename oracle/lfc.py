"""ORACLE (test infrastructure): localized functions as dense arrays.

Phi_M(G) on the whole grid, built from:
  * the cubic spline of c/bmgs/spline.c:11-75 (restated below),
  * the real solid harmonics r^l Y_lm of c/bmgs/spherical_harmonics.h:5-48
    (l <= 2, same m order),
  * every periodic image of every atom whose sphere (r < rcut) reaches the
    grid (what gd.get_boxes + spline_to_grid cover, c/lfc.c:887-977).
add / integrate / derivative are then plain matrix products:
  add:        a_x += sum_M c_xM conj(phase) Phi_M          (c/lfc.c:818-885)
  integrate:  c_xM = dv sum_G a_x(G) phase Phi_M(G)         (c/lfc.c:432-505)
  derivative: c_xMv = dv sum_G a_x(G) phase dPhi_M/dv(G)    (c/lfc.c:1449-1601)
with phase = exp(2 pi i k.n) for the image displaced by n cells.
Pinned against the reference C (spline_to_grid / LFC) in
tests/test_oracle_lfc.py and tests/golden/lfc.npz.
"""
from __future__ import annotations

import itertools

import numpy as np


def spline_coefficients(f, rmax):
    """bmgs_spline (c/bmgs/spline.c:11-47) on f (last value set to 0)."""
    f = np.array(f, float)
    f[-1] = 0.0
    nbins = len(f) - 1
    dr = rmax / nbins
    c = 3.0 / (dr * dr)
    f2 = np.empty(nbins + 1)
    u = np.empty(nbins)
    f2[0] = -0.5
    u[0] = (f[1] - f[0]) * c
    for b in range(1, nbins):
        p = 0.5 * f2[b - 1] + 2.0
        f2[b] = -0.5 / p
        u[b] = ((f[b + 1] - 2.0 * f[b] + f[b - 1]) * c - 0.5 * u[b - 1]) / p
    f2[nbins] = (f[nbins - 1] * c - 0.5 * u[nbins - 1]) / (0.5 * f2[nbins - 1] + 1.0)
    for b in range(nbins - 1, -1, -1):
        f2[b] = f2[b] * f2[b + 1] + u[b]
    s = np.zeros((nbins + 1, 4))
    for b in range(nbins):
        s[b] = (f[b], (f[b + 1] - f[b]) / dr - (f2[b] / 3 + f2[b + 1] / 6) * dr,
                0.5 * f2[b], (f2[b + 1] - f2[b]) / (6 * dr))
    return s, dr, nbins


def spline_eval(coef, r):
    s, dr, nbins = coef
    b = (np.asarray(r) / dr).astype(int)
    ok = b < nbins
    b = np.where(ok, b, nbins)
    u = r - b * dr
    t = s[b]
    f = t[:, 0] + u * (t[:, 1] + u * (t[:, 2] + u * t[:, 3]))
    df = t[:, 1] + u * (2 * t[:, 2] + u * 3 * t[:, 3])
    return np.where(ok, f, 0.0), np.where(ok, df, 0.0)


def solid_harmonics(l, x, y, z):
    """c/bmgs/spherical_harmonics.h (l <= 2) and its gradient."""
    c0 = 0.28209479177387814
    c1 = 0.48860251190291992
    c2 = 1.0925484305920792
    c20 = 0.31539156525252005
    c22 = 0.54627421529603959
    r2 = x * x + y * y + z * z
    zero = np.zeros_like(x)
    if l == 0:
        return np.array([c0 + zero]), np.array([[zero, zero, zero]])
    if l == 1:
        Y = np.array([c1 * y, c1 * z, c1 * x])
        one = np.ones_like(x)
        dY = c1 * np.array([[zero, one, zero], [zero, zero, one], [one, zero, zero]])
        return Y, dY
    if l == 2:
        Y = np.array([c2 * x * y, c2 * y * z, c20 * (3 * z * z - r2), c2 * x * z,
                      c22 * (x * x - y * y)])
        dY = np.array([[c2 * y, c2 * x, zero], [zero, c2 * z, c2 * y],
                       [-2 * c20 * x, -2 * c20 * y, 4 * c20 * z],
                       [c2 * z, zero, c2 * x], [2 * c22 * x, -2 * c22 * y, zero]])
        return Y, dY
    raise NotImplementedError


def dense_functions(N_c, cell_cv, pbc_c, spos_ac, splines_aj, k_c=None,
                    derivative=False):
    """Phi (Mmax, nG) (or dPhi (Mmax, 3, nG)) on the local grid; complex with
    the Bloch phases of the images when k_c is given.  splines_aj[a] =
    [(l, rmax, f_g), ...]."""
    N_c = np.asarray(N_c)
    cell_cv = np.asarray(cell_cv, float)
    if cell_cv.ndim == 1:
        cell_cv = np.diag(cell_cv)
    pbc_c = np.asarray(pbc_c, bool)
    beg_c = np.where(pbc_c, 0, 1)
    n_c = N_c - beg_c
    h_cv = cell_cv / N_c[:, None]
    g = np.indices(tuple(n_c)).reshape(3, -1).T + beg_c
    r_gv = g @ h_cv
    Mmax = sum(2 * l + 1 for sj in splines_aj for (l, _, _) in sj)
    dt = complex if k_c is not None else float
    shape = (Mmax, 3, len(g)) if derivative else (Mmax, len(g))
    Phi = np.zeros(shape, dt)
    M = 0
    for a, sj in enumerate(splines_aj):
        for (l, rmax, f) in sj:
            coef = spline_coefficients(f, rmax)
            nm = 2 * l + 1
            nimg = [int(np.ceil(rmax / np.linalg.norm(cell_cv[c]))) + 1 if pbc_c[c] else 0
                    for c in range(3)]
            for n in itertools.product(*[range(-m, m + 1) for m in nimg]):
                n = np.array(n)
                R = (np.asarray(spos_ac[a]) + n) @ cell_cv
                d = r_gv - R
                r = np.sqrt((d**2).sum(1))
                ins = r < rmax
                if not ins.any():
                    continue
                fr, dfr = spline_eval(coef, r[ins])
                x, y, z = d[ins].T
                Y, dY = solid_harmonics(l, x, y, z)
                ph = np.exp(2j * np.pi * np.dot(k_c, n)) if k_c is not None else 1.0
                if derivative:
                    rr = r[ins]
                    fr_r = np.where(rr > 1e-15, dfr / np.where(rr > 0, rr, 1), 0.0)
                    val = fr * dY + (fr_r * Y)[:, None, :] * d[ins].T[None]
                    Phi[M:M + nm, :, ins] += ph * val
                else:
                    Phi[M:M + nm, ins] += ph * (fr * Y)
            M += nm
    return Phi


def add(a_xG, c_xM, Phi):
    """a += c Phi (Phi carries conj(image phase))."""
    return a_xG + (c_xM @ Phi.reshape(Phi.shape[0], -1)).reshape(a_xG.shape)


def integrate(a_xG, Phi, dv):
    xs = a_xG.shape[:-3]
    A = a_xG.reshape(int(np.prod(xs)) if xs else 1, -1)
    return (dv * A @ Phi.reshape(Phi.shape[0], -1).conj().T).reshape(xs + (Phi.shape[0],))
