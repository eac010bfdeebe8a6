"""HGH norm-conserving pseudopotentials (the setups GPAW builds with
setups='hgh', gpaw/hgh.py), as radial functions for the FD path.

Published forms (Hartwigsen, Goedecker & Hutter, PRB 58, 3641 (1998)):
  v_loc(r) = -Z erf(r / (sqrt2 r_loc)) / r
             + exp(-r^2 / (2 r_loc^2)) sum_i C_i (r / r_loc)^(2i-2)
  p_i^l(r) = sqrt2 r^(l+2i-2) exp(-r^2 / (2 r_l^2))
             / (r_l^(l+(4i-1)/2) sqrt(Gamma(l + (4i-1)/2)))
  V_nl = sum_lm sum_ij |p_i^l Y_lm> h^l_ij <p_j^l Y_lm|
with the off-diagonal h^l_ij fixed by the diagonal ones (the paper's
relations; gpaw/hgh.py:307-345).  The parameters below are the published
LDA values for H, O and Si (the same numbers as gpaw/hgh_parameters.py).

For the grid: the long-range part of v_loc is the potential of a Gaussian
ion charge of width r_g (well resolved on the fine grid), handled by the
Poisson solver; the remainder  dv(r) = v_loc(r) + Z erf(r/(sqrt2 r_g))/r  is
short-ranged and is added with an LFC ('vbar').
"""
from __future__ import annotations

from math import erf, gamma, pi, sqrt

import numpy as np

# symbol: (Z_valence, r_loc, [C1..C4], [(r_l, [h_11, h_22, h_33]) for l = 0, 1, ...])
HGH_LDA = {
    'H': (1, 0.200000, [-4.180237, 0.725075], []),
    'O': (6, 0.247621, [-16.580318, 2.395701], [(0.221786, [18.266917]),
                                                 (0.256829, [0.0])]),
    'Si': (4, 0.440000, [-7.336103], [(0.422738, [5.906928, 3.258196]),
                                      (0.484278, [2.727013, 0.0])]),
}

# off-diagonal relations h_12, h_13, h_23 in units of h_22, h_33, h_33
_HCOEF = [[-0.5 * sqrt(3 / 5), 0.5 * sqrt(5 / 21), -0.5 * sqrt(100 / 63)],
          [-0.5 * sqrt(5 / 7), 1 / 6 * sqrt(35 / 11), -1 / 6 * 14 / sqrt(11)],
          [-0.5 * sqrt(7 / 9), 0.5 * sqrt(63 / 143), -0.5 * 18 / sqrt(143)]]


def h_matrix(l, h_diag):
    n = len(h_diag)
    h = np.diag(np.array(h_diag, float))
    if n > 1:
        h[0, 1] = h[1, 0] = _HCOEF[l][0] * h_diag[1]
    if n > 2:
        h[0, 2] = h[2, 0] = _HCOEF[l][1] * h_diag[2]
        h[1, 2] = h[2, 1] = _HCOEF[l][2] * h_diag[2]
    return h


class HGHSetup:
    """Radial data of one element for the grid calculation."""

    def __init__(self, symbol, r_gauss=0.6, ngrid=400):
        from gpaw_b200.spline import Spline
        Z, rloc, C, nl = HGH_LDA[symbol]
        self.symbol = symbol
        self.Z = Z
        self.rloc = rloc
        self.r_gauss = max(r_gauss, rloc)
        rg = self.r_gauss
        Y00 = 1 / sqrt(4 * pi)
        # short-range local potential dv(r) (times sqrt(4 pi): LFC functions carry Y00)
        rc = rg * 7.0
        r = np.linspace(0, rc, ngrid + 1)
        with np.errstate(invalid='ignore', divide='ignore'):
            t1 = np.array([erf(x / (sqrt(2) * rloc)) for x in r])
            t2 = np.array([erf(x / (sqrt(2) * rg)) for x in r])
            lr = np.where(r > 0, -Z * (t1 - t2) / np.where(r > 0, r, 1), 0.0)
        lr[0] = -Z * sqrt(2 / pi) * (1 / rloc - 1 / rg)
        x2 = (r / rloc)**2
        poly = sum(c * x2**i for i, c in enumerate(C))
        dv = lr + np.exp(-0.5 * x2) * poly
        self.vbar = Spline.from_data(0, rc, dv / Y00)
        # Gaussian ion charge (magnitude; the ion density is minus this, and
        # its potential is -Z erf(r/(sqrt2 rg))/r)
        rc_g = rg * 7.0
        r = np.linspace(0, rc_g, ngrid + 1)
        rho = Z * np.exp(-r**2 / (2 * rg**2)) / ((2 * pi)**1.5 * rg**3)
        self.ghat = Spline.from_data(0, rc_g, rho / Y00)
        # valence density guess: Gaussian of width 1 Bohr holding Z electrons
        rc_n = 6.0
        r = np.linspace(0, rc_n, ngrid + 1)
        nv = Z * np.exp(-r**2 / 2.0) / ((2 * pi)**1.5)
        self.nguess = Spline.from_data(0, rc_n, nv / Y00)
        # projectors: radial part p(r) / r^l
        self.pt_j = []
        self.l_j = []
        hblocks = []
        for l, (rl, hd) in enumerate(nl):
            nproj = len(hd)
            if not np.any(hd):
                continue
            rc_p = rl * sqrt(2 * 45.0)
            r = np.linspace(0, rc_p, ngrid + 1)
            for i in range(1, nproj + 1):
                A = rl**(l + (4 * i - 1) / 2.0)
                B = sqrt(gamma(l + (4 * i - 1) / 2.0))
                f = sqrt(2.0) / A / B * r**(2 * (i - 1)) * np.exp(-0.5 * r**2 / rl**2)
                self.pt_j.append(Spline.from_data(l, rc_p, f))
                self.l_j.append(l)
            hblocks.append((l, h_matrix(l, hd)))
        # expand h^l_ij to the (j, m) function index used by the projector LFC
        ni = sum(2 * l + 1 for l in self.l_j)
        self.ni = ni
        H = np.zeros((ni, ni))
        offs = []
        o = 0
        for l in self.l_j:
            offs.append(o)
            o += 2 * l + 1
        jl = {}
        for j, l in enumerate(self.l_j):
            jl.setdefault(l, []).append(j)
        for l, h in hblocks:
            js = jl[l]
            for a, ja in enumerate(js):
                for b, jb in enumerate(js):
                    for m in range(2 * l + 1):
                        H[offs[ja] + m, offs[jb] + m] = h[a, b]
        self.dH_ii = H
