"""Radial cubic splines (drop-in for gpaw.spline.Spline).

``Spline.from_data(l, rmax, f_g)`` tabulates f on nbins+1 equidistant points
r = 0..rmax (the last value is forced to 0, gpaw/spline.py:19-31) and builds
the cubic spline of c/bmgs/spline.c:11-47: zero slope at r = 0, the
tridiagonal second-derivative solve of that routine, per-bin polynomial
s0 + u (s1 + u (s2 + u s3)) with u = r - b dr; values beyond rmax are 0.
The construction has to be the reference's for the localized functions to
agree point by point, so the recurrences are kept as they are there.
Host-side (numpy): splines are evaluated when positions change, not per
SCF step.
"""
from __future__ import annotations

import numpy as np


class Spline:
    def __init__(self, l, rmax, f_g):
        f_g = np.ascontiguousarray(f_g, float)
        self.l = int(l)
        self.rmax = float(rmax)
        self.nbins = len(f_g) - 1
        self.dr = self.rmax / self.nbins
        self.f_g = f_g
        self.coef_b4 = self._build(f_g, self.dr)

    @classmethod
    def from_data(cls, l, rmax, f_g):
        assert rmax > 0.0
        f_g = np.array(f_g, float)
        f_g[-1] = 0.0
        return cls(l, rmax, f_g)

    @staticmethod
    def _build(f, dr):
        nbins = len(f) - 1
        c = 3.0 / (dr * dr)
        f2 = np.empty(nbins + 1)
        u = np.empty(nbins)
        f2[0] = -0.5
        u[0] = (f[1] - f[0]) * c
        for b in range(1, nbins):
            p = 0.5 * f2[b - 1] + 2.0
            f2[b] = -0.5 / p
            u[b] = ((f[b + 1] - 2.0 * f[b] + f[b - 1]) * c - 0.5 * u[b - 1]) / p
        f2[nbins] = ((f[nbins - 1] * c - 0.5 * u[nbins - 1]) /
                     (0.5 * f2[nbins - 1] + 1.0))
        for b in range(nbins - 1, -1, -1):
            f2[b] = f2[b] * f2[b + 1] + u[b]
        s = np.zeros((nbins + 1, 4))
        s[:nbins, 0] = f[:nbins]
        s[:nbins, 1] = ((f[1:] - f[:-1]) / dr -
                        (f2[:-1] / 3 + f2[1:] / 6) * dr)
        s[:nbins, 2] = 0.5 * f2[:-1]
        s[:nbins, 3] = (f2[1:] - f2[:-1]) / (6 * dr)
        return s

    # -- device object ----------------------------------------------------
    @property
    def handle(self):
        """The gb_spline of this function (made on first use; holds the
        coefficient table in device memory)."""
        h = getattr(self, '_handle', None)
        if h is None:
            from gpaw_b200 import _native as nat
            h = nat.c_void_p()
            nat.check(nat.lib().gb_spline_new(self.l, self.rmax, self.nbins,
                                              nat.f64(self.f_g), nat.ctypes.byref(h)),
                      'gb_spline_new')
            self._handle = h
        return h

    def __del__(self):
        h = getattr(self, '_handle', None)
        if h is not None and h.value:
            try:
                from gpaw_b200 import _native as nat
                nat.lib().gb_spline_free(h)
            except Exception:
                pass

    # -- reference interface ----------------------------------------------
    def get_cutoff(self):
        return self.rmax

    def get_angular_momentum_number(self):
        return self.l

    def get_npoints(self):
        return self.nbins + 1

    def __repr__(self):
        return 'Spline(l={}, rmax={:.2f}, ...)'.format(self.l, self.rmax)

    def value_and_derivative(self, r):
        """Vectorised f(r), f'(r) (bmgs_get_value_and_derivative)."""
        r = np.asarray(r, float)
        b = (r / self.dr).astype(np.int64)
        inside = b < self.nbins
        b = np.where(inside, b, self.nbins)
        u = r - b * self.dr
        s = self.coef_b4[b]
        f = s[..., 0] + u * (s[..., 1] + u * (s[..., 2] + u * s[..., 3]))
        df = s[..., 1] + u * (2.0 * s[..., 2] + u * 3.0 * s[..., 3])
        return np.where(inside, f, 0.0), np.where(inside, df, 0.0)

    def __call__(self, r):
        return float(self.value_and_derivative(np.array([r]))[0][0])

    def map(self, r_x):
        return self.value_and_derivative(np.asarray(r_x))[0]

    def get_value_and_derivative(self, r):
        f, df = self.value_and_derivative(np.array([r]))
        return float(f[0]), float(df[0])


# ---------------------------------------------------------------------------
# Real solid spherical harmonics r^l Y_lm (l <= 2 here; l = 3, 4 follow the
# same construction).  Normalisation constants are the standard ones,
# c_00 = 1/sqrt(4 pi), c_1 = sqrt(3/(4 pi)), c_2a = sqrt(15/(4 pi)),
# c_20 = sqrt(5/(16 pi)), c_22 = sqrt(15/(16 pi)); the m ordering is that of
# c/bmgs/spherical_harmonics.h (l=1: y, z, x; l=2: xy, yz, 3z^2-r^2, xz,
# x^2-y^2).
_C00 = 1 / np.sqrt(4 * np.pi)
_C1 = np.sqrt(3 / (4 * np.pi))
_C2A = np.sqrt(15 / (4 * np.pi))
_C20 = np.sqrt(5 / (16 * np.pi))
_C22 = np.sqrt(15 / (16 * np.pi))


def rlYlm(l, x, y, z):
    """(2l+1, ...) array of r^l Y_lm at the points (x, y, z)."""
    if l == 0:
        return np.array([_C00 * np.ones_like(x)])
    if l == 1:
        return _C1 * np.array([y, z, x])
    if l == 2:
        r2 = x * x + y * y + z * z
        return np.array([_C2A * x * y, _C2A * y * z, _C20 * (3 * z * z - r2),
                         _C2A * x * z, _C22 * (x * x - y * y)])
    raise NotImplementedError('l > 2 localized functions')
