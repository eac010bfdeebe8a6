"""Finite-difference operators on the GPU (drop-in for gpaw.fd_operators).

Same classes and signatures as the reference (gpaw/fd_operators.py:36-309):
``FDOperator(coef_p, offset_pc, gd, dtype)``, ``Laplace(gd, scale, n, dtype)``
/ ``GUCLaplace``, ``Gradient(gd, v, scale, n, dtype)``, with
``.apply(in_xg, out_xg, phase_cd)``, ``.relax(...)`` and
``.get_diagonal_element()``.  Arrays are CUDA torch tensors of shape
``(..., n0, n1, n2)``; float64/float32 for ``dtype=float``,
complex128/complex64 for ``dtype=complex``.  The stencil itself runs in
libgpawb200 (gb_operator_*), one launch for all leading (band, k) dims.

The stencil coefficients are rebuilt here from the mathematics the reference
uses: Chelikowsky et al., Phys. Rev. B 50, 11355 (1994) central-difference
weights for the Laplacian and first derivative, a least-squares fit of the
second-derivative identity over the shortest lattice directions for general
cells, and Voronoi nearest neighbours for gradients.
"""
from __future__ import annotations

from fractions import Fraction

import numpy as np
import torch

from gpaw_b200 import _native as nat
from gpaw_b200.grid_descriptor import is_real


def _central_second_derivative(n: int) -> list[float]:
    """Weights w_0..w_n of the order-2n central second derivative
    f''(0) ~ w_0 f(0) + sum_k w_k (f(k) + f(-k)), from Taylor matching:
    sum_k 2 w_k k^(2j) = [j == 1] * 2 for j = 1..n (exact rationals)."""
    A = [[Fraction(2 * k**(2 * j)) for k in range(1, n + 1)]
         for j in range(1, n + 1)]
    b = [Fraction(2 if j == 1 else 0) for j in range(1, n + 1)]
    w = _solve_exact(A, b)
    w0 = -2 * sum(w)
    return [float(w0)] + [float(x) for x in w]


def _central_first_derivative(n: int) -> list[float]:
    """Weights d_1..d_n of the order-2n first derivative
    f'(0) ~ sum_k d_k (f(k) - f(-k)): sum_k 2 d_k k^(2j-1) = [j == 1]."""
    A = [[Fraction(2 * k**(2 * j - 1)) for k in range(1, n + 1)]
         for j in range(1, n + 1)]
    b = [Fraction(1 if j == 1 else 0) for j in range(1, n + 1)]
    return [float(x) for x in _solve_exact(A, b)]


def _solve_exact(A, b):
    n = len(b)
    M = [row[:] + [bb] for row, bb in zip(A, b)]
    for i in range(n):
        p = next(r for r in range(i, n) if M[r][i] != 0)
        M[i], M[p] = M[p], M[i]
        for r in range(n):
            if r != i and M[r][i] != 0:
                f = M[r][i] / M[i][i]
                M[r] = [x - f * y for x, y in zip(M[r], M[i])]
    return [M[i][n] / M[i][i] for i in range(n)]


# Tables indexed like the reference's `laplace[n]` (n = 1..6) and
# `derivatives[n - 1]` (n = 1..4).
laplace = [[0.0]] + [_central_second_derivative(n) for n in range(1, 7)]
derivatives = [_central_first_derivative(n) for n in range(1, 5)]


class FDOperator:
    """Stencil ``out = sum_p coef_p in[. + offset_p]`` with in-kernel
    boundary conditions (zero or periodic/Bloch)."""

    def __init__(self, coef_p, offset_pc, gd, dtype=float, description=None,
                 xp=None):
        offset_pc = np.asarray(offset_pc, int).reshape(-1, 3)
        cfd = all((o != 0).sum() < 2 for o in offset_pc)
        mp = int(np.abs(offset_pc).max())
        assert (mp <= gd.n_c).all(), 'Stencil longer than domain'
        n_c = gd.n_c
        M_c = n_c + 2 * mp
        stride_c = np.array([M_c[1] * M_c[2], M_c[2], 1])
        offset_p = offset_pc.dot(stride_c)
        coef_p = np.ascontiguousarray(coef_p, float)
        assert coef_p.ndim == 1 and coef_p.shape == offset_p.shape
        self.dtype = dtype
        self.real = is_real(dtype)
        self.shape = tuple(int(x) for x in n_c)
        self.mp = mp
        self.gd = gd
        self.npoints = len(coef_p)
        self.coef_p = coef_p
        self.offset_p = offset_p
        self.offset_pc = offset_pc
        self.cfd = cfd
        self.xp = xp
        h = nat.c_void_p()
        nat.check(nat.lib().gb_operator_new(
            nat.f64(coef_p), nat.i64(offset_p), len(coef_p), nat.i64(n_c), mp,
            nat.i64(gd.neighbor_cd), int(self.real), int(cfd), nat.ctypes.byref(h)),
            'gb_operator_new')
        self._handle = h
        self.description = (description or
                            '%d point finite-difference stencil' % self.npoints)

    def __del__(self):
        h = getattr(self, '_handle', None)
        if h is not None and h.value:
            try:
                nat.lib().gb_operator_free(h)
            except Exception:
                pass

    def __str__(self):
        return '<' + self.description + '>'

    @property
    def handle(self):
        return self._handle

    def apply(self, in_xg, out_xg, phase_cd=None):
        nat.require_cuda(in_xg, out_xg)
        if in_xg.shape != out_xg.shape or tuple(in_xg.shape[-3:]) != self.shape:
            raise ValueError(f'shape mismatch: {tuple(in_xg.shape)} -> '
                             f'{tuple(out_xg.shape)} for grid {self.shape}')
        if in_xg.dtype != out_xg.dtype:
            raise ValueError('in/out dtype mismatch')
        if in_xg.dtype.is_complex == self.real:
            raise ValueError('array dtype does not match the operator dtype')
        if in_xg.dtype.is_complex and phase_cd is None:
            phase_cd = np.ones((3, 2), complex)
        nin = int(np.prod(in_xg.shape[:-3], dtype=np.int64))
        nat.check(nat.lib().gb_operator_apply(
            self._handle, nat.ptr(in_xg), nat.ptr(out_xg), nin,
            nat.dtype_code(in_xg), nat.phases(phase_cd) if in_xg.dtype.is_complex
            else None, nat.stream_of(in_xg)), 'gb_operator_apply')
        return out_xg

    def apply_potential(self, in_xg, out_xg, vt_g, phase_cd=None):
        """out = op(in) + vt * in (vt: one real grid, broadcast over the
        leading dims) in one fused pass -- the local pseudo-Hamiltonian."""
        nat.require_cuda(in_xg, out_xg, vt_g)
        if in_xg.shape != out_xg.shape or tuple(in_xg.shape[-3:]) != self.shape:
            raise ValueError('shape mismatch')
        if tuple(vt_g.shape) != self.shape:
            raise ValueError('potential must have the grid shape')
        real_t = torch.float32 if in_xg.dtype in (torch.float32, torch.complex64) else torch.float64
        if vt_g.dtype != real_t:
            raise ValueError(f'potential dtype must be {real_t}')
        if in_xg.dtype.is_complex and phase_cd is None:
            phase_cd = np.ones((3, 2), complex)
        nin = int(np.prod(in_xg.shape[:-3], dtype=np.int64))
        nat.check(nat.lib().gb_operator_apply_potential(
            self._handle, nat.ptr(in_xg), nat.ptr(out_xg), nin, nat.dtype_code(in_xg),
            nat.ptr(vt_g), nat.phases(phase_cd) if in_xg.dtype.is_complex else None,
            nat.stream_of(in_xg)), 'gb_operator_apply_potential')
        return out_xg

    def __call__(self, in_xg, out_xg=None, phase_cd=None):
        if out_xg is None:
            out_xg = torch.empty_like(in_xg)
        return self.apply(in_xg, out_xg, phase_cd)

    def relax(self, relax_method, f_g, s_g, n, w=None):
        nat.require_cuda(f_g, s_g)
        assert f_g.dtype == torch.float64 and tuple(f_g.shape) == self.shape
        nat.check(nat.lib().gb_operator_relax(
            self._handle, relax_method, nat.ptr(f_g), nat.ptr(s_g), n,
            1.0 if w is None else w, nat.stream_of(f_g)), 'gb_operator_relax')

    def get_diagonal_element(self):
        d = nat.c_double()
        nat.check(nat.lib().gb_operator_get_diagonal_element(
            self._handle, nat.ctypes.byref(d)), 'get_diagonal_element')
        return d.value

    def get_async_sizes(self):
        return (0, 1, 1)


def Laplace(gd, scale=1.0, n=1, dtype=float, xp=None):
    if n == 9:
        raise NotImplementedError('FTLaplace (n=9) is not part of this build')
    return GUCLaplace(gd, scale, n, dtype, xp=xp)


class GUCLaplace(FDOperator):
    def __init__(self, gd, scale=1.0, n=1, dtype=float, xp=None):
        """Laplacian for a general (possibly non-orthorhombic) cell.

        The second-derivative identity sum_d a_d (h_d . grad)^2 = nabla^2 is
        fitted by least squares over the D = 3..6 shortest lattice directions
        (the same construction as gpaw/fd_operators.py:192-216); each
        direction then gets the 1-D order-2n weights."""
        M_ic = np.indices((3, 3, 3)).reshape((3, -3)).T[-13:] - 1
        u_cv = gd.h_cv / (gd.h_cv**2).sum(1)[:, np.newaxis]**0.5
        u2_i = (np.dot(M_ic, u_cv)**2).sum(1)
        i_d = u2_i.argsort()
        m_mv = np.array([(2, 0, 0), (0, 2, 0), (0, 0, 2),
                         (0, 1, 1), (1, 0, 1), (1, 1, 0)])
        for D in range(3, 7):
            h_dv = np.dot(M_ic[i_d[:D]], gd.h_cv)
            A_md = (h_dv**m_mv[:, np.newaxis, :]).prod(2)
            a_d, residual, rank, s = np.linalg.lstsq(
                A_md, [1, 1, 1, 0, 0, 0], rcond=-1)
            if residual.sum() < 1e-14:
                if rank != D:
                    raise ValueError('You have a weird unit cell!  Try to use '
                                     'the maximally reduced Niggli cell.')
                break
        a_d *= scale
        offsets = [(0, 0, 0)]
        coefs = [laplace[n][0] * a_d.sum()]
        for d in range(D):
            M_c = M_ic[i_d[d]]
            offsets.extend(np.arange(1, n + 1)[:, np.newaxis] * M_c)
            coefs.extend(a_d[d] * np.array(laplace[n][1:]))
            offsets.extend(np.arange(-1, -n - 1, -1)[:, np.newaxis] * M_c)
            coefs.extend(a_d[d] * np.array(laplace[n][1:]))
        FDOperator.__init__(self, coefs, offsets, gd, dtype, xp=xp)
        self.description = (
            '%d*%d+1=%d point O(h^%d) finite-difference Laplacian' %
            ((self.npoints - 1) // n, n, self.npoints, 2 * n))


class Gradient(FDOperator):
    def __init__(self, gd, v, scale=1.0, n=1, dtype=float, xp=None):
        """Symmetric gradient along Cartesian direction v for a general cell
        (Voronoi nearest neighbours + a 3x3 solve per lattice direction, as
        gpaw/fd_operators.py:251-303)."""
        from scipy.spatial import Voronoi
        M_ic = np.indices((3, 3, 3)).reshape((3, -1)).T - 1
        h_iv = M_ic.dot(gd.h_cv)
        voro = Voronoi(h_iv)
        i_d = []
        for i1, i2 in voro.ridge_points:
            if i1 == 13 and i2 > 13:
                i_d.append(i2)
            elif i2 == 13 and i1 > 13:
                i_d.append(i1)
        D = len(i_d)
        h_dv = h_iv[i_d]
        invh_vc = np.linalg.inv(gd.h_cv)
        n_cv = (invh_vc / (invh_vc**2).sum(axis=0)**0.5).T
        coef_cd = np.zeros((3, D))
        for c, n_v in enumerate(n_cv):
            ok_d = abs(h_dv.dot(n_v)) > 1e-10
            h_mv = h_dv[ok_d]
            A_jm = np.array([h_mv.dot(n_v), h_mv.dot(gd.h_cv[c - 1]),
                             h_mv.dot(gd.h_cv[c - 2])])
            U_jm, S_m, V_mm = np.linalg.svd(A_jm, full_matrices=False)
            coef_cd[c, ok_d] = V_mm.T.dot(np.diag(S_m**-1).dot(
                U_jm.T.dot([1, 0, 0])))
        coef_d = np.linalg.inv(n_cv)[v].dot(coef_cd) * scale
        offsets = []
        coefs = []
        stencil = np.array(derivatives[n - 1])
        for d, c in enumerate(coef_d):
            if abs(c) < 1e-10:
                continue
            M_c = M_ic[i_d[d]]
            offsets.extend(np.arange(1, n + 1)[:, np.newaxis] * M_c)
            coefs.extend(c * stencil)
            offsets.extend(np.arange(-1, -n - 1, -1)[:, np.newaxis] * M_c)
            coefs.extend(-c * stencil)
        FDOperator.__init__(self, coefs, offsets, gd, dtype, xp=xp)
        self.description = (
            'Finite-difference {}-derivative with O(h^{}) error ({} points)'
            .format('xyz'[v], 2 * n, self.npoints))
