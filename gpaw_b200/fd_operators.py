"""Finite-difference operators on the GPU (drop-in for gpaw.fd_operators).

Same classes and signatures as the reference (gpaw/fd_operators.py:36-309):
``FDOperator(coef_p, offset_pc, gd, dtype)``, ``Laplace(gd, scale, n, dtype)``
/ ``GUCLaplace``, ``Gradient(gd, v, scale, n, dtype)``, with
``.apply(in_xg, out_xg, phase_cd)``, ``.relax(...)`` and
``.get_diagonal_element()``.  Arrays are CUDA torch tensors of shape
``(..., n0, n1, n2)``; float64/float32 for ``dtype=float``,
complex128/complex64 for ``dtype=complex``.  The stencil itself runs in
libgpawb200 (gb_operator_*), one launch for all leading (band, k) dims.

The stencil coefficients are derived here from the mathematics:
central-difference weights of order 2n for the second and first derivative
(exact Taylor matching, as tabulated by Chelikowsky et al., Phys. Rev. B 50,
11355 (1994)); for general cells the Laplacian is a combination of
second derivatives along the shortest grid steps whose second-moment
tensors sum to the identity, and the gradient combines first differences
along the steps to the Voronoi neighbours of a grid point.
"""
from __future__ import annotations

import itertools
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
        if in_xg.dtype.is_complex and nat.is_phase_batch(phase_cd):
            return self._apply_k(in_xg, out_xg, nin, phase_cd, None)
        nat.check(nat.lib().gb_operator_apply(
            self._handle, nat.ptr(in_xg), nat.ptr(out_xg), nin,
            nat.dtype_code(in_xg), nat.phases(phase_cd) if in_xg.dtype.is_complex
            else None, nat.stream_of(in_xg)), 'gb_operator_apply')
        return out_xg

    def _apply_k(self, in_xg, out_xg, nin, phase_kcd, vt_g):
        """A k-point batch: leading dims hold nk equal groups of grids,
        group k with the Bloch phases phase_kcd[k] (one launch)."""
        nk, ph = nat.phase_sets(phase_kcd)
        nat.check(nat.lib().gb_operator_apply_k(
            self._handle, nat.ptr(in_xg), nat.ptr(out_xg), nin, nat.dtype_code(in_xg), nk,
            ph, nat.ptr(vt_g) if vt_g is not None else None, nat.stream_of(in_xg)),
            'gb_operator_apply_k')
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
        if in_xg.dtype.is_complex and nat.is_phase_batch(phase_cd):
            return self._apply_k(in_xg, out_xg, nin, phase_cd, vt_g)
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


def _half_space_steps():
    """The 13 grid steps M in {-1, 0, 1}^3 that are lexicographically
    positive (one of each +-M pair), in lexicographic order."""
    return np.array([m for m in itertools.product((-1, 0, 1), repeat=3)
                     if m > (0, 0, 0)])


def _second_moments(E_dv):
    """Rows xx, yy, zz, yz, xz, xy of the tensors e_d e_d^T (one column per
    step vector e_d)."""
    x, y, z = E_dv.T
    return np.array([x * x, y * y, z * z, y * z, x * z, x * y])


def laplace_stencil(h_cv, scale=1.0, n=1):
    """(coef_p, offset_pc) of the order-2n Laplacian on a general grid.

    nabla^2 = sum_d a_d (e_d . nabla)^2 holds exactly when the step vectors
    e_d (lattice steps M_d h_cv) satisfy sum_d a_d e_d e_d^T = 1, six
    equations in the a_d.  The steps are taken shortest first, where
    "short" is measured on the grid axes normalised to unit length (so
    the choice depends on the angles between the axes, not on their
    spacing), with ties kept in lexicographic order; the first 3, 4, 5 or 6
    of them whose moment equations have an exact solution are used, and a
    set whose moment tensors are linearly dependent is an error, as in the
    reference (gpaw/fd_operators.py:179-235).  Along each step the 1-D
    order-2n second-derivative weights apply: centre sum_d a_d w_0, then
    a_d w_k at +-k M_d."""
    h_cv = np.asarray(h_cv, float)
    steps = _half_space_steps()
    axes = h_cv / np.linalg.norm(h_cv, axis=1)[:, None]
    length2 = ((steps @ axes)**2).sum(1)
    order = np.argsort(length2, kind='stable')
    target = np.array([1.0, 1.0, 1.0, 0.0, 0.0, 0.0])
    for D in range(3, 7):
        M_d = steps[order[:D]]
        A = _second_moments(M_d @ h_cv)              # (6, D)
        Q, R = np.linalg.qr(A)
        sv = np.linalg.svd(A, compute_uv=False)
        if sv[-1] <= sv[0] * 1e-12:
            raise ValueError('You have a weird unit cell!  Try to use the '
                             'maximally reduced Niggli cell.')
        a_d = np.linalg.solve(R, Q.T @ target)
        if D == 6 or ((A @ a_d - target)**2).sum() < 1e-14:
            break
    a_d = a_d * scale
    w = laplace[n]
    coefs = [w[0] * a_d.sum()]
    offsets = [np.zeros(3, int)]
    for a, M in zip(a_d, M_d):
        for sign in (1, -1):
            for k in range(1, n + 1):
                offsets.append(sign * k * M)
                coefs.append(a * w[k])
    return np.array(coefs), np.array(offsets).reshape(-1, 3)


def _voronoi_relevant_steps(h_cv):
    """Steps M (one of each +-M pair, lexicographic order) whose grid point
    shares a face of positive area with the Voronoi cell of the origin,
    among the 27 points {-1, 0, 1}^3 h_cv.  The face between 0 and p is
    symmetric about p / 2, so it has positive area exactly when p / 2 is
    strictly closer to 0 and p than to every other point q:
    q . (q - p) > 0 (up to rounding)."""
    pts = np.array(list(itertools.product((-1, 0, 1), repeat=3))) @ h_cv
    tol = 1e-10 * (np.asarray(h_cv)**2).sum(1).max()
    out = []
    for M in _half_space_steps():
        p = M @ h_cv
        others = [q for q in pts if np.any(np.abs(q) > 0) and
                  np.any(np.abs(q - p) > 1e-14 * np.abs(p).max())]
        if all(q @ (q - p) > tol for q in others):
            out.append(M)
    return np.array(out)


def gradient_stencil(h_cv, v, scale=1.0, n=1):
    """(coef_p, offset_pc) of the order-2n derivative along Cartesian axis
    v on a general grid.

    Uses the steps M_d to the Voronoi neighbours of a grid point.  For each
    grid axis c, n_c is the unit normal of the plane of the two other axes
    (the normalised reciprocal vector); the weights b_cd are the
    minimum-norm solution of sum_d b_cd e_d = n_c over the steps not lying
    in that plane (e_d = M_d h_cv), so that sum_d b_cd (f(r + e_d) -
    f(r - e_d)) / 2 approximates n_c . grad f.  The Cartesian derivative is
    the combination sum_c (N^-1)_vc of these (N the matrix of the n_c), and
    each step carries the 1-D order-2n first-derivative weights
    (gpaw/fd_operators.py:238-303 builds the same operator)."""
    h_cv = np.asarray(h_cv, float)
    M_d = _voronoi_relevant_steps(h_cv)
    E_dv = M_d @ h_cv
    recip = np.linalg.inv(h_cv).T                     # rows: reciprocal vectors
    N_cv = recip / np.linalg.norm(recip, axis=1)[:, None]
    b_cd = np.zeros((3, len(M_d)))
    for c in range(3):
        use = np.abs(E_dv @ N_cv[c]) > 1e-10
        B = E_dv[use].T                               # (3, m) steps as columns
        # n_c lies in the span of the steps used; lstsq gives the
        # minimum-norm weights also when they span less than 3 dimensions
        b_cd[c, use] = np.linalg.lstsq(B, N_cv[c], rcond=None)[0]
    coef_d = np.linalg.inv(N_cv)[v] @ b_cd * scale
    d_k = derivatives[n - 1]
    coefs, offsets = [], []
    for c, M in zip(coef_d, M_d):
        if abs(c) < 1e-10:
            continue
        for sign in (1, -1):
            for k in range(1, n + 1):
                offsets.append(sign * k * M)
                coefs.append(sign * c * d_k[k - 1])
    return np.array(coefs), np.array(offsets).reshape(-1, 3)


def Laplace(gd, scale=1.0, n=1, dtype=float, xp=None):
    if n == 9:
        return FTLaplace(gd, scale, dtype)
    return GUCLaplace(gd, scale, n, dtype, xp=xp)


class FTLaplace:
    """The spectral Laplacian that Laplace(gd, scale, n=9) returns
    (gpaw/fd_operators.py:357-382): on a periodic grid,
    out = Re F^-1[-scale |k|^2 F[in]] with k the reciprocal-lattice vectors of
    the FFT frequencies (folded to -N/2 .. N/2 - 1 per axis), applied to all
    leading (band) dimensions at once through cuFFT (torch.fft).  Like the
    reference it keeps the real part, and its diagonal element is
    6 / h_00^2 whatever the scale."""

    def __init__(self, gd, scale=1.0, dtype=float, xp=None):
        if not np.all(gd.pbc_c):
            raise ValueError('FTLaplace needs a periodic grid')
        N_c = np.asarray(gd.N_c)
        i_cq = np.indices(tuple(N_c)).reshape(3, -1)
        half = (N_c // 2)[:, None]
        i_cq = (i_cq + half) % N_c[:, None] - half
        k_vq = (2.0 * np.pi * gd.icell_cv.T) @ i_cq
        k2 = -scale * (k_vq**2).sum(0).reshape(tuple(N_c))
        self.gd = gd
        self.k2_Q = torch.as_tensor(k2, dtype=torch.float64, device=gd.device)
        self.d = 6.0 / gd.h_cv[0, 0]**2
        self.npoints = 1000
        self.description = 'FFT Laplacian'

    def apply(self, in_xg, out_xg, phase_cd=None):
        if not in_xg.is_cuda:
            raise nat.GPAWB200Error('FTLaplace.apply needs CUDA tensors')
        f = torch.fft.fftn(in_xg.to(torch.complex128), dim=(-3, -2, -1))
        y = torch.fft.ifftn(f * self.k2_Q, dim=(-3, -2, -1)).real
        out_xg.copy_(y.to(out_xg.dtype) if not out_xg.dtype.is_complex else y)
        return out_xg

    def get_diagonal_element(self):
        return self.d


class GUCLaplace(FDOperator):
    def __init__(self, gd, scale=1.0, n=1, dtype=float, xp=None):
        """Order-2n Laplacian for a general (possibly non-orthorhombic)
        grid; coefficients from `laplace_stencil`."""
        coefs, offsets = laplace_stencil(gd.h_cv, scale, n)
        FDOperator.__init__(self, coefs, offsets, gd, dtype, xp=xp)
        ndir = (self.npoints - 1) // (2 * n)
        self.description = (f'{ndir} directions x {2 * n} + 1 = {self.npoints} '
                            f'point O(h^{2 * n}) finite-difference Laplacian')


class Gradient(FDOperator):
    def __init__(self, gd, v, scale=1.0, n=1, dtype=float, xp=None):
        """Order-2n derivative along Cartesian axis v for a general grid;
        coefficients from `gradient_stencil`."""
        coefs, offsets = gradient_stencil(gd.h_cv, v, scale, n)
        FDOperator.__init__(self, coefs, offsets, gd, dtype, xp=xp)
        self.description = (f'O(h^{2 * n}) finite-difference derivative along '
                            f'{"xyz"[v]} ({self.npoints} points)')
