"""ORACLE (test infrastructure): boundary padding, FD stencils, restriction,
interpolation and the multigrid preconditioner V-cycle in numpy.

References (GPAW source tree):
  c/bc.c:146-258          halo fill: zero boundaries, periodic copies with
                          Bloch phases (phase[c][0] on the upper halo,
                          phase[c][1] on the lower halo), axes 0, 1, 2 in turn
  c/bmgs/fd.c:9-33        out[j] = sum_c coefs[c] * a[i + offsets[c]]
                          (summed from 0.0 in coefficient order)
  c/bmgs/restrict.c:17-62,136-155   separable restriction, passes along the
                          last axis first, 0.5*(a0 + w1(a1+a-1) + w3(...)...)
  c/bmgs/interpolate.c:10-46,227-257 separable interpolation with skip flags
  gpaw/transformers.py:27-47        pad/skip geometry
  c/fd_preconditioner.c:207-348 == gpaw/preconditioner.py:74-93  V-cycle
"""
from __future__ import annotations

from fractions import Fraction

import numpy as np


# ------------------------------------------------------------------ padding
def pad_bc(a_xg, pad_cd, pbc_c, phase_cd=None):
    """Pad the last three axes by pad_cd[c] = (lo, hi) cells following
    c/bc.c:146-258 for one domain: zeros on non-periodic axes; on periodic
    axes the upper halo holds the first cells times phase_cd[c][0], the
    lower halo the last cells times phase_cd[c][1].  Axes are processed in
    order 0, 1, 2 over the full extent already padded, so corners carry the
    product of the phases (the non-cfd path of c/bc.c:108-112)."""
    a = np.asarray(a_xg)
    nd = a.ndim
    out = a
    for c in range(3):
        lo, hi = int(pad_cd[c][0]), int(pad_cd[c][1])
        ax = nd - 3 + c
        n = out.shape[ax]
        if pbc_c[c]:
            assert lo <= n and hi <= n
            low = np.take(out, range(n - lo, n), axis=ax)
            high = np.take(out, range(0, hi), axis=ax)
            if phase_cd is not None:
                low = low * phase_cd[c][1]
                high = high * phase_cd[c][0]
        else:
            shp = list(out.shape)
            shp[ax] = lo
            low = np.zeros(shp, out.dtype)
            shp[ax] = hi
            high = np.zeros(shp, out.dtype)
        out = np.concatenate([low.astype(out.dtype), out,
                              high.astype(out.dtype)], axis=ax)
    return out


# ------------------------------------------------------------------ stencil
def fd_apply(coef_p, offset_pc, a_xg, pbc_c, phase_cd=None):
    """bmgs_fd / bmgs_fdz (c/bmgs/fd.c:9-33) on a bc-padded copy."""
    a = np.asarray(a_xg)
    offset_pc = np.asarray(offset_pc, int).reshape(-1, 3)
    mp = int(np.abs(offset_pc).max()) if len(offset_pc) else 0
    n = a.shape[-3:]
    b = pad_bc(a, [(mp, mp)] * 3, pbc_c, phase_cd)
    out = np.zeros_like(a)
    for coef, (o0, o1, o2) in zip(coef_p, offset_pc):
        out = out + b[..., mp + o0:mp + o0 + n[0], mp + o1:mp + o1 + n[1],
                      mp + o2:mp + o2 + n[2]] * coef
    return out


def jacobi_relax(coef_p, offset_pc, f_g, s_g, pbc_c, nrelax, w):
    """Weighted Jacobi sweeps, c/bmgs/relax.c:40-66 (relax_method 2):
    f <- (1 - w) f + w (s - sum_{c >= 1} coef_c f[. + o_c]) / coef_0, with
    the centre coefficient first in the list as Laplace builds it."""
    offset_pc = np.asarray(offset_pc, int).reshape(-1, 3)
    f = np.array(f_g, dtype=float)
    c0 = coef_p[0]
    assert not offset_pc[0].any()
    for _ in range(nrelax):
        x = fd_apply(coef_p[1:], offset_pc[1:], f, pbc_c)
        f = (1.0 - w) * f + w * (np.asarray(s_g) - x) / c0
    return f


# ------------------------------------------------------------------ transformer weights
def midpoint_weights(k: int) -> list[float]:
    """Lagrange weights of the degree-(k-1) interpolant through the k points
    +-1/2, +-3/2, ... evaluated at 0 (the weights of restrict.c:36-56 and
    interpolate.c:184-197): returns w for the pairs at distance 1/2, 3/2..."""
    xs = [Fraction(2 * i - k + 1, 2) for i in range(k)]
    w = []
    for i, xi in enumerate(xs):
        num, den = Fraction(1), Fraction(1)
        for j, xj in enumerate(xs):
            if j != i:
                num *= (0 - xj)
                den *= (xi - xj)
        w.append(num / den)
    # symmetric: pair j (distance (2j+1)/2) has weight w[k//2 + j]
    return [float(w[k // 2 + j]) for j in range(k // 2)]


def transformer_geometry(gdin_beg, gdin_end, gdout_beg, gdout_end, nn,
                         restrict):
    """pad_cd, neighborpad_cd, skip_cd of gpaw/transformers.py:27-47."""
    gdin_beg, gdin_end = np.asarray(gdin_beg), np.asarray(gdin_end)
    gdout_beg, gdout_end = np.asarray(gdout_beg), np.asarray(gdout_end)
    pad = np.empty((3, 2), int)
    npad = np.empty((3, 2), int)
    skip = np.zeros((3, 2), int)
    if restrict:
        pad[:, 0] = 2 * nn - 1 - 2 * gdout_beg + gdin_beg
        pad[:, 1] = 2 * nn - 2 + 2 * gdout_end - gdin_end
        npad[:, 0] = 2 * nn - 2 + 2 * gdout_beg - gdin_beg
        npad[:, 1] = 2 * nn - 1 - 2 * gdout_end + gdin_end
    else:
        pad[:, 0] = nn - 1 - gdout_beg // 2 + gdin_beg
        pad[:, 1] = nn + gdout_end // 2 - gdin_end
        npad[:, 0] = nn + gdout_beg // 2 - gdin_beg
        npad[:, 1] = nn - 1 - gdout_end // 2 + gdin_end
        skip[:, 0] = gdout_beg % 2
        skip[:, 1] = gdout_end % 2
    return pad, npad, skip


def _restrict_1d(a, axis, k):
    """RST1D (c/bmgs/restrict.c:29-59) along `axis` of a padded array."""
    w = midpoint_weights(k)
    n = a.shape[axis]
    nout = (n - 2 * k + 3) // 2
    c = (k - 1) + 2 * np.arange(nout)
    take = lambda idx: np.take(a, idx, axis=axis)
    x = take(c)
    for j, wj in enumerate(w):
        d = 2 * j + 1
        x = x + wj * (take(c + d) + take(c - d))
    return 0.5 * x


def _interpolate_1d(a, axis, k, skip):
    """IP1D (c/bmgs/interpolate.c:10-46) along `axis` of a padded array."""
    w = midpoint_weights(k)
    size = a.shape[axis]
    n = size - (k - 1) + skip[1]
    base = k // 2 - 1
    i = np.arange(n)
    take = lambda idx: np.take(a, idx, axis=axis)
    even = take(base + i)
    odd = None
    for j, wj in enumerate(w):
        t = wj * (take(base + i - j) + take(base + i + 1 + j))
        odd = t if odd is None else odd + t
    shp = list(a.shape)
    shp[axis] = 2 * n
    out = np.empty(shp, np.result_type(a.dtype, float))
    idx_e = [slice(None)] * a.ndim
    idx_o = [slice(None)] * a.ndim
    idx_e[axis] = slice(0, 2 * n, 2)
    idx_o[axis] = slice(1, 2 * n, 2)
    out[tuple(idx_e)] = even
    out[tuple(idx_o)] = odd
    lo = 1 if skip[0] else 0
    hi = 2 * n - (1 if skip[1] else 0)
    sl = [slice(None)] * a.ndim
    sl[axis] = slice(lo, hi)
    return out[tuple(sl)]


def restrict(a_xg, nn, pad_cd, pbc_c, phase_cd=None):
    """bmgs_restrict (c/bmgs/restrict.c:136-155) after bc padding."""
    k = 2 * nn
    b = pad_bc(a_xg, pad_cd, pbc_c, phase_cd)
    nd = b.ndim
    for ax in (nd - 1, nd - 2, nd - 3):
        b = _restrict_1d(b, ax, k)
    return b


def interpolate(a_xg, nn, pad_cd, skip_cd, pbc_c, phase_cd=None):
    """bmgs_interpolate (c/bmgs/interpolate.c:227-257) after bc padding."""
    k = 2 * nn
    b = pad_bc(a_xg, pad_cd, pbc_c, phase_cd)
    nd = b.ndim
    for c, ax in ((2, nd - 1), (1, nd - 2), (0, nd - 3)):
        b = _interpolate_1d(b, ax, k, skip_cd[c])
    return b


# ------------------------------------------------------------------ grids
class Grid:
    """Single-domain geometry (gpaw/grid_descriptor.py:129-157)."""

    def __init__(self, N_c, cell_cv, pbc_c):
        self.N_c = np.array(N_c, int)
        cell = np.array(cell_cv, float)
        self.cell_cv = np.diag(cell) if cell.ndim == 1 else cell
        self.pbc_c = np.array(pbc_c, bool)
        self.beg_c = np.where(self.pbc_c, 0, 1)
        self.end_c = self.N_c.copy()
        self.n_c = self.end_c - self.beg_c
        self.h_cv = self.cell_cv / self.N_c[:, None]
        self.dv = abs(np.linalg.det(self.cell_cv)) / self.N_c.prod()

    def coarsen(self):
        return Grid(self.N_c // 2, self.cell_cv, self.pbc_c)


class Transformer:
    def __init__(self, gdin: Grid, gdout: Grid, nn=1):
        self.restrict = (gdin.N_c == 2 * gdout.N_c).all()
        self.nn = nn
        self.pbc_c = gdin.pbc_c
        self.pad, self.npad, self.skip = transformer_geometry(
            gdin.beg_c, gdin.end_c, gdout.beg_c, gdout.end_c, nn,
            self.restrict)

    def apply(self, a, phase_cd=None):
        if self.restrict:
            return restrict(a, self.nn, self.pad, self.pbc_c, phase_cd)
        return interpolate(a, self.nn, self.pad, self.skip, self.pbc_c,
                           phase_cd)


# Chelikowsky et al., Phys. Rev. B 50, 11355 (1994), central differences
# (the table of gpaw/fd_operators.py:21-33), as exact rationals.
LAPLACE = [[Fraction(0)],
           [Fraction(-2), Fraction(1)],
           [Fraction(-5, 2), Fraction(4, 3), Fraction(-1, 12)],
           [Fraction(-49, 18), Fraction(3, 2), Fraction(-3, 20), Fraction(1, 90)],
           [Fraction(-205, 72), Fraction(8, 5), Fraction(-1, 5), Fraction(8, 315),
            Fraction(-1, 560)],
           [Fraction(-5269, 1800), Fraction(5, 3), Fraction(-5, 21),
            Fraction(5, 126), Fraction(-5, 1008), Fraction(1, 3150)],
           [Fraction(-5369, 1800), Fraction(12, 7), Fraction(-15, 56),
            Fraction(10, 189), Fraction(-1, 112), Fraction(2, 1925),
            Fraction(-1, 16632)]]
DERIVATIVES = [[Fraction(1, 2)],
               [Fraction(2, 3), Fraction(-1, 12)],
               [Fraction(3, 4), Fraction(-3, 20), Fraction(1, 60)],
               [Fraction(4, 5), Fraction(-1, 5), Fraction(4, 105), Fraction(-1, 280)]]


def guc_laplace(h_cv, scale, n):
    """(coefs, offsets) of GUCLaplace (gpaw/fd_operators.py:192-228): least
    squares over the 3..6 shortest lattice directions, centre first, then per
    direction offsets +1..+n followed by -1..-n."""
    table = [float(x) for x in LAPLACE[n]]
    h_cv = np.asarray(h_cv, float)
    M_ic = np.indices((3, 3, 3)).reshape((3, -3)).T[-13:] - 1
    u_cv = h_cv / (h_cv**2).sum(1)[:, np.newaxis]**0.5
    u2_i = (np.dot(M_ic, u_cv)**2).sum(1)
    i_d = u2_i.argsort()
    m_mv = np.array([(2, 0, 0), (0, 2, 0), (0, 0, 2),
                     (0, 1, 1), (1, 0, 1), (1, 1, 0)])
    for D in range(3, 7):
        h_dv = np.dot(M_ic[i_d[:D]], h_cv)
        A_md = (h_dv**m_mv[:, np.newaxis, :]).prod(2)
        a_d, residual, rank, s = np.linalg.lstsq(A_md, [1, 1, 1, 0, 0, 0],
                                                 rcond=-1)
        if residual.sum() < 1e-14:
            break
    a_d *= scale
    offsets = [(0, 0, 0)]
    coefs = [table[0] * a_d.sum()]
    for d in range(D):
        M_c = M_ic[i_d[d]]
        offsets.extend(np.arange(1, n + 1)[:, np.newaxis] * M_c)
        coefs.extend(a_d[d] * np.array(table[1:]))
        offsets.extend(np.arange(-1, -n - 1, -1)[:, np.newaxis] * M_c)
        coefs.extend(a_d[d] * np.array(table[1:]))
    return np.array(coefs), np.array(offsets).reshape(-1, 3)


def ortho_gradient(h_cv, v, scale, n):
    """(coefs, offsets) of Gradient(v) for an orthorhombic cell: offsets
    +1..+n along axis v with weights d_k/h, then -1..-n with -d_k/h
    (gpaw/fd_operators.py:289-303 with one Voronoi neighbour per axis)."""
    h = float(np.asarray(h_cv)[v, v])
    d = np.array([float(x) for x in DERIVATIVES[n - 1]]) * scale / h
    offsets, coefs = [], []
    e = np.zeros(3, int)
    e[v] = 1
    offsets.extend(np.arange(1, n + 1)[:, None] * e)
    coefs.extend(d)
    offsets.extend(np.arange(-1, -n - 1, -1)[:, None] * e)
    coefs.extend(-d)
    return np.array(coefs), np.array(offsets).reshape(-1, 3)


def precondition(R_xg, gd0: Grid, kin0, step, phase_cd=None):
    """3-level V-cycle of gpaw/preconditioner.py:74-93 (identical sequence
    to c/fd_preconditioner.c:207-348); kin0 = (coefs, offsets) of the fine
    kinetic operator, coarse levels use Laplace(scale=-0.5, n=1) and the
    transformers use nn=1."""
    gd1 = gd0.coarsen()
    gd2 = gd1.coarsen()
    kin1 = guc_laplace(gd1.h_cv, -0.5, 1)
    kin2 = guc_laplace(gd2.h_cv, -0.5, 1)
    r0 = Transformer(gd0, gd1, 1)
    r1_ = Transformer(gd1, gd2, 1)
    i2 = Transformer(gd2, gd1, 1)
    i1 = Transformer(gd1, gd0, 1)
    pbc = gd0.pbc_c
    R = np.asarray(R_xg)
    r1 = r0.apply(-R, phase_cd)
    d1 = 4 * step * r1
    q1 = fd_apply(*kin1, d1, pbc, phase_cd) - r1
    r2 = r1_.apply(q1, phase_cd)
    d2 = 16 * step * r2
    q2 = fd_apply(*kin2, d2, pbc, phase_cd) - r2
    d2 = d2 - 16 * step * q2
    q1 = i2.apply(d2, phase_cd)
    d1 = d1 - q1
    q1 = fd_apply(*kin1, d1, pbc, phase_cd) - r1
    d1 = d1 - 4 * step * q1
    d0 = i1.apply(-d1, phase_cd)
    q0 = fd_apply(*kin0, d0, pbc, phase_cd) - R
    d0 = d0 - step * q0
    return -d0
