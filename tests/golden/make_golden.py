"""Generate the golden vectors under tests/golden/ from the reference itself.

Run where the reference source tree is present, with REF naming its root
and GPAW's C extension built from it by oracle/Makefile:

    make -C oracle REF=<root> && REF=<root> python tests/golden/make_golden.py [sets]

Outputs (committed; read by the CPU and GPU tests, which never need the
reference tree at run time):
  stencils.json  coefficient / offset lists of the reference's
                 gpaw.fd_operators.Laplace / Gradient for a set of cells
  fd_kernels.npz outputs of _gpaw.Operator / Transformer / fd_precond on
                 seeded inputs (numpy default_rng(seed).standard_normal, so
                 inputs are regenerated from the seed, not stored)
  xc.npz         _gpaw.XCFunctional outputs (LDA, PBE, revPBE, RPBE)
  lfc.npz        _gpaw.spline_to_grid / LFC add, integrate, derivative
  density.npz    _gpaw.add_to_density accumulations
  spline_to_grid.npz  _gpaw.spline_to_grid tables and runs, box by box
"""
from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
REF = os.environ.get('REF')
if not REF:
    sys.exit('make_golden.py: set REF to the root of the reference source tree')
sys.path.insert(0, str(REPO / 'oracle' / '_ref'))
sys.path.insert(1, REF)
sys.path.insert(2, str(REPO))
sys.path.insert(3, str(HERE))

import _gpaw  # noqa: E402  (the reference C extension built from source)
import gpaw.fd_operators as ref_fd  # noqa: E402
from oracle import ref as oref  # noqa: E402
from oracle.fd import transformer_geometry  # noqa: E402

from cells import CELLS  # noqa: E402


class StubComm:
    size = 1
    rank = 0

    def get_c_object(self):
        return None


class StubGD:
    """The attributes gpaw.fd_operators reads from a GridDescriptor."""

    def __init__(self, N_c, cell, pbc):
        cell = np.array(cell, float)
        self.cell_cv = np.diag(cell) if cell.ndim == 1 else cell
        self.N_c = np.array(N_c)
        self.pbc_c = np.array(pbc, bool)
        self.beg_c = np.where(self.pbc_c, 0, 1)
        self.n_c = self.N_c - self.beg_c
        self.h_cv = self.cell_cv / self.N_c[:, None]
        self.neighbor_cd = np.ascontiguousarray(
            np.where(self.pbc_c[:, None], 0, -1) * np.ones((3, 2), int))
        self.comm = StubComm()


def stencils():
    out = {}
    for name, cell in CELLS.items():
        gd = StubGD((12, 12, 12), cell, (1, 1, 1))
        for n in (1, 2, 3, 4):
            lap = ref_fd.Laplace(gd, -0.5, n)
            out[f'laplace/{name}/{n}'] = {
                'coef': lap.coef_p.tolist(),
                'offset': np.asarray(lap.offset_pc).tolist()}
            for v in range(3):
                g = ref_fd.Gradient(gd, v, 1.0, n)
                out[f'gradient/{name}/{n}/{v}'] = {
                    'coef': np.asarray(g.coef_p).tolist(),
                    'offset': np.asarray(g.offset_pc).tolist()}
    return out


def phases(pbc, k_c):
    sd = np.zeros((3, 2))
    p = np.asarray(pbc, bool)
    sd[p, 0] = 1
    sd[p, 1] = -1
    return np.exp(2j * np.pi * sd * np.asarray(k_c)[:, None])


def seeded(seed, shape, cplx):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(shape)
    if cplx:
        a = a + 1j * rng.standard_normal(shape)
    return a


K_C = (0.1, 0.25, -0.3)
N_KERNEL = (6, 7, 8)


def kernels(sten):
    res = {}
    seed = 100
    # stencils: orthorhombic Laplace nn=1..3, GUC (hexagonal, fcc) n=2, gradients
    cases = [('laplace/ortho/3', 'ortho'), ('laplace/ortho/1', 'ortho'),
             ('laplace/ortho/2', 'ortho'), ('laplace/hexagonal/2', 'hexagonal'),
             ('laplace/fcc/2', 'fcc'), ('gradient/ortho/3/0', 'ortho'),
             ('gradient/ortho/3/2', 'ortho'), ('gradient/hexagonal/2/1', 'hexagonal')]
    for key, _ in cases:
        st = sten[key]
        for pbc in ((0, 0, 0), (1, 1, 1), (1, 0, 1)):
            for cplx in (False, True):
                seed += 1
                n_c = np.array(N_KERNEL) - (1 - np.array(pbc))
                a = seeded(seed, (1,) + tuple(n_c), cplx)
                op = oref.operator(st['coef'], st['offset'], n_c, pbc, not cplx)
                b = np.zeros_like(a)
                if cplx:
                    op.apply(a, b, phases(pbc, K_C))
                else:
                    op.apply(a, b)
                res[f'op|{key}|{"".join(map(str, pbc))}|{int(cplx)}|{seed}'] = b
    # transformers: restrict / interpolate, k = 2..8
    # (grids large enough for the reference's own "Cannot construct
    # interpolator" rule, gpaw/transformers.py:49-55; smaller ones are invalid)
    for pbc in ((0, 0, 0), (1, 1, 1)):
        N = np.array((16, 16, 20))
        beg_f = np.where(pbc, 0, 1)
        for nn in (1, 2, 3, 4):
            for cplx in ((False, True) if nn in (1, 3) else (False,)):
                for restrict in (True, False):
                    seed += 1
                    Nin = N if restrict else N // 2
                    Nout = N // 2 if restrict else N
                    beg_in = beg_f
                    beg_out = beg_f
                    pad, npad, skip = transformer_geometry(
                        beg_in, Nin, beg_out, Nout, nn, restrict)
                    n_in = Nin - beg_in
                    n_out = Nout - beg_out
                    t = oref.transformer(n_in, n_out, nn, pad, npad, skip, pbc,
                                         not cplx, not restrict)
                    a = seeded(seed, (1,) + tuple(n_in), cplx)
                    b = np.zeros((1,) + tuple(n_out), a.dtype)
                    if cplx:
                        t.apply(a, b, phases(pbc, K_C))
                    else:
                        t.apply(a, b)
                    res[f'tr|{"".join(map(str, pbc))}|{nn}|{int(cplx)}|'
                        f'{"R" if restrict else "I"}|{seed}'] = b
    # multigrid preconditioner
    for pbc, cplx in (((0, 0, 0), False), ((1, 1, 1), False), ((1, 1, 1), True)):
        seed += 1
        N0 = np.array((12, 12, 16))
        cell = np.array([3.2, 3.2, 4.0])
        gds = [StubGD(N0 // 2**lvl, cell, pbc) for lvl in range(3)]
        kin = [ref_fd.Laplace(gds[0], -0.5, 3, float if not cplx else complex)]
        kin += [ref_fd.Laplace(g, -0.5, 1, float if not cplx else complex) for g in gds[1:]]
        ops = [k.operator for k in kin]

        def T(gi, go):
            r = (gi.N_c == 2 * go.N_c).all()
            pad, npad, skip = transformer_geometry(gi.beg_c, gi.N_c, go.beg_c, go.N_c, 1, r)
            return oref.transformer(gi.n_c, go.n_c, 1, pad, npad, skip, pbc, not cplx, not r)

        rest0, rest1 = T(gds[0], gds[1]), T(gds[1], gds[2])
        intp2, intp1 = T(gds[2], gds[1]), T(gds[1], gds[0])
        B = 2
        dt = complex if cplx else float
        R = seeded(seed, (B,) + tuple(gds[0].n_c), cplx).astype(dt)
        d0 = np.zeros_like(R)
        q0 = np.zeros_like(R)
        w1 = [np.zeros((B,) + tuple(gds[1].n_c), dt) for _ in range(3)]
        w2 = [np.zeros((B,) + tuple(gds[2].n_c), dt) for _ in range(3)]
        step = 0.66666666 / kin[0].get_diagonal_element()
        _gpaw.fd_precond(rest0, rest1, intp1, intp2, *ops, d0, q0, *w1, *w2,
                         R, -R, step, phases(pbc, K_C))
        res[f'pc|{"".join(map(str, pbc))}|{int(cplx)}|{seed}'] = d0
    return res


def xc_golden():
    from oracle.xc import log_uniform_inputs
    res = {}
    for code in (-1, 0, 1, 2):
        for nspins in (1, 2):
            n_sg, sigma_xg = log_uniform_inputs(1000 + 10 * code + nspins, nspins, 1000)
            e_g = np.zeros(n_sg.shape[1])
            v_sg = np.zeros_like(n_sg)
            dedsigma_xg = np.zeros_like(sigma_xg)
            X = _gpaw.XCFunctional(code)
            if code == -1:
                X.calculate(e_g, n_sg, v_sg)
            else:
                X.calculate(e_g, n_sg, v_sg, sigma_xg, dedsigma_xg)
            key = f'{code}|{nspins}'
            res[f'e|{key}'] = e_g
            res[f'v|{key}'] = v_sg
            if code != -1:
                res[f'dedsigma|{key}'] = dedsigma_xg
    return res


# ---------------------------------------------------------------- LFC
from lfc_cases import LFC_CASES  # noqa: E402


def lfc_golden():
    """Reference-built LFC data: _gpaw.spline_to_grid for every box of
    gd.get_boxes (restated from gpaw/grid_descriptor.py:344-411 in
    gpaw_b200.grid_descriptor), the boundary sort of gpaw/lfc.py:330-344 and
    _gpaw.LFC add / integrate / derivative on seeded coefficients."""
    sys.path.insert(0, str(REPO))
    from gpaw_b200.grid_descriptor import GridDescriptor
    res = {}
    for name, (N_c, cell, pbc, spos_ac, spl, k_c) in LFC_CASES.items():
        gd = GridDescriptor(N_c, cell, pbc, device='cpu')
        rs = [[_gpaw.Spline(l, rmax, np.append(np.array(f, float)[:-1], 0.0))   # Spline.from_data
               for (l, rmax, f) in sj] for sj in spl]
        A_W, M_W, G_l, W_l, sdisp_W, pos_W, spl_M = [], [], [], [], [], [], []
        W = 0
        Ma = 0
        for a, sj in enumerate(rs):
            M = 0
            for s in sj:
                l = s.get_angular_momentum_number()
                for beg, end, sdisp in gd.get_boxes(np.array(spos_ac[a]), s.get_cutoff(), True):
                    pos_v = np.dot(np.array(spos_ac[a]) - sdisp, gd.cell_cv)
                    A_gm, G_b = _gpaw.spline_to_grid(s, beg, end, pos_v,
                                                     np.ascontiguousarray(gd.h_cv), gd.n_c, gd.beg_c)
                    if len(G_b) == 0:
                        continue
                    A_W.append(A_gm)
                    M_W.append(Ma + M)
                    G_l.append(G_b)
                    w = np.empty(len(G_b), np.intc)
                    w[0::2] = W
                    w[1::2] = -W - 1
                    W_l.append(w)
                    sdisp_W.append(sdisp)
                    pos_W.append(pos_v)
                    W += 1
                M += 2 * l + 1
                spl_M.extend([s] * (2 * l + 1))
            Ma += M
        Mmax = Ma
        G_B = np.concatenate(G_l)
        W_B = np.concatenate(W_l)
        idx = np.argsort(G_B, kind='mergesort')
        G_B = np.ascontiguousarray(G_B[idx], np.intc)
        W_B = np.ascontiguousarray(W_B[idx], np.intc)
        M_W = np.array(M_W, np.intc)
        cplx = k_c is not None
        if cplx:
            phase_qW = np.exp(2j * np.pi * np.inner(np.array([k_c]), np.array(sdisp_W)))
        else:
            phase_qW = np.empty((0, W), complex)
        lfc = _gpaw.LFC(A_W, M_W, G_B, W_B, gd.dv, phase_qW)
        rng = np.random.default_rng(7)
        nx = 2
        c_xM = rng.standard_normal((nx, Mmax))
        a_xG = rng.standard_normal((nx,) + tuple(gd.n_c))
        if cplx:
            c_xM = c_xM + 1j * rng.standard_normal(c_xM.shape)
            a_xG = a_xG + 1j * rng.standard_normal(a_xG.shape)
        q = 0 if cplx else -1
        b_xG = np.zeros_like(a_xG)
        lfc.add(c_xM, b_xG, q)
        i_xM = np.zeros_like(c_xM)
        lfc.integrate(a_xG, i_xM, q)
        d_xMv = np.zeros(c_xM.shape + (3,), c_xM.dtype)
        lfc.derivative(a_xG, d_xMv, np.ascontiguousarray(gd.h_cv), gd.n_c, spl_M, gd.beg_c,
                       np.array(pos_W), q)
        res[f'{name}|add'] = b_xG
        res[f'{name}|integrate'] = i_xM
        res[f'{name}|derivative'] = d_xMv
    return res


# ---------------------------------------------------------------- density
DENSITY_CASES = {
    # name: (grid, bands, complex)
    'real_4x31': ((31, 31, 31), 4, False),
    'real_7x12x10x14': ((12, 10, 14), 7, False),
    'complex_5x16': ((16, 16, 16), 5, True),
}


def density_golden():
    """_gpaw.add_to_density (c/utilities.c:313-352) accumulated band by band
    with occupations f_n = 2, 1.5, 1, ... as gpaw/wavefunctions/fd.py:95-100
    calls it, on seeded wave functions (seed 3, regenerated by the tests)."""
    res = {}
    for name, (n_c, nb, cplx) in DENSITY_CASES.items():
        rng = np.random.default_rng(3)
        psit = rng.standard_normal((nb,) + n_c)
        if cplx:
            psit = psit + 1j * rng.standard_normal(psit.shape)
        nt = np.full(n_c, 0.25)
        f_n = 2.0 - 0.5 * np.arange(nb)
        for f, psit_G in zip(f_n, psit):
            _gpaw.add_to_density(float(f), np.ascontiguousarray(psit_G), nt)
        res[name] = nt
    return res


# ---------------------------------------------------------------- splines
SPLINE_CASES = {
    # name: (N_c, cell_cv (Bohr), pbc, spos_c, l, rmax, nbins)
    'zero_l0': ((20, 22, 24), np.diag([5.0, 5.5, 6.0]), (0, 0, 0), (0.5, 0.45, 0.52), 0, 2.3, 40),
    'periodic_l1': ((20, 20, 24), np.diag([5.0, 5.0, 6.0]), (1, 1, 1), (0.05, 0.9, 0.5), 1, 2.6, 52),
    'mixed_l2': ((18, 20, 22), np.diag([4.5, 5.0, 5.5]), (0, 1, 1), (0.3, 0.02, 0.97), 2, 2.2, 30),
    'fcc_l2': ((16, 16, 16), np.array([[0, 3.4, 3.4], [3.4, 0, 3.4], [3.4, 3.4, 0]]),
               (1, 1, 1), (0.1, 0.3, 0.6), 2, 2.0, 25),
}


def spline_radial(rmax, nbins):
    f = np.exp(-(np.linspace(0, rmax, nbins + 1) / (0.4 * rmax))**2)
    f[-1] = 0.0
    return f


def spline_golden():
    """_gpaw.spline_to_grid (c/lfc.c:887-977) on every box
    (gpaw/grid_descriptor.py:344-411) of one atom per case."""
    sys.path.insert(0, str(REPO))
    from oracle.scf import Grid, boxes
    res = {}
    for name, (N_c, cell_cv, pbc, spos, l, rmax, nbins) in SPLINE_CASES.items():
        g = Grid(N_c, cell_cv, pbc)
        s = _gpaw.Spline(l, rmax, spline_radial(rmax, nbins))
        for i, (beg, end, sdisp) in enumerate(boxes(g, np.array(spos), rmax)):
            pos_v = (np.array(spos) - sdisp) @ g.cell_cv
            A_gm, G_b = _gpaw.spline_to_grid(s, beg, end, pos_v, np.ascontiguousarray(g.h_cv),
                                             g.n_c, g.beg_c)
            res[f'{name}|{i}|A'] = A_gm
            res[f'{name}|{i}|G'] = G_b
    return res


def main(which):
    if 'xc' in which:
        np.savez_compressed(HERE / 'xc.npz', **xc_golden())
    if 'kernels' in which:
        sten = stencils()
        (HERE / 'stencils.json').write_text(json.dumps(sten))
        res = kernels(sten)
        np.savez_compressed(HERE / 'fd_kernels.npz', **res)
        print(f'{len(sten)} stencils, {len(res)} kernel outputs')
    if 'lfc' in which:
        np.savez_compressed(HERE / 'lfc.npz', **lfc_golden())
    if 'density' in which:
        np.savez_compressed(HERE / 'density.npz', **density_golden())
    if 'spline' in which:
        np.savez_compressed(HERE / 'spline_to_grid.npz', **spline_golden())


if __name__ == '__main__':
    # python make_golden.py [xc] [kernels] [lfc] [density] [spline]  (default: all)
    main(set(sys.argv[1:]) or {'xc', 'kernels', 'lfc', 'density', 'spline'})
