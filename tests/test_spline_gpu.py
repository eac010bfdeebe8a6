"""spline_to_grid and the LFC derivative through the C ABI with the
reference's arguments (rows a5 / b: _gpaw.spline_to_grid, c/lfc.c:887-977;
LFC.derivative, c/lfc.c:1449-1601).

CPU: the box rule of gpaw_b200.grid_descriptor.get_boxes against the
oracle's restatement of gpaw/grid_descriptor.py:344-411, and the host
tabulation (CPU grid descriptors) against the reference's tables
(tests/golden/spline_to_grid.npz, made by _gpaw.spline_to_grid).
GPU: gb_spline_to_grid against the same golden tables -- identical runs and
values to the last bit -- on zero, periodic, mixed and fcc grids, l = 0, 1, 2;
gb_lfc_derivative on an object built with the reference's own per-function
volumes (arguments exactly as gpaw/lfc.py:680-682 passes them) against the
live reference _gpaw.LFC.derivative, real and Bloch (1e-12)."""
import ctypes
import sys

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import ref

sys.path.insert(0, str(GOLDEN))


# the cases of tests/golden/make_golden.py (spline set)
SPLINE_CASES = {
    'zero_l0': ((20, 22, 24), np.diag([5.0, 5.5, 6.0]), (0, 0, 0), (0.5, 0.45, 0.52), 0, 2.3, 40),
    'periodic_l1': ((20, 20, 24), np.diag([5.0, 5.0, 6.0]), (1, 1, 1), (0.05, 0.9, 0.5), 1, 2.6, 52),
    'mixed_l2': ((18, 20, 22), np.diag([4.5, 5.0, 5.5]), (0, 1, 1), (0.3, 0.02, 0.97), 2, 2.2, 30),
    'fcc_l2': ((16, 16, 16), np.array([[0, 3.4, 3.4], [3.4, 0, 3.4], [3.4, 3.4, 0]]),
               (1, 1, 1), (0.1, 0.3, 0.6), 2, 2.0, 25),
}


def radial(rmax, nbins):
    f = np.exp(-(np.linspace(0, rmax, nbins + 1) / (0.4 * rmax))**2)
    f[-1] = 0.0
    return f


@pytest.fixture(scope='module')
def golden():
    with np.load(GOLDEN / 'spline_to_grid.npz') as f:
        return {k: f[k] for k in f.files}


def _boxes(name):
    from oracle.scf import Grid, boxes
    N_c, cell, pbc, spos, l, rmax, nbins = SPLINE_CASES[name]
    g = Grid(N_c, cell, pbc)
    return g, boxes(g, np.array(spos), rmax)


@pytest.mark.parametrize('name', sorted(SPLINE_CASES))
def test_box_rule_matches_oracle(name):
    from gpaw_b200.grid_descriptor import GridDescriptor
    N_c, cell, pbc, spos, l, rmax, nbins = SPLINE_CASES[name]
    gd = GridDescriptor(N_c, cell, pbc, device='cpu')
    mine = gd.get_boxes(np.array(spos), rmax, True)
    _, theirs = _boxes(name)
    assert len(mine) == len(theirs)
    for (b1, e1, d1), (b2, e2, d2) in zip(mine, theirs):
        assert np.array_equal(b1, b2) and np.array_equal(e1, e2) and np.allclose(d1, d2)


@pytest.mark.parametrize('name', sorted(SPLINE_CASES))
def test_host_tables_match_reference(golden, name):
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.lfc import _box_functions
    from gpaw_b200.spline import Spline
    N_c, cell, pbc, spos, l, rmax, nbins = SPLINE_CASES[name]
    gd = GridDescriptor(N_c, cell, pbc, device='cpu')
    s = Spline.from_data(l, rmax, radial(rmax, nbins))
    g, bx = _boxes(name)
    for i, (beg, end, sdisp) in enumerate(bx):
        A, G = _box_functions(s, beg, end, (np.array(spos) - sdisp) @ g.cell_cv, gd)
        assert np.array_equal(G, golden[f'{name}|{i}|G'])
        assert np.allclose(A, golden[f'{name}|{i}|A'], rtol=1e-13, atol=1e-15)


@pytest.mark.gpu
@pytest.mark.parametrize('name', sorted(SPLINE_CASES))
def test_device_spline_to_grid_matches_reference(golden, name):
    from gpaw_b200.lfc import spline_to_grid
    from gpaw_b200.spline import Spline
    N_c, cell, pbc, spos, l, rmax, nbins = SPLINE_CASES[name]
    s = Spline.from_data(l, rmax, radial(rmax, nbins))
    g, bx = _boxes(name)
    assert bx
    for i, (beg, end, sdisp) in enumerate(bx):
        A, G = spline_to_grid(s, beg, end, (np.array(spos) - sdisp) @ g.cell_cv, g.h_cv,
                              g.n_c, g.beg_c)
        assert np.array_equal(G, golden[f'{name}|{i}|G'])
        A = A.cpu().numpy()
        want = golden[f'{name}|{i}|A']
        assert A.shape == want.shape
        assert np.abs(A - want).max() <= 1e-15 * np.abs(want).max()


@pytest.mark.gpu
@pytest.mark.skipif(not ref.available(), reason='oracle/_ref not built')
@pytest.mark.parametrize('bloch', [False, True])
def test_derivative_with_the_reference_arguments(bloch):
    """An object built from the reference's per-function volumes
    (_gpaw.spline_to_grid boxes, gpaw/lfc.py:259-374 ordering) and
    gb_lfc_derivative called with the arguments gpaw/lfc.py:680-682 passes
    to _gpaw.LFC.derivative."""
    import torch
    from gpaw_b200 import _native as nat
    from gpaw_b200.lfc import _Native
    from gpaw_b200.spline import Spline
    from oracle.scf import Grid, boxes
    gp = ref.load()
    g = Grid((18, 20, 16), np.diag([4.5, 5.0, 4.0]), (1, 1, 1))
    spos_ac = np.array([[0.1, 0.85, 0.5], [0.55, 0.3, 0.05]])
    funcs = [[(0, 2.0, 30), (1, 2.2, 33)], [(2, 1.9, 28), (0, 1.7, 25)]]
    k_c = np.array([0.25, -0.125, 0.5])
    A_W, M_W, G_l, W_l, pos_W, sdisp_W, spl_M_ref, spl_M_dev = [], [], [], [], [], [], [], []
    keep = []
    W = 0
    M = 0
    for a, fl in enumerate(funcs):
        for (l, rmax, nbins) in fl:
            f = radial(rmax, nbins)
            rs = gp.Spline(l, rmax, f)
            ds = Spline.from_data(l, rmax, f)
            keep += [rs, ds]
            for beg, end, sdisp in boxes(g, spos_ac[a], rmax):
                pos_v = (spos_ac[a] - sdisp) @ g.cell_cv
                A_gm, G_b = gp.spline_to_grid(rs, beg, end, pos_v, np.ascontiguousarray(g.h_cv),
                                              g.n_c, g.beg_c)
                if len(G_b) == 0:
                    continue
                A_W.append(A_gm)
                M_W.append(M)
                G_l.append(G_b)
                w = np.empty(len(G_b), np.intc)
                w[0::2] = W
                w[1::2] = -W - 1
                W_l.append(w)
                pos_W.append(pos_v)
                sdisp_W.append(sdisp)
                W += 1
            spl_M_ref += [rs] * (2 * l + 1)
            spl_M_dev += [ds] * (2 * l + 1)
            M += 2 * l + 1
    G_B = np.concatenate(G_l)
    W_B = np.concatenate(W_l)
    order = np.argsort(G_B, kind='mergesort')
    G_B = np.ascontiguousarray(G_B[order], np.intc)
    W_B = np.ascontiguousarray(W_B[order], np.intc)
    M_W = np.array(M_W, np.intc)
    if bloch:
        phase_qW = np.exp(2j * np.pi * np.inner(k_c[None], np.array(sdisp_W)))
    else:
        phase_qW = np.empty((0, W), complex)
    pos_Wv = np.ascontiguousarray(pos_W, float)
    rlfc = gp.LFC(A_W, M_W, G_B, W_B, g.dv, phase_qW)
    rng = np.random.default_rng(4)
    nx = 3
    a_xG = rng.standard_normal((nx,) + tuple(g.n_c))
    if bloch:
        a_xG = a_xG + 1j * rng.standard_normal(a_xG.shape)
    want = np.zeros((nx, M, 3), a_xG.dtype)
    rlfc.derivative(a_xG, want, np.ascontiguousarray(g.h_cv), g.n_c, spl_M_ref, g.beg_c,
                    pos_Wv, 0 if bloch else -1)
    dev = _Native(A_W, M_W, G_B, W_B, g.dv, phase_qW, int(np.prod(g.n_c)), M)
    a = torch.from_numpy(a_xG).cuda()
    c = torch.zeros((nx, M, 3), dtype=a.dtype, device='cuda')
    handles = (ctypes.c_void_p * M)(*[s.handle.value for s in spl_M_dev])
    nat.check(nat.lib().gb_lfc_derivative(
        dev.handle, nat.ptr(a), nat.ptr(c), nx, nat.f64(np.ascontiguousarray(g.h_cv)),
        nat.i64(g.n_c), handles, nat.i64(g.beg_c), nat.f64(pos_Wv), 0 if bloch else -1,
        nat.dtype_code(a), nat.stream_of(a)), 'gb_lfc_derivative')
    got = c.cpu().numpy()
    assert np.abs(got - want).max() < 1e-12 * np.abs(want).max()
