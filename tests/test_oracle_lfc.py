"""Pin the LFC oracle (oracle/lfc.py) and the host-side sphere construction
of gpaw_b200.lfc against the reference's own C (spline_to_grid, LFC) through
golden vectors (tests/golden/lfc.npz) and, when oracle/_ref is built, live."""
import sys

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import lfc as ol
from oracle import ref

sys.path.insert(0, str(GOLDEN))


def cases():
    import importlib.util
    spec = importlib.util.spec_from_file_location('lfc_cases', GOLDEN / 'lfc_cases.py')
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m.LFC_CASES


def oracle_outputs(name):
    N_c, cell, pbc, spos, spl, k = cases()[name]
    Phi = ol.dense_functions(N_c, cell, pbc, spos, spl, k)
    dPhi = ol.dense_functions(N_c, cell, pbc, spos, spl, k, derivative=True)
    beg = np.where(np.array(pbc, bool), 0, 1)
    n_c = np.array(N_c) - beg
    dv = np.prod(cell) / np.prod(N_c)
    rng = np.random.default_rng(7)
    nx, Mmax = 2, Phi.shape[0]
    c = rng.standard_normal((nx, Mmax))
    a = rng.standard_normal((nx,) + tuple(n_c))
    if k is not None:
        c = c + 1j * rng.standard_normal(c.shape)
        a = a + 1j * rng.standard_normal(a.shape)
    b = ol.add(np.zeros_like(a), c, Phi)
    i = ol.integrate(a, Phi, dv)
    d = ol.integrate(a, dPhi.reshape(-1, dPhi.shape[-1]), dv).reshape(nx, Mmax, 3)
    return (c, a), (b, i, d)


@pytest.mark.parametrize('name', ['zero', 'periodic', 'bloch'])
def test_oracle_lfc_matches_golden(name):
    g = np.load(GOLDEN / 'lfc.npz')
    _, (b, i, d) = oracle_outputs(name)
    r = lambda x, y: np.abs(x - y).max() / np.abs(y).max()
    assert r(b, g[f'{name}|add']) < 1e-13
    assert r(i, g[f'{name}|integrate']) < 1e-13
    assert r(d, g[f'{name}|derivative']) < 1e-12


@pytest.mark.skipif(not ref.available(), reason='oracle/_ref not built')
def test_host_box_functions_match_spline_to_grid():
    """gpaw_b200.lfc._box_functions == _gpaw.spline_to_grid (values, order
    and z-runs) for l = 0, 1, 2 on zero and periodic grids."""
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.lfc import _box_functions
    from gpaw_b200.spline import Spline
    g = ref.load()
    f = np.exp(-np.linspace(0, 2.3, 24)**2)
    f[-1] = 0.0   # gpaw/spline.py:30 (Spline.from_data)
    for pbc in ((0, 0, 0), (1, 1, 1), (0, 1, 1)):
        gd = GridDescriptor((18, 20, 22), (4.5, 5.0, 5.5), pbc, device='cpu')
        for l in (0, 1, 2):
            rs = g.Spline(l, 2.3, np.array(f))
            ps = Spline.from_data(l, 2.3, f)
            spos = np.array([0.13, 0.52, 0.91])
            for beg, end, sdisp in gd.get_boxes(spos, 2.3, True):
                pos_v = (spos - sdisp) @ gd.cell_cv
                A1, G1 = g.spline_to_grid(rs, beg, end, pos_v, np.ascontiguousarray(gd.h_cv),
                                          gd.n_c, gd.beg_c)
                A2, G2 = _box_functions(ps, beg, end, pos_v, gd)
                assert np.array_equal(G1, G2)
                assert np.allclose(A1, A2, rtol=1e-13, atol=1e-15)
