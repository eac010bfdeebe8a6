"""Pin the oracle (oracle/fd.py) before trusting it:
  * against golden vectors made by the reference itself (tests/golden/),
  * against the reference's own known-answer tests
    (gpaw/test/fd_ops/test_gradient.py, test_laplace.py,
     test_transformations.py, test_non_periodic.py),
  * against the live reference C extension when oracle/_ref is built.
All CPU-only."""
import numpy as np
import pytest

from conftest import seeded, bloch_phases, relerr
from oracle import fd, ref

N_KERNEL = (6, 7, 8)


def _op_cases(golden_kernels):
    for key, out in golden_kernels.items():
        if key.startswith('op|'):
            _, st, pbc, cplx, seed = key.split('|')
            yield st, tuple(int(c) for c in pbc), bool(int(cplx)), int(seed), out


def test_oracle_stencil_matches_golden(golden_kernels, golden_stencils):
    n = 0
    for st, pbc, cplx, seed, out in _op_cases(golden_kernels):
        s = golden_stencils[st]
        n_c = np.array(N_KERNEL) - (1 - np.array(pbc))
        a = seeded(seed, (1,) + tuple(n_c), cplx)
        got = fd.fd_apply(s['coef'], s['offset'], a, pbc,
                          bloch_phases(pbc) if cplx else None)
        assert relerr(got, out) < 1e-14, (st, pbc, cplx)
        n += 1
    assert n == 48


def test_oracle_stencil_builders_match_reference_lists(golden_stencils):
    import sys
    from conftest import GOLDEN
    sys.path.insert(0, str(GOLDEN))
    from cells import CELLS
    for key, s in golden_stencils.items():
        kind, cell, n, *v = key.split('/')
        if kind != 'laplace':
            continue
        cell_cv = np.array(CELLS[cell], float)
        cell_cv = np.diag(cell_cv) if cell_cv.ndim == 1 else cell_cv
        h_cv = cell_cv / 12
        c, o = fd.guc_laplace(h_cv, -0.5, int(n))
        assert np.array_equal(o, np.array(s['offset']))
        assert np.allclose(c, s['coef'], rtol=1e-13, atol=0)


def test_oracle_transformers_match_golden(golden_kernels):
    n = 0
    for key, out in golden_kernels.items():
        if not key.startswith('tr|'):
            continue
        _, pbc, nn, cplx, kind, seed = key.split('|')
        pbc = tuple(int(c) for c in pbc)
        nn, cplx, seed = int(nn), bool(int(cplx)), int(seed)
        N = np.array((16, 16, 20))
        gfine = fd.Grid(N, (3.0, 3.0, 3.5), pbc)
        gcoarse = gfine.coarsen()
        gi, go = (gfine, gcoarse) if kind == 'R' else (gcoarse, gfine)
        a = seeded(seed, (1,) + tuple(gi.n_c), cplx)
        got = fd.Transformer(gi, go, nn).apply(a, bloch_phases(pbc) if cplx else None)
        assert got.shape == out.shape
        assert relerr(got, out) < 1e-14, key
        n += 1
    assert n == 24


def test_oracle_precond_matches_golden(golden_kernels):
    n = 0
    for key, out in golden_kernels.items():
        if not key.startswith('pc|'):
            continue
        _, pbc, cplx, seed = key.split('|')
        pbc = tuple(int(c) for c in pbc)
        cplx, seed = bool(int(cplx)), int(seed)
        gd0 = fd.Grid((12, 12, 16), (3.2, 3.2, 4.0), pbc)
        kin0 = fd.guc_laplace(gd0.h_cv, -0.5, 3)
        R = seeded(seed, (2,) + tuple(gd0.n_c), cplx)
        step = 0.66666666 / kin0[0][0]
        got = fd.precondition(R, gd0, kin0, step, bloch_phases(pbc) if cplx else None)
        assert relerr(got, out) < 1e-13, key
        n += 1
    assert n == 3


# ---- known answers of the reference test suite --------------------------
def test_gradient_golden_vectors():
    """gpaw/test/fd_ops/test_gradient.py:17-38: d/dx of 0..7 on a periodic
    8-point line is [-3, 1, 1, 1, 1, 1, 1, -3]; the backward difference gives
    [-7, 1, ...]."""
    g = fd.Grid((8, 1, 1), (8.0, 1.0, 1.0), (1, 1, 1))
    a = np.zeros((8, 1, 1))
    a[:, 0, 0] = np.arange(8)
    c, o = fd.ortho_gradient(g.h_cv, 0, 1.0, 1)
    d = fd.fd_apply(c, o, a, (1, 1, 1))
    assert not (d[:, 0, 0] - [-3, 1, 1, 1, 1, 1, 1, -3]).any()
    d = fd.fd_apply([-1, 1], [[-1, 0, 0], [0, 0, 0]], a, (1, 1, 1))
    assert not (d[:, 0, 0] - [-7, 1, 1, 1, 1, 1, 1, 1]).any()
    # zero boundary along y: [0.5, 1, 1, 1, 1, 1, -2.5]
    g = fd.Grid((1, 8, 1), (1.0, 8.0, 1.0), (1, 0, 1))
    a = np.zeros((1, 7, 1))
    a[0, :, 0] = np.arange(1, 8) - 1
    c, o = fd.ortho_gradient(g.h_cv, 1, 1.0, 1)
    d = fd.fd_apply(c, o, a, (1, 0, 1))
    assert d[0, 0, 0] == 0.5 and np.sum(d[0, :, 0]) == 3.0


@pytest.mark.parametrize('n', [1, 2, 3, 4])
def test_laplace_polynomial_exactness(n):
    """gpaw/test/fd_ops/test_laplace.py:82-101 (orthorhombic 'sc' cell)."""
    N = 2 * n + 2
    g = fd.Grid((N, N, N), (1.1, 1.02, 1.03), (1, 1, 1))
    r = [(np.arange(N) * g.h_cv[c, c])[(slice(None),) + (None,) * (2 - c)] for c in range(3)]
    c_v = np.diag(g.cell_cv) / 2
    coefs, offs = fd.guc_laplace(g.h_cv, 1.0, n)
    for m in range(0, 2 * n + 1):
        for ix in range(m + 1):
            for iy in range(m - ix + 1):
                iz = m - ix - iy
                a = ((r[0] - c_v[0])**ix * (r[1] - c_v[1])**iy *
                     (r[2] - c_v[2])**iz) * np.ones((N, N, N))
                expect = 2.0 if (m == 2 and max(ix, iy, iz) == 2) else 0.0
                b = fd.fd_apply(coefs, offs, a, (1, 1, 1))
                assert abs(b[n + 1, n + 1, n + 1] - expect) < 2e-12


@pytest.mark.parametrize('pbc', [0, 1])
def test_transformations_conserve_integral(pbc):
    """gpaw/test/fd_ops/test_transformations.py and test_non_periodic.py."""
    n = 20
    L = 1.0 if pbc else 8.0     # the cells of the two reference tests
    g = fd.Grid((n, n, n), (L, L, L), (pbc,) * 3)
    rng = np.random.RandomState(8)
    a = rng.random(tuple(g.n_c))
    gf = fd.Grid((2 * n,) * 3, (L, L, L), (pbc,) * 3)
    gc = g.coarsen()
    tol = 1e-14 if pbc else 1e-10
    for nn in ((1, 2, 3, 4) if pbc else (1,)):
        b = fd.Transformer(g, gf, nn).apply(a)
        assert abs(a.sum() * g.dv - b.sum() * gf.dv) < tol
        if pbc:
            b = fd.Transformer(g, gc, nn).apply(a)
            assert abs(a.sum() * g.dv - b.sum() * gc.dv) < tol


@pytest.mark.skipif(not ref.available(), reason='oracle/_ref not built')
def test_oracle_matches_live_reference_random():
    rng = np.random.default_rng(5)
    for pbc in ((0, 0, 0), (1, 1, 1), (0, 1, 0)):
        for real in (True, False):
            n_c = np.array([9, 10, 11])
            coefs, offs = fd.guc_laplace(np.diag([0.3, 0.35, 0.4]), -0.5, 3)
            a = rng.standard_normal((2, *n_c))
            ph = None
            if not real:
                a = a + 1j * rng.standard_normal(a.shape)
                ph = bloch_phases(pbc)
            op = ref.operator(coefs, offs, n_c, pbc, real)
            out = np.zeros_like(a)
            op.apply(a, out) if real else op.apply(a, out, ph)
            got = fd.fd_apply(coefs, offs, a, pbc, ph)
            if real:
                assert np.array_equal(got, out)
            else:
                assert relerr(got, out) < 1e-15
