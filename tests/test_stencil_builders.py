"""CPU: the product's stencil constructions (gpaw_b200.fd_operators
laplace_stencil / gradient_stencil) against the coefficient lists the
reference's own gpaw.fd_operators.Laplace / Gradient produced for seven cells
and orders 1-4 (tests/golden/stencils.json), compared as sets of
(offset, coefficient) pairs; plus the defining identities on random cells."""
import sys

import numpy as np
import pytest

from conftest import GOLDEN
from gpaw_b200.fd_operators import gradient_stencil, laplace_stencil

sys.path.insert(0, str(GOLDEN))
from cells import CELLS  # noqa: E402


def _canonical(coef, offset):
    o = np.asarray(offset, int).reshape(-1, 3)
    idx = np.lexsort(o.T[::-1])
    return np.asarray(coef, float)[idx], o[idx]


def _h_cv(name):
    cell = np.array(CELLS[name], float)
    cell = np.diag(cell) if cell.ndim == 1 else cell
    return cell / 12


def test_builders_match_reference_lists(golden_stencils):
    n = 0
    for key, s in golden_stencils.items():
        kind, cell, order, *v = key.split('/')
        h_cv = _h_cv(cell)
        if kind == 'laplace':
            c, o = laplace_stencil(h_cv, -0.5, int(order))
        else:
            c, o = gradient_stencil(h_cv, int(v[0]), 1.0, int(order))
        c1, o1 = _canonical(c, o)
        c2, o2 = _canonical(s['coef'], s['offset'])
        assert np.array_equal(o1, o2), key
        assert np.abs(c1 - c2).max() <= 1e-12 * np.abs(c2).max(), key
        n += 1
    assert n == 112


@pytest.mark.parametrize('seed', range(6))
def test_identities_on_random_cells(seed):
    """sum_p c_p o_p o_p^T = 2 x identity for the Laplacian (second moments,
    scale 1) and sum_p c_p o_p = e_v for the derivative along v, with
    o_p = offset_p h_cv; both annihilate constants."""
    rng = np.random.default_rng(seed)
    h_cv = np.eye(3) * rng.uniform(0.15, 0.3, 3) + rng.uniform(-0.03, 0.03, (3, 3))
    for n in (1, 2, 3):
        c, o = laplace_stencil(h_cv, 1.0, n)
        r = o @ h_cv
        assert abs(c.sum()) < 1e-9 * np.abs(c).max()
        assert np.allclose(np.einsum('p,pi,pj->ij', c, r, r), 2 * np.eye(3), atol=1e-9)
        for v in range(3):
            c, o = gradient_stencil(h_cv, v, 1.0, n)
            r = o @ h_cv
            assert abs(c.sum()) < 1e-9 * np.abs(c).max()
            assert np.allclose(c @ r, np.eye(3)[v], atol=1e-9)


def test_degenerate_cell_is_refused():
    # two identical axes: the step moments cannot reach the identity
    h_cv = np.array([[0.2, 0, 0], [0.2, 1e-9, 0], [0, 0, 0.2]])
    with pytest.raises((ValueError, np.linalg.LinAlgError)):
        laplace_stencil(h_cv, 1.0, 1)
