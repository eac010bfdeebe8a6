"""Warm start from a .gpw file (row f4): a converged state written in the
reference's layout and read back restarts the SCF at convergence -- the
same energy (FP64: 1e-6 eV; FP32: 1e-5 eV per electron) and occupied
eigenvalues (1e-4 eV) in a few iterations instead of the cold start's many;
a file of another grid is refused."""
import numpy as np
import pytest

from gpaw_b200.gpw import read_gpw, warm_start, write_gpw

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('name,precision', [('H2', 'fp64'), ('Si8', 'fp32')])
def test_warm_start(tmp_path, name, precision):
    from gpaw_b200.scf import Calculation, h2, si_diamond
    if name == 'H2':
        (sym, pos, cell), pbc, h, nb = h2(), False, 0.2, 4
    else:
        (sym, pos, cell), pbc, h, nb = si_diamond(1, 5.43), True, 0.18, 32
    tol = dict(energy_tol=1e-7, density_tol=1e-6) if precision == 'fp64' else dict(energy_tol=1e-6)
    c = Calculation(sym, pos, cell, pbc, h=h, nbands=nb, xc='LDA', precision=precision)
    log = c.run(maxiter=120, **tol)
    assert log.converged
    path = tmp_path / f'{name}.gpw'
    write_gpw(c, path)
    s = read_gpw(path)
    assert s.psit.shape[:3] == (1, 1, nb)
    d = Calculation(sym, pos, cell, pbc, h=h, nbands=nb, xc='LDA', precision=precision, seed=5)
    warm_start(d, s)
    logd = d.run(maxiter=120, **tol)
    assert logd.converged
    assert logd.iterations <= max(5, log.iterations // 3), (logd.iterations, log.iterations)
    dE = abs(logd.energies[-1] - log.energies[-1])
    assert dE < (1e-6 if precision == 'fp64' else 1e-5 * c.nvalence), dE
    occ = np.arange(nb) < c.nvalence // 2
    assert np.abs(d.eigenvalues()[occ] - c.eigenvalues()[occ]).max() < 1e-4


def test_other_grid_is_refused(tmp_path):
    from gpaw_b200.scf import Calculation, h2
    sym, pos, cell = h2()
    c = Calculation(sym, pos, cell, False, h=0.2, nbands=4, xc='LDA')
    c.run(maxiter=5)
    write_gpw(c, tmp_path / 'a.gpw')
    d = Calculation(sym, pos, cell, False, h=0.25, nbands=4, xc='LDA')
    with pytest.raises(ValueError):
        warm_start(d, read_gpw(tmp_path / 'a.gpw'))
