"""Forces (Hellmann-Feynman, eV / Angstrom).

CPU (the oracle, oracle/scf.py, whose projector / vbar / ion-charge terms
come from the reference's own LFC.derivative, c/lfc.c:1449-1601): the
analytic force is the derivative of the total energy -- against central
differences of converged H2 energies, Richardson-extrapolated over two
steps, to 2e-4 eV/Angstrom.
GPU: the device forces against the oracle's from the same start (FP64,
1e-3 eV/Angstrom, the precision bar for forces), FP32 against FP64 (1e-3),
and the device forces against Richardson-extrapolated differences of the
device's own energies on a rattled Si8 cell."""
import numpy as np
import pytest

from oracle import ref

BOHR = 0.52917721067
TIGHT = dict(energy_tol=1e-10, density_tol=1e-9, eigenstates_tol=1e-15)

pytestmark = pytest.mark.skipif(not ref.available(),
                                reason='oracle/_ref (the reference C extension) not built')


def _richardson(energy, d):
    """-dE/dx from central differences at steps d and d/2 (Richardson)."""
    f1 = -(energy(d) - energy(-d)) / (2 * d)
    f2 = -(energy(d / 2) - energy(-d / 2)) / d
    return (4 * f2 - f1) / 3


def test_oracle_force_is_the_energy_gradient():
    import sys
    sys.path.insert(0, str(__import__('conftest').REPO / 'tests'))
    from test_scf_oracle import cpu_start
    from oracle import scf as osf
    args = list(cpu_start('H2'))
    spos, cell_cv = args[1], args[2]

    def energy(dz):     # atom 1 moved by dz Bohr along z; eV
        a = list(args)
        a[1] = spos + np.outer([0, 1], dz * np.linalg.inv(cell_cv)[2])
        return osf.SCF(*a).run(maxiter=200, **TIGHT).energies[-1]
    F = osf.SCF(*args).run(maxiter=200, **TIGHT).forces()
    fd = _richardson(energy, 0.01) / BOHR
    assert abs(F[1, 2] - fd) < 2e-4, (F[1, 2], fd)
    assert abs(F[0, 2] + F[1, 2]) < 1e-6         # Newton's third law


def _system(name):
    from gpaw_b200.scf import h2, si_diamond
    if name == 'H2':
        sym, pos, cell = h2()
        return sym, pos, cell, False, 0.2, 4
    sym, pos, cell = si_diamond(1, 5.43, rattle=0.05, seed=1)
    return sym, pos, cell, True, 0.18, 32


def _calc(name, precision='fp64', pos=None):
    from gpaw_b200.scf import Calculation
    sym, p, cell, pbc, h, nb = _system(name)
    return Calculation(sym, p if pos is None else pos, cell, pbc, h=h, nbands=nb,
                       precision=precision)


@pytest.fixture(scope='module')
def fp64_runs():
    out = {}
    for name in ('H2', 'Si8'):
        c = _calc(name)
        log = c.run(maxiter=150, **TIGHT)
        assert log.converged
        out[name] = c
    return out


@pytest.mark.gpu
@pytest.mark.parametrize('name', ['H2', 'Si8'])
def test_forces_match_oracle(fp64_runs, name):
    from oracle import scf as osf
    c0 = _calc(name)
    o = osf.from_calculation(c0, xc='LDA').run(maxiter=150, **TIGHT)
    assert o.converged
    F = fp64_runs[name].forces()
    Fo = o.forces()
    assert np.abs(F - Fo).max() < 1e-3, np.abs(F - Fo).max()
    assert np.abs(F).max() > 0.05          # a geometry with real forces


@pytest.mark.gpu
@pytest.mark.parametrize('name', ['H2', 'Si8'])
def test_forces_fp32_against_fp64(fp64_runs, name):
    c = _calc(name, 'fp32')
    log = c.run(maxiter=150, energy_tol=1e-6)
    assert log.converged
    dF = np.abs(c.forces() - fp64_runs[name].forces()).max()
    assert dF < 1e-3, dF


@pytest.mark.gpu
def test_device_force_is_the_energy_gradient(fp64_runs):
    sym, pos, cell, pbc, h, nb = _system('Si8')
    F = fp64_runs['Si8'].forces()
    a, v = 3, 0

    def energy(dx):      # atom a moved by dx Angstrom along v; eV
        p = pos.copy()
        p[a, v] += dx
        return _calc('Si8', pos=p).run(maxiter=150, **TIGHT).energies[-1]
    fd = _richardson(energy, 0.01)
    assert abs(F[a, v] - fd) < 2e-4, (F[a, v], fd)


@pytest.mark.gpu
def test_h2o_cluster_precision():
    """The precision configuration: 32 H2O (seeded orientations and jitter,
    15 A box, zero boundaries, h = 0.2 A -> 76^3), 160 bands (128
    occupied), PBE.  The FP32 run (stencils, LFC, preconditioner and band
    GEMMs in FP32; Cholesky, eigh, Poisson, XC and energy sums in FP64)
    against the FP64 run from the same start: total energy within 1e-5 eV
    per valence electron, occupied eigenvalues within 1e-4 eV, forces
    within 1e-3 eV / Angstrom.  Both runs converge the density to 1e-6 per
    electron: forces are not variational, and at GPAW's default 1e-4 the
    FP64 run's own forces are still 1e-2 eV / Angstrom from their converged
    values (the FP32 floor is ~6e-8)."""
    from gpaw_b200.scf import Calculation, h2o_cluster
    sym, pos, cell = h2o_cluster()
    out = {}
    for prec, tol in (('fp64', 1e-7), ('fp32', 1e-6)):
        c = Calculation(sym, pos, cell, False, h=0.2, nbands=160, xc='PBE',
                        precision=prec, mixer_beta=0.1)
        assert tuple(c.gd.N_c) == (76, 76, 76)
        log = c.run(maxiter=300, energy_tol=tol, density_tol=1e-6)
        assert log.converged, (prec, log.iterations)
        out[prec] = (log.energies[-1], c.eigenvalues()[:128], c.forces(), c.nvalence)
        del c
    (E64, e64, F64, nel), (E32, e32, F32, _) = out['fp64'], out['fp32']
    assert nel == 256
    assert abs(E32 - E64) / nel < 1e-5
    assert np.abs(e32 - e64).max() < 1e-4
    assert np.abs(F32 - F64).max() < 1e-3
