"""The SCF against its CPU oracle (oracle/scf.py): the same algorithm built
from GPAW's own C kernels (oracle/_ref) and numpy restatements of the
reference's RMM-DIIS (gpaw/eigensolvers/rmmdiis.py:63-272), residuals and
subspace diagonalisation (gpaw/eigensolvers/eigensolver.py:121-236),
orthonormalisation (gpaw/wavefunctions/fdpw.py:394-424) and Poisson solver
(gpaw/poisson.py:842-1007).

CPU (the oracle on its own): the reference's blocked-RMM-DIIS invariant
(gpaw/test/eigen/test_blocked_rmm_diis.py: band blocks of 3 give the same
energy to 1e-6 eV in the same number of iterations) and the Kohn-Sham
equations at self-consistency, on the H2 configuration.

GPU (FP64 unless stated): from identical inputs -- the new potential and
energy terms (1e-12), the subspace Hamiltonian (1e-12), one RMM-DIIS pass
after the rotation and the orthonormalisation that follows (1e-10); then
full SCFs from the same start, FP64 and FP32, on H2 (zero boundaries) and
Si8 (periodic, Gamma): total energy within 1e-5 eV per valence electron and
occupied eigenvalues within 1e-4 eV of the oracle's converged run."""
import numpy as np
import pytest

from oracle import ref

pytestmark = pytest.mark.skipif(not ref.available(),
                                reason='oracle/_ref (the reference C extension) not built')

TIGHT = dict(energy_tol=1e-7, density_tol=1e-6, eigenstates_tol=1e-11)


def system(name):
    from gpaw_b200.scf import h2, si_diamond
    if name == 'H2':
        sym, pos, cell = h2()
        return sym, pos, cell, False, 0.2, 4
    sym, pos, cell = si_diamond(1, 5.43)
    return sym, pos, cell, True, 0.18, 32


def cpu_start(name, seed=0):
    """Oracle inputs with a numpy start: random combinations of
    atom-centred s and p Gaussians plus 1 % noise, orthonormalised."""
    from gpaw_b200.hgh import HGHSetup
    from oracle import scf as osf
    sym, pos, cell, pbc, h, nb = system(name)
    bohr = 0.52917721067
    cell_cv = np.diag(cell) / bohr
    pbc_c = np.array([pbc] * 3)
    N_c = osf.h2gpts(h / bohr, cell_cv)
    kinds = {s: HGHSetup(s) for s in set(sym)}
    setups = [osf.setup_data(kinds[s]) for s in sym]
    spos = np.linalg.solve(cell_cv.T, (np.asarray(pos) / bohr).T).T
    if pbc:
        spos %= 1.0
    g = osf.Grid(N_c, cell_cv, pbc_c)
    r = np.linspace(0, 5.0, 201)
    gau = np.exp(-r**2 / (2 * 1.2**2))
    basis = osf.LFC(g, [[(0, 5.0, gau), (1, 5.0, gau)] for _ in sym], spos)
    rng = np.random.default_rng(seed)
    psit = np.zeros((nb,) + tuple(g.n_c))
    basis.add(psit, rng.standard_normal((nb, basis.Mmax)))
    psit += 0.01 * rng.standard_normal(psit.shape) * np.abs(psit).max()
    A = psit.reshape(nb, -1)
    psit = np.linalg.solve(np.linalg.cholesky(A @ A.T * g.dv), A).reshape(psit.shape)
    nel = sum(s['Z'] for s in setups)
    f_n = np.array([2.0] * (nel // 2) + [0.0] * (nb - nel // 2))
    return setups, spos, cell_cv, pbc_c, N_c, psit, f_n


def test_oracle_blocked_rmm_diis_invariant():
    from oracle import scf as osf
    args = cpu_start('H2')
    a = osf.SCF(*args).run(maxiter=60)
    b = osf.SCF(*args, blocksize=3).run(maxiter=60)
    assert a.converged and b.converged
    assert abs(a.energies[-1] - b.energies[-1]) < 1e-6
    assert a.iterations == b.iterations


def test_oracle_kohn_sham_equations_at_self_consistency():
    """Converged tightly, every occupied state satisfies H psi = eps psi
    in the final potential, and the density the states make is the one the
    potential came from."""
    from oracle import scf as osf
    o = osf.SCF(*cpu_start('H2')).run(maxiter=80, **TIGHT)
    assert o.converged
    H = o.apply_H(o.psit)
    o.residuals(o.psit, o.pt.integrate(o.psit), o.eps, H)
    occ = o.f_n > 0
    r = np.sqrt(o.dot(H, H))[occ]
    assert r.max() < 1e-5, r
    nt = np.einsum('n,n...->...', o.f_n, o.psit**2)
    assert np.abs(nt - o.nt_G).sum() * o.g.dv / o.nvalence < 1e-5


# ------------------------------------------------------------------ GPU
def gpu_calc(name, precision='fp64', blocksize=None):
    from gpaw_b200.scf import Calculation
    sym, pos, cell, pbc, h, nb = system(name)
    return Calculation(sym, pos, cell, pbc, h=h, nbands=nb, xc='LDA',
                       precision=precision, blocksize=blocksize)


def oracle_for(calc):
    """The oracle on the device calculation's geometry, setups and start
    (its orthonormalised initial wave functions, widened to FP64)."""
    from oracle import scf as osf
    return osf.from_calculation(calc, xc='LDA')


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.gpu
@pytest.mark.parametrize('name', ['H2', 'Si8'])
def test_one_pass_matches_oracle(name):
    calc = gpu_calc(name)
    o = oracle_for(calc)
    wfs, kpt, es = calc.wfs, calc.wfs.kpt_u[0], calc.eigensolver
    # the potential from the same density
    calc.update_hamiltonian()
    o.update_hamiltonian()
    assert rel(calc.vt_G.cpu().numpy(), o.vt_G) < 1e-12
    assert rel(calc.e_terms.cpu().numpy(), o.e_terms) < 1e-12
    o.vt_G = calc.vt_G.cpu().numpy()
    # the subspace Hamiltonian of the same wave functions
    if o.P.size:
        assert rel(kpt.P_nM.cpu().numpy(), o.P) < 1e-12
    H, _ = es.subspace_matrix(calc, wfs, kpt)
    Ho = o.subspace_diagonalize()
    assert rel(H.cpu().numpy(), Ho) < 1e-12
    # one RMM-DIIS pass from the same rotated state (the rotation itself is
    # defined only up to signs / degenerate subspaces, so the device's is used)
    es.subspace_diagonalize(calc, wfs, kpt)
    o.psit = kpt.psit_nG.cpu().numpy().copy()
    o.Htpsit = es.Htpsit_nG.cpu().numpy().copy()
    o.P = kpt.P_nM.cpu().numpy().copy()
    o.eps = kpt.eps_n.cpu().numpy().copy()
    err = es.update_bands(calc, wfs, kpt, es.weights(kpt, wfs)).item()
    erro = o.update_bands()
    assert abs(err - erro) < 1e-10 * abs(erro)
    assert rel(kpt.psit_nG.cpu().numpy(), o.psit) < 1e-10
    wfs.orthonormalize(kpt)
    o.orthonormalize()
    assert rel(kpt.psit_nG.cpu().numpy(), o.psit) < 1e-10


@pytest.fixture(scope='module')
def oracle_runs():
    """Converged oracle SCFs from the device start of each system (the
    device start does not depend on the precision: FP32 runs start from
    the same FP64 combination rounded to FP32)."""
    out = {}
    for name in ('H2', 'Si8'):
        calc = gpu_calc(name)
        o = oracle_for(calc).run(maxiter=120, **TIGHT)
        assert o.converged, name
        out[name] = o
    return out


@pytest.mark.gpu
@pytest.mark.parametrize('name', ['H2', 'Si8'])
@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
def test_scf_matches_oracle(oracle_runs, name, precision):
    o = oracle_runs[name]
    calc = gpu_calc(name, precision)
    tol = TIGHT if precision == 'fp64' else dict(energy_tol=1e-6)
    log = calc.run(maxiter=120, **tol)
    assert log.converged
    nel = calc.nvalence
    dE = abs(log.energies[-1] - o.energies[-1]) / nel
    assert dE < 1e-5, dE
    occ = np.asarray(calc.wfs.kpt_u[0].f_n) > 0
    deps = np.abs(calc.eigenvalues()[occ] - o.eigenvalues()[occ]).max()
    assert deps < 1e-4, deps


@pytest.mark.gpu
def test_gpu_blocked_rmm_diis_invariant():
    """The reference's invariant on the device: the reference's band blocks
    of 10 and one block of every band reach the same energy (1e-6 eV) in the
    same number of iterations (Si8, FP64)."""
    a = gpu_calc('Si8').run(maxiter=80)
    b = gpu_calc('Si8', blocksize=10).run(maxiter=80)
    assert a.converged and b.converged
    assert abs(a.energies[-1] - b.energies[-1]) < 1e-6
    assert a.iterations == b.iterations
