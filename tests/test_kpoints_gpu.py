"""GPU: k-point batching on the Si8 configuration -- diamond Si, 8-atom
cubic cell (a = 5.43 A), periodic, h = 0.18 A (32^3), 2 x 2 x 2
Monkhorst-Pack grid reduced by time reversal to 4 k-points of weight 1/4,
32 bands, complex wave functions, LDA.

* The batched form (every k-point and band in each stencil, V-cycle and
  LFC launch; band-space products batched over k) against the reference's
  structure (one KPoint per k-point, RMM-DIIS blocks of 10 bands, the
  eigensolver looping over k-points): the same energy (1e-6 eV) in the same
  number of iterations, complex128.
* complex64 against complex128 (both batched, the FP32 one replayed as
  CUDA graphs): total energy within 1e-5 eV per valence electron and every
  occupied eigenvalue within 1e-4 eV.
* One launch per operator for all k-points: an eager iteration of the
  4-k-point batch launches the stencil kernel as often as a single
  k-point's iteration does."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def si8(precision='fp64', **kw):
    from gpaw_b200.scf import Calculation, si_diamond
    s, p, c = si_diamond(1, 5.43)
    return Calculation(s, p, c, True, h=0.18, nbands=32, precision=precision, **kw)


def test_kpoint_set():
    c = si8(kpts=(2, 2, 2))
    assert len(c.ibz_kc) == 4 and np.allclose(c.w_k, 0.25)
    kpt = c.wfs.kpt_u[0]
    assert kpt.nk == 4 and kpt.psit_nG.shape[0] == 4 * 32
    assert kpt.psit_nG.dtype == torch.complex128


@pytest.fixture(scope='module')
def batched64():
    c = si8(kpts=(2, 2, 2))
    log = c.run(maxiter=100, energy_tol=1e-7)
    assert log.converged
    return c, log


def test_batched_matches_per_kpoint_loop(batched64):
    c, log = batched64
    d = si8(kpts=(2, 2, 2), kbatch=False, blocksize=10)
    assert len(d.wfs.kpt_u) == 4
    logd = d.run(maxiter=100, energy_tol=1e-7)
    assert logd.converged
    assert abs(log.energies[-1] - logd.energies[-1]) < 1e-6
    assert log.iterations == logd.iterations
    assert np.abs(c.eigenvalues() - d.eigenvalues()).max() < 1e-6


def test_complex64_against_complex128(batched64):
    c, log = batched64
    f = si8('fp32', kpts=(2, 2, 2))
    assert f.wfs.kpt_u[0].psit_nG.dtype == torch.complex64
    logf = f.run(maxiter=100, energy_tol=1e-6, graph=True)
    assert logf.converged and logf.graphed
    nel = c.nvalence
    assert abs(logf.energies[-1] - log.energies[-1]) / nel < 1e-5
    occ = slice(0, nel // 2)
    assert np.abs(f.eigenvalues()[:, occ] - c.eigenvalues()[:, occ]).max() < 1e-4


def _stencil_launches(calc):
    calc.update_hamiltonian()
    calc.iteration()
    torch.cuda.synchronize()
    with torch.profiler.profile(activities=[torch.profiler.ProfilerActivity.CUDA]) as prof:
        calc.iteration()
        torch.cuda.synchronize()
    return sum(e.count for e in prof.key_averages() if 'star_kernel' in e.key)


def test_one_stencil_launch_for_all_kpoints():
    batch = _stencil_launches(si8(kpts=(2, 2, 2)))
    single = _stencil_launches(si8(k_c=(0.25, 0.25, 0.25)))
    assert batch > 0 and batch == single, (batch, single)
