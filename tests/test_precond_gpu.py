"""GPU parity of the batched multigrid V-cycle (gb_fd_precond) against the
oracle restatement of c/fd_preconditioner.c and the reference's golden
vectors (1e-12 FP64, 1e-5 FP32, norm-wise relative)."""
import numpy as np
import pytest
import torch

from conftest import seeded, bloch_phases, relerr
from oracle import fd

pytestmark = pytest.mark.gpu


def make(N, cell, pbc, dtype):
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200.preconditioner import Preconditioner
    gd = GridDescriptor(N, cell, pbc)
    dt = complex if dtype.is_complex else float
    kin = Laplace(gd, -0.5, 3, dt)
    return gd, kin, Preconditioner(gd, kin, dt, block=10)


class Kpt:
    def __init__(self, phase_cd):
        self.phase_cd = phase_cd


def test_golden_precond(golden_kernels):
    n = 0
    for key, out in golden_kernels.items():
        if not key.startswith('pc|'):
            continue
        _, pbc, cplx, seed = key.split('|')
        pbc = tuple(int(c) for c in pbc)
        cplx, seed = bool(int(cplx)), int(seed)
        dtype = torch.complex128 if cplx else torch.float64
        gd, kin, P = make((12, 12, 16), (3.2, 3.2, 4.0), pbc, dtype)
        R = torch.from_numpy(seeded(seed, (2,) + tuple(gd.n_c), cplx)).cuda()
        d0 = P(R, Kpt(bloch_phases(pbc)) if cplx else None)
        assert relerr(d0.cpu().numpy(), out) < 1e-12, key
        n += 1
    assert n == 3


@pytest.mark.parametrize('N,pbc', [((32, 32, 32), (0, 0, 0)),      # H2 config
                                   ((32, 32, 32), (1, 1, 1)),      # Si8 config
                                   ((56, 56, 56), (1, 1, 1)),      # Si64 config
                                   ((24, 16, 40), (1, 0, 1))])
@pytest.mark.parametrize('dtype', [torch.float64, torch.float32,
                                   torch.complex128, torch.complex64])
def test_precond_random(N, pbc, dtype):
    gd, kin, P = make(N, 0.2 / 0.529177 * np.array(N), pbc, dtype)
    rng = np.random.default_rng(7)
    B = 5
    a = rng.standard_normal((B,) + tuple(gd.n_c))
    phase = None
    if dtype.is_complex:
        a = a + 1j * rng.standard_normal(a.shape)
        phase = bloch_phases(pbc, (0.25, 0.0, -0.25))
    R = torch.from_numpy(a).to('cuda', dtype)
    d0 = P(R, Kpt(phase) if phase is not None else None)
    og = fd.Grid(gd.N_c, gd.cell_cv, gd.pbc_c)
    expect = fd.precondition(R.cpu().numpy().astype(
        np.complex128 if dtype.is_complex else np.float64), og,
        (kin.coef_p, kin.offset_pc), P.step, phase)
    tol = 1e-12 if dtype in (torch.float64, torch.complex128) else 1e-5
    assert relerr(d0.cpu().numpy(), expect) < tol
    # single band (3-D input) goes through the same batched path
    d1 = P(R[1], Kpt(phase) if phase is not None else None)
    assert relerr(d1.cpu().numpy(), expect[1]) < tol
