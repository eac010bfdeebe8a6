"""Both stencil kernels (the cp.async kernel and the TMA pipeline) against
the oracle on layouts where both apply, plus the bounded-wait error flag."""
import ctypes

import numpy as np
import pytest
import torch

from conftest import relerr
from oracle import fd

pytestmark = pytest.mark.gpu

TOL = {torch.float64: 1e-12, torch.complex128: 1e-12,
       torch.float32: 1e-5, torch.complex64: 1e-5}


def set_path(mode):
    from gpaw_b200 import _native as nat
    nat.check(nat.lib().gb_set_stencil_path(mode), 'gb_set_stencil_path')


def device_error():
    from gpaw_b200 import _native as nat
    code = ctypes.c_int()
    nat.check(nat.lib().gb_device_errors(1, ctypes.byref(code)), 'gb_device_errors')
    return code.value


@pytest.fixture(autouse=True)
def restore_path():
    yield
    set_path(0)


@pytest.mark.parametrize('n_c,pbc,n', [((32, 32, 32), (1, 1, 1), 3),
                                       ((32, 32, 32), (0, 0, 0), 3),
                                       ((24, 40, 16), (1, 0, 1), 2),
                                       ((48, 48, 48), (1, 1, 1), 1),
                                       ((56, 56, 56), (1, 1, 1), 3),
                                       ((20, 18, 64), (0, 1, 0), 4)])
@pytest.mark.parametrize('dtype', [torch.float64, torch.float32,
                                   torch.complex128, torch.complex64])
@pytest.mark.parametrize('mode', [1, 2])
def test_paths_agree_with_oracle(n_c, pbc, n, dtype, mode):
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.fd_operators import Laplace
    pbc_a = np.array(pbc, bool)
    gd = GridDescriptor(np.array(n_c) + (1 - pbc_a), 0.2 * (np.array(n_c) + 1), pbc)
    lap = Laplace(gd, -0.5, n, complex if dtype.is_complex else float)
    rng = np.random.default_rng(4)
    a = rng.standard_normal((5,) + tuple(n_c))
    if dtype.is_complex:
        a = a + 1j * rng.standard_normal(a.shape)
    x = torch.from_numpy(a).to('cuda', dtype)
    y = torch.full_like(x, float('nan'))
    set_path(mode)
    try:
        lap.apply(x, y, np.ones((3, 2), complex) if dtype.is_complex else None)
    except Exception as e:
        if mode == 2 and 'not applicable' in str(e):
            pytest.skip('TMA path not applicable to this layout')
        raise
    torch.cuda.synchronize()
    assert device_error() == 0
    ah = x.cpu().numpy().astype(np.complex128 if dtype.is_complex else np.float64)
    expect = fd.fd_apply(lap.coef_p, lap.offset_pc, ah, pbc)
    assert relerr(y.cpu().numpy(), expect) < TOL[dtype]


@pytest.mark.parametrize('mode', [1, 2])
def test_paths_epilogue_via_precond(mode):
    """The V-cycle exercises the fused epilogues of both kernels."""
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200.preconditioner import Preconditioner
    gd = GridDescriptor((64, 64, 64), (12.0, 12.0, 12.0), True)
    kin = Laplace(gd, -0.5, 3)
    P = Preconditioner(gd, kin, float, block=10)
    R = torch.randn((6, 64, 64, 64), dtype=torch.float64, device='cuda')
    set_path(mode)
    d = P(R)
    torch.cuda.synchronize()
    assert device_error() == 0
    og = fd.Grid(gd.N_c, gd.cell_cv, gd.pbc_c)
    expect = fd.precondition(R.cpu().numpy(), og, (kin.coef_p, kin.offset_pc), P.step)
    assert relerr(d.cpu().numpy(), expect) < 1e-12
