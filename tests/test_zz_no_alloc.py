"""GPU: gb_fd_precond_noalloc, the multigrid V-cycle for callers that cannot
allocate device memory while they run (a C or Fortran host program that owns
only its residual and result buffers, or a process with a device-memory
budget fixed at start-up).  It takes its work grids from a fixed array inside
the library instead of from the caller.

Checked through the C ABI against gb_fd_precond (the entry point whose work
grids the caller allocates) on two calls in a row with different residuals,
so that a second call cannot lean on what the first left in the shared
array; the second call must leave the device's free memory and torch's
allocation count unchanged; a call with no grids does the one-time set-up
only; and a request larger than the fixed array is refused with an error
before anything is launched.  This file is collected last on purpose."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = {torch.float64: 1e-12, torch.float32: 1e-5, torch.complex128: 1e-12}


def _setup(N, pbc, dtype):
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200.preconditioner import Preconditioner
    gd = GridDescriptor(N, 0.2 / 0.52917721 * np.array(N), pbc)
    cplx = dtype.is_complex
    kin = Laplace(gd, -0.5, 3, complex if cplx else float)
    return gd, Preconditioner(gd, kin, complex if cplx else float)


def _noalloc(P, res, out, phases):
    from gpaw_b200 import _native as nat
    return nat.lib().gb_fd_precond_noalloc(
        P.restrictor_object0.handle, P.restrictor_object1.handle,
        P.interpolator_object1.handle, P.interpolator_object2.handle,
        P.kin0.handle, P.kin1.handle, P.kin2.handle,
        nat.ptr(out), nat.ptr(res), P.step, res.shape[0], nat.dtype_code(res),
        nat.phases(phases) if phases is not None else None, nat.stream_of(res))


class _K:
    def __init__(self, phase_cd):
        self.phase_cd = phase_cd


@pytest.mark.parametrize('N,pbc,dtype', [
    ((32, 32, 32), (1, 1, 1), torch.float64),
    ((24, 28, 32), (0, 0, 0), torch.float32),
    ((24, 24, 32), (1, 1, 0), torch.complex128),
])
def test_noalloc_matches_fd_precond(N, pbc, dtype):
    from gpaw_b200 import _native as nat
    gd, P = _setup(N, pbc, dtype)
    phases = None
    if dtype.is_complex:
        k_c = np.array([0.25, -0.125, 0.0])
        phases = np.exp(2j * np.pi * np.outer(k_c, [1, -1]))
    g = torch.Generator(device='cuda').manual_seed(11)
    real = torch.float64 if dtype == torch.complex128 else dtype
    # set-up only: nothing to precondition, the array's address is looked up
    nat.check(_noalloc(P, torch.empty(0, device='cuda', dtype=dtype),
                       torch.empty(0, device='cuda', dtype=dtype), phases),
              'gb_fd_precond_noalloc set-up')
    for call in range(2):
        shape = (5 + call,) + tuple(gd.n_c)
        res = torch.randn(shape, generator=g, device='cuda', dtype=real)
        if dtype.is_complex:
            res = torch.complex(res, torch.randn(shape, generator=g, device='cuda', dtype=real))
        want = P(res, _K(phases) if phases is not None else None)
        got = torch.full_like(res, float('nan'))
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        used0 = torch.cuda.memory_allocated()
        nat.check(_noalloc(P, res, got, phases), 'gb_fd_precond_noalloc')
        torch.cuda.synchronize()
        if call == 1:
            # the kernels are loaded by now: the call itself takes nothing
            assert torch.cuda.mem_get_info()[0] == free0
            assert torch.cuda.memory_allocated() == used0
        err = ((got - want).abs().max() / want.abs().max()).item()
        assert err < TOL[dtype], (call, err)


def test_noalloc_rejects_oversize():
    from gpaw_b200 import _native as nat
    gd, P = _setup((56, 56, 56), (1, 1, 1), torch.float64)
    # 64 grids of 56^3 FP64 need about 1.41 x 64 x 1.4 MB = 127 MB > 64 MiB
    res = torch.zeros((64,) + tuple(gd.n_c), device='cuda', dtype=torch.float64)
    out = torch.full_like(res, 7.0)
    status = _noalloc(P, res, out, None)
    assert status == -1
    msg = nat.lib().gb_last_error().decode()
    assert 'fewer grids per call' in msg and str(64 << 20) in msg
    torch.cuda.synchronize()
    assert bool((out == 7.0).all())
