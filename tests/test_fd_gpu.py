"""GPU parity of the FD stencil kernels (gb_operator_apply through the C ABI)
against the oracle and the reference's golden vectors.

Tolerances (norm-wise relative, max|gpu - ref| / max|ref|): 1e-12 for
float64/complex128, 1e-5 for float32/complex64 (the float32 input is the
float64 input rounded; the oracle runs in float64)."""
import numpy as np
import pytest
import torch

from conftest import seeded, bloch_phases, relerr
from oracle import fd

pytestmark = pytest.mark.gpu

TOL = {torch.float64: 1e-12, torch.complex128: 1e-12,
       torch.float32: 1e-5, torch.complex64: 1e-5}


def gd_for(n_c, pbc, cell=None):
    from gpaw_b200.grid_descriptor import GridDescriptor
    pbc = np.array(pbc, bool)
    N_c = np.array(n_c) + (1 - pbc)
    if cell is None:
        cell = 0.2 * N_c
    return GridDescriptor(N_c, cell, pbc)


def to_dev(a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a)).to('cuda', dtype)


def run_op(coefs, offs, gd, a, dtype, phase=None):
    from gpaw_b200.fd_operators import FDOperator
    op = FDOperator(coefs, offs, gd, complex if dtype.is_complex else float)
    x = to_dev(a, dtype)
    y = torch.empty_like(x)
    op.apply(x, y, phase)
    torch.cuda.synchronize()
    return y.cpu().numpy()


def test_golden_stencils(golden_kernels, golden_stencils):
    n = 0
    for key, out in golden_kernels.items():
        if not key.startswith('op|'):
            continue
        _, st, pbc, cplx, seed = key.split('|')
        pbc = tuple(int(c) for c in pbc)
        cplx = bool(int(cplx))
        s = golden_stencils[st]
        n_c = np.array((6, 7, 8)) - (1 - np.array(pbc))
        a = seeded(int(seed), (1,) + tuple(n_c), cplx)
        gd = gd_for(n_c, pbc)
        dt = torch.complex128 if cplx else torch.float64
        got = run_op(s['coef'], s['offset'], gd, a, dt,
                     bloch_phases(pbc) if cplx else None)
        assert relerr(got, out) < 1e-12, key
        n += 1
    assert n == 48


CASES = [
    # (n_c, pbc, stencil order n)
    ((31, 31, 31), (0, 0, 0), 3),     # H2 config: N=32 zero boundary
    ((32, 32, 32), (1, 1, 1), 3),     # Si8 config grid
    ((13, 7, 40), (1, 0, 1), 3),      # ragged, mixed boundaries
    ((5, 6, 7), (0, 1, 0), 1),
    ((4, 4, 4), (1, 1, 1), 2),        # stencil nearly as long as the domain
    ((9, 10, 11), (1, 1, 1), 4),
    ((14, 13, 12), (0, 0, 1), 6),
    ((75, 3, 33), (0, 1, 1), 1),
]


@pytest.mark.parametrize('n_c,pbc,n', CASES)
@pytest.mark.parametrize('dtype', [torch.float64, torch.float32,
                                   torch.complex128, torch.complex64])
def test_laplace_random(n_c, pbc, n, dtype):
    from gpaw_b200.fd_operators import Laplace
    gd = gd_for(n_c, pbc)
    lap = Laplace(gd, -0.5, n, complex if dtype.is_complex else float)
    rng = np.random.default_rng(11)
    a = rng.standard_normal((3,) + tuple(n_c))
    phase = None
    if dtype.is_complex:
        a = a + 1j * rng.standard_normal(a.shape)
        phase = bloch_phases(pbc, (0.13, -0.21, 0.37))
    x = to_dev(a, dtype)
    ahost = x.cpu().numpy().astype(np.complex128 if dtype.is_complex else np.float64)
    y = torch.empty_like(x)
    lap.apply(x, y, phase)
    torch.cuda.synchronize()
    expect = fd.fd_apply(lap.coef_p, lap.offset_pc, ahost, pbc, phase)
    assert relerr(y.cpu().numpy(), expect) < TOL[dtype]


@pytest.mark.parametrize('cell', ['hexagonal', 'fcc', 'bcc'])
@pytest.mark.parametrize('dtype', [torch.float64, torch.complex128, torch.float32])
def test_guc_laplace_box_path(cell, dtype, golden_stencils):
    import sys
    from conftest import GOLDEN
    sys.path.insert(0, str(GOLDEN))
    from cells import CELLS
    cell_cv = np.array(CELLS[cell], float) * 2.0
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.fd_operators import Laplace
    gd = GridDescriptor((12, 12, 12), cell_cv, True)
    lap = Laplace(gd, -0.5, 2, complex if dtype.is_complex else float)
    assert not lap.cfd
    rng = np.random.default_rng(3)
    a = rng.standard_normal((2, 12, 12, 12))
    phase = None
    if dtype.is_complex:
        a = a + 1j * rng.standard_normal(a.shape)
        phase = bloch_phases((1, 1, 1))
    x = to_dev(a, dtype)
    y = torch.empty_like(x)
    lap.apply(x, y, phase)
    expect = fd.fd_apply(lap.coef_p, lap.offset_pc, x.cpu().numpy().astype(
        np.complex128 if dtype.is_complex else np.float64), (1, 1, 1), phase)
    assert relerr(y.cpu().numpy(), expect) < TOL[dtype]


@pytest.mark.parametrize('v', [0, 1, 2])
@pytest.mark.parametrize('pbc', [(0, 0, 0), (1, 1, 1)])
def test_gradient(v, pbc):
    from gpaw_b200.fd_operators import Gradient
    gd = gd_for((20, 21, 22), pbc)
    g = Gradient(gd, v, 1.0, 3)
    a = np.random.default_rng(v).standard_normal((2, 20, 21, 22))
    x = to_dev(a, torch.float64)
    y = torch.empty_like(x)
    g.apply(x, y)
    expect = fd.fd_apply(g.coef_p, g.offset_pc, a, pbc)
    assert relerr(y.cpu().numpy(), expect) < 1e-12


def test_gradient_golden_vectors_gpu():
    """gpaw/test/fd_ops/test_gradient.py known answers on the GPU."""
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.fd_operators import Gradient, FDOperator
    gd = GridDescriptor((8, 1, 1), (8.0, 1.0, 1.0))
    a = gd.zeros()
    a[:, 0, 0] = torch.arange(8, dtype=torch.float64)
    d = gd.zeros()
    Gradient(gd, v=0).apply(a, d)
    assert d[:, 0, 0].tolist() == [-3, 1, 1, 1, 1, 1, 1, -3]
    FDOperator([-1, 1], [[-1, 0, 0], [0, 0, 0]], gd).apply(a, d)
    assert d[:, 0, 0].tolist() == [-7, 1, 1, 1, 1, 1, 1, 1]
    gd = GridDescriptor((1, 8, 1), (1.0, 8.0, 1.0), (1, 0, 1))
    a = gd.zeros()
    a[0, :, 0] = torch.arange(7, dtype=torch.float64)
    d = gd.zeros()
    Gradient(gd, v=1).apply(a, d)
    assert d[0, 0, 0].item() == 0.5 and d[0, :, 0].sum().item() == 3.0
    gd = GridDescriptor((1, 7, 1), ((1.0, 0.0, 0.0), (5.0, 5.0, 0.0),
                                    (0.0, 0.0, 0.7)))
    a = gd.zeros()
    a[0, :, 0] = torch.arange(7, dtype=torch.float64) - 1
    d = gd.zeros()
    Gradient(gd, v=1).apply(a, d)
    assert abs(d[0, 0, 0].item() + 3.5) < 1e-12 and abs(d[0, :, 0].sum().item()) < 1e-12


@pytest.mark.parametrize('cellname,cell', [
    ('sc', [1.1, 1.02, 1.03]),
    ('hexagonal', [(1, 0, 0), (0.5, 3**0.5 / 2, 0), (0, 0, 1.1)]),
    ('fcc', [(0, 1, 1), (1, 0, 1), (1, 1, 0)])])
@pytest.mark.parametrize('n', [1, 2, 3])
def test_polynomial_exactness_gpu(cellname, cell, n):
    """gpaw/test/fd_ops/test_laplace.py:82-101 on the GPU kernels."""
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.fd_operators import Laplace, Gradient
    N = 2 * n + 2
    gd = GridDescriptor((N, N, N), cell)
    idx = np.indices((N, N, N)).reshape(3, -1).T
    r_gv = (idx @ gd.h_cv).reshape(N, N, N, 3) - gd.cell_cv.sum(0) / 2
    lap = Laplace(gd, 1.0, n)
    grads = [Gradient(gd, v, n=n) for v in range(3)]
    b = gd.zeros()
    for m in range(0, 2 * n + 1):
        for ix in range(m + 1):
            for iy in range(m - ix + 1):
                iz = m - ix - iy
                a = torch.from_numpy((r_gv**(ix, iy, iz)).prod(3)).cuda()
                r = 2.0 if (m == 2 and max(ix, iy, iz) == 2) else 0.0
                lap.apply(a, b)
                assert abs(b[n + 1, n + 1, n + 1].item() - r) < 2e-12
                for v in range(3):
                    grads[v].apply(a, b)
                    r = 1.0 if (m == 1 and (ix, iy, iz)[v] == 1) else 0.0
                    assert abs(b[n + 1, n + 1, n + 1].item() - r) < 4e-12


def test_empty_batch_and_errors():
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200 import _native as nat
    gd = gd_for((8, 8, 8), (1, 1, 1))
    lap = Laplace(gd, -0.5, 3)
    x = torch.zeros((0, 8, 8, 8), dtype=torch.float64, device='cuda')
    lap.apply(x, torch.empty_like(x))
    with pytest.raises(ValueError):
        lap.apply(torch.zeros((8, 8, 9), dtype=torch.float64, device='cuda'),
                  torch.zeros((8, 8, 9), dtype=torch.float64, device='cuda'))
    with pytest.raises(ValueError):
        lap.apply(torch.zeros((8, 8, 8), dtype=torch.complex128, device='cuda'),
                  torch.zeros((8, 8, 8), dtype=torch.complex128, device='cuda'))
    with pytest.raises(nat.GPAWB200Error):
        lap.apply(torch.zeros((8, 8, 8), dtype=torch.float64, device='cuda'),
                  torch.zeros((8, 8, 16), dtype=torch.float64, device='cuda')[:, :, ::2])


@pytest.mark.parametrize('dtype,pbc', [(torch.float64, (1, 1, 1)),
                                       (torch.float32, (0, 0, 0))])
def test_full_size_microbench_grid(dtype, pbc):
    """(256, 96, 96, 96) (the kernel-microbench array): bands are independent
    (a permuted batch gives permuted outputs), one band matches the oracle,
    and for periodic boundaries every band's Laplacian sums to zero."""
    from gpaw_b200.fd_operators import Laplace
    gd = gd_for((96, 96, 96), pbc)
    lap = Laplace(gd, -0.5, 3)
    g = torch.Generator(device='cuda').manual_seed(0)
    x = torch.randn((256, 96, 96, 96), generator=g, device='cuda', dtype=dtype)
    y = torch.empty_like(x)
    lap.apply(x, y)
    perm = torch.randperm(256, device='cuda')
    y2 = torch.empty_like(x)
    lap.apply(x[perm].contiguous(), y2)
    assert torch.equal(y2, y[perm])
    b = 137
    expect = fd.fd_apply(lap.coef_p, lap.offset_pc,
                         x[b].double().cpu().numpy(), pbc)
    assert relerr(y[b].double().cpu().numpy(), expect) < TOL[dtype]
    if all(pbc):
        s = y.double().sum(dim=(1, 2, 3)).abs().max().item()
        scale = y.double().abs().sum(dim=(1, 2, 3)).max().item()
        assert s < 1e-12 * scale * (1e7 if dtype == torch.float32 else 1)
