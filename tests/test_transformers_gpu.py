"""GPU parity of restriction / interpolation (gb_transformer_apply) against
the oracle and the reference's golden vectors; tolerances as in
test_fd_gpu.py (1e-12 FP64, 1e-5 FP32, norm-wise relative)."""
import numpy as np
import pytest
import torch

from conftest import seeded, bloch_phases, relerr
from oracle import fd

pytestmark = pytest.mark.gpu

TOL = {torch.float64: 1e-12, torch.complex128: 1e-12,
       torch.float32: 1e-5, torch.complex64: 1e-5}


def grids(N, pbc, cell=(3.0, 3.0, 3.5)):
    from gpaw_b200.grid_descriptor import GridDescriptor
    gfine = GridDescriptor(N, cell, pbc)
    return gfine, gfine.coarsen()


def test_golden_transformers(golden_kernels):
    from gpaw_b200.transformers import Transformer
    n = 0
    for key, out in golden_kernels.items():
        if not key.startswith('tr|'):
            continue
        _, pbc, nn, cplx, kind, seed = key.split('|')
        pbc = tuple(int(c) for c in pbc)
        nn, cplx, seed = int(nn), bool(int(cplx)), int(seed)
        gf, gc = grids((16, 16, 20), pbc)
        gi, go = (gf, gc) if kind == 'R' else (gc, gf)
        a = seeded(seed, (1,) + tuple(gi.n_c), cplx)
        t = Transformer(gi, go, nn, complex if cplx else float)
        x = torch.from_numpy(a).cuda()
        y = t.apply(x, None, bloch_phases(pbc) if cplx else None)
        assert relerr(y.cpu().numpy(), out) < 1e-12, key
        n += 1
    assert n == 24


@pytest.mark.parametrize('N,pbc', [((32, 32, 32), (0, 0, 0)),
                                   ((32, 32, 32), (1, 1, 1)),
                                   ((24, 40, 16), (1, 0, 1)),
                                   ((56, 56, 56), (1, 1, 1)),
                                   ((28, 28, 28), (1, 1, 1)),
                                   ((76, 20, 12), (0, 0, 0))])
@pytest.mark.parametrize('nn', [1, 2, 3, 4])
@pytest.mark.parametrize('dtype', [torch.float64, torch.float32,
                                   torch.complex128, torch.complex64])
def test_transformers_random(N, pbc, nn, dtype):
    from gpaw_b200.transformers import Transformer
    gf, gc = grids(N, pbc)
    rng = np.random.default_rng(nn)
    phase = bloch_phases(pbc, (0.3, -0.1, 0.45)) if dtype.is_complex else None
    for gi, go in ((gf, gc), (gc, gf)):
        if not pbc[0] and go is gf:
            # the reference's "Cannot construct interpolator" rule
            inpoints = (gi.n_c[0] + 2 * nn - 1) * (gi.n_c[1] + 2 * nn - 1)
            if inpoints > go.n_c[0] * go.n_c[1]:
                continue
        a = rng.standard_normal((2,) + tuple(gi.n_c))
        if dtype.is_complex:
            a = a + 1j * rng.standard_normal(a.shape)
        t = Transformer(gi, go, nn, complex if dtype.is_complex else float)
        x = torch.from_numpy(a).to('cuda', dtype)
        y = t.apply(x, None, phase)
        ahost = x.cpu().numpy().astype(np.complex128 if dtype.is_complex else np.float64)
        ot = fd.Transformer(fd.Grid(gi.N_c, gi.cell_cv, gi.pbc_c),
                            fd.Grid(go.N_c, go.cell_cv, go.pbc_c), nn)
        expect = ot.apply(ahost, phase)
        assert y.shape == expect.shape
        assert relerr(y.cpu().numpy(), expect) < TOL[dtype], (gi.N_c, go.N_c)


@pytest.mark.parametrize('pbc', [0, 1])
def test_integral_conservation_gpu(pbc):
    """gpaw/test/fd_ops/test_transformations.py / test_non_periodic.py."""
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.transformers import Transformer
    n = 20
    L = 1.0 if pbc else 8.0
    gd = GridDescriptor((n, n, n), (L, L, L), pbc)
    rng = np.random.RandomState(8)
    a = torch.from_numpy(rng.random(tuple(gd.n_c))).cuda()
    gd2 = gd.refine()
    tol = 1e-14 if pbc else 1e-10
    for nn in ((1, 2, 3, 4) if pbc else (1,)):
        b = Transformer(gd, gd2, nn).apply(a)
        assert abs(gd.integrate(a) - gd2.integrate(b)) < tol
    if pbc:
        gd3 = gd.coarsen()
        for nn in (1, 2, 3, 4):
            b = Transformer(gd, gd3, nn).apply(a)
            assert abs(gd.integrate(a) - gd3.integrate(b)) < tol


@pytest.mark.parametrize('nn', [1, 3])
def test_full_size_microbench_transformers(nn):
    """(256, 96^3) <-> (256, 48^3): one band against the oracle, integral
    conservation of every band (periodic), batch order independence."""
    from gpaw_b200.transformers import Transformer
    gf, gc = grids((96, 96, 96), (1, 1, 1), (19.2, 19.2, 19.2))
    g = torch.Generator(device='cuda').manual_seed(0)
    x = torch.randn((256, 96, 96, 96), generator=g, device='cuda', dtype=torch.float64)
    r = Transformer(gf, gc, nn).apply(x)
    b = 200
    ot = fd.Transformer(fd.Grid(gf.N_c, gf.cell_cv, gf.pbc_c),
                        fd.Grid(gc.N_c, gc.cell_cv, gc.pbc_c), nn)
    assert relerr(r[b].cpu().numpy(), ot.apply(x[b].cpu().numpy())) < 1e-12
    s_f = x.sum(dim=(1, 2, 3)) * gf.dv
    s_c = r.sum(dim=(1, 2, 3)) * gc.dv
    assert (s_f - s_c).abs().max().item() < 1e-9
    i = Transformer(gc, gf, nn).apply(r)
    assert (i.sum(dim=(1, 2, 3)) * gf.dv - s_c).abs().max().item() < 1e-9
    perm = torch.randperm(256, device='cuda')
    assert torch.equal(Transformer(gf, gc, nn).apply(x[perm].contiguous()), r[perm])
