"""GPU: per-band inner products of RMM-DIIS (gb_band_dots, gb_band_gram)
against a plain PyTorch FP64 reference of the same sums
(gpaw/eigensolvers/rmmdiis.py:133-145, 175-190).  FP64 inputs: 1e-12
relative; FP32 inputs: the kernels accumulate in FP64, so the only error is
the FP32 rounding of the stored data, which the reference sees as well
(1e-12 relative to the sum of absolute values)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DT = [torch.float64, torch.float32, torch.complex128, torch.complex64]


class wfs_for:
    """the two module functions under their FDWaveFunctions method names"""

    def __init__(self, n_c):
        from gpaw_b200 import bandops as w
        self.band_dots = w.band_dots
        self.band_gram = w.band_gram


def rand(shape, dtype, g):
    real = torch.float64 if dtype in (torch.float64, torch.complex128) else torch.float32
    x = torch.randn(shape, generator=g, device='cuda', dtype=real)
    if dtype.is_complex:
        x = torch.complex(x, torch.randn(shape, generator=g, device='cuda', dtype=real))
    return x


@pytest.mark.parametrize('dtype', DT)
@pytest.mark.parametrize('n_c', [(12, 14, 16), (7, 9, 5)])
def test_band_dots(dtype, n_c):
    wfs = wfs_for(n_c)
    g = torch.Generator(device='cuda').manual_seed(1)
    a = rand((13,) + n_c, dtype, g)
    b = rand((13,) + n_c, dtype, g)
    got = wfs.band_dots(a, b)
    A = a.reshape(13, -1).to(torch.complex128)
    B = b.reshape(13, -1).to(torch.complex128)
    want = (A.conj() * B).real.sum(1)
    scale = (A.abs() * B.abs()).sum(1)
    assert torch.all((got - want).abs() <= 1e-12 * scale)
    # a strided band view (every other band of a larger array)
    big = rand((26,) + n_c, dtype, g)
    v = big[::2]
    got = wfs.band_dots(v, v)
    V = v.reshape(13, -1).to(torch.complex128)
    assert torch.allclose(got, (V.abs()**2).sum(1), rtol=1e-12, atol=0)


@pytest.mark.parametrize('dtype', DT)
@pytest.mark.parametrize('k', [1, 2, 3])
def test_band_gram(dtype, k):
    wfs = wfs_for((10, 12, 8))
    g = torch.Generator(device='cuda').manual_seed(2)
    X = rand((9, 3, 10, 12, 8), dtype, g)        # (bands, stored vectors, grid)
    got = wfs.band_gram(X, k)
    Xk = X[:, :k].reshape(9, k, -1).to(torch.complex128)
    want = torch.einsum('bix,bjx->bij', Xk.conj(), Xk).real
    scale = torch.einsum('bix,bjx->bij', Xk.abs(), Xk.abs())
    assert got.shape == (9, k, k)
    assert torch.all((got - want).abs() <= 1e-12 * scale)


@pytest.mark.parametrize('n', [1, 3, 4, 8])
def test_small_solve(n):
    from gpaw_b200.bandops import small_solve
    g = torch.Generator(device='cuda').manual_seed(n)
    A = torch.randn((50, n, n), generator=g, device='cuda', dtype=torch.float64)
    A = A + n * torch.eye(n, device='cuda', dtype=torch.float64)
    b = torch.randn((50, n), generator=g, device='cuda', dtype=torch.float64)
    x, info = small_solve(A, b)
    want = torch.linalg.solve(A, b)
    assert int(info.sum()) == 0
    assert torch.allclose(x, want, rtol=1e-11, atol=1e-12)
    # a bordered DIIS system (nearly parallel residuals) and a singular one
    A[0] = 0.0
    x, info = small_solve(A, b)
    assert int(info[0]) == 1 and bool((x[0] == 0).all()) and int(info[1:].sum()) == 0


@pytest.mark.parametrize('dtype', DT)
@pytest.mark.parametrize('k', [1, 2, 3, 4])
def test_band_combine(dtype, k):
    from gpaw_b200.bandops import band_combine
    g = torch.Generator(device='cuda').manual_seed(3 + k)
    hist = rand((7, 4, 6, 10, 9), dtype, g)          # a DIIS history, bands first
    coef = torch.randn((7, k), generator=g, device='cuda', dtype=torch.float64)
    xs = [hist[:, i] for i in range(k)]
    out = torch.empty_like(hist[:, 0])
    band_combine(out, coef, xs)
    real = torch.float64 if dtype in (torch.float64, torch.complex128) else torch.float32
    c = coef.to(real)                                 # the kernel's rounding
    want = sum(c[:, i].reshape(-1, 1, 1, 1).to(torch.complex128) * xs[i].to(torch.complex128)
               for i in range(k))
    tol = 1e-14 if real == torch.float64 else 1e-6
    assert (out.to(torch.complex128) - want).abs().max() <= tol * want.abs().max()
    # in place: y <- y + a x
    y = xs[0].clone()
    a = torch.randn(7, generator=g, device='cuda', dtype=torch.float64)
    band_combine(y, torch.stack([torch.ones_like(a), a], 1), [y, hist[:, 1]])
    want = xs[0].to(torch.complex128) + a.to(real).reshape(-1, 1, 1, 1) * hist[:, 1].to(torch.complex128)
    assert (y.to(torch.complex128) - want).abs().max() <= tol * want.abs().max()
