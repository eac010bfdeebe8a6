"""FTLaplace, the spectral Laplacian of Laplace(gd, scale, n=9)
(gpaw/fd_operators.py:172-173, 357-382).

CPU: the |k|^2 table of a cubic cell against (2 pi / L)^2 (i^2 + j^2 + k^2)
with the frequencies folded to -N/2 .. N/2 - 1, and the diagonal element.
GPU: apply() against a numpy restatement of the reference's
ifftn(fftn(a) k2).real on a skewed periodic cell (1e-12, real and complex
input, a batch of bands in one call), and the plane-wave identity."""
import numpy as np
import pytest

from gpaw_b200.fd_operators import FTLaplace, Laplace
from gpaw_b200.grid_descriptor import GridDescriptor


def test_table_and_diagonal():
    L, N = 5.0, 8
    gd = GridDescriptor((N, N, N), (L, L, L), True, device='cpu')
    op = Laplace(gd, -0.5, n=9)
    assert isinstance(op, FTLaplace)
    f = np.fft.fftfreq(N, 1.0 / N)                 # 0, 1, .., N/2 - 1, -N/2, .., -1
    want = 0.5 * (2 * np.pi / L)**2 * (f[:, None, None]**2 + f[None, :, None]**2 + f[None, None, :]**2)
    assert np.allclose(op.k2_Q.numpy(), want, rtol=1e-14, atol=0)
    assert op.get_diagonal_element() == 6.0 / (L / N)**2


def test_needs_periodic_grid():
    gd = GridDescriptor((8, 8, 8), (5.0, 5.0, 5.0), (1, 0, 1), device='cpu')
    with pytest.raises(ValueError):
        FTLaplace(gd, -0.5)


def restated(a, gd, scale):
    """The reference's construction and apply, in numpy."""
    N_c = np.asarray(gd.N_c)
    i_cq = np.indices(N_c).reshape((3, -1))
    i_cq += N_c[:, None] // 2
    i_cq %= N_c[:, None]
    i_cq -= N_c[:, None] // 2
    k_vq = np.dot(2.0 * np.pi * gd.icell_cv.T, i_cq)
    k2 = (k_vq**2).sum(axis=0).reshape(N_c) * -scale
    return np.array([np.fft.ifftn(np.fft.fftn(x) * k2).real for x in a])


@pytest.mark.gpu
@pytest.mark.parametrize('cplx', [False, True])
def test_apply_matches_restatement(cplx):
    import torch
    cell = np.array([[4.0, 0.0, 0.0], [1.0, 4.5, 0.0], [0.5, 0.3, 5.0]])
    gd = GridDescriptor((12, 14, 16), cell, True)
    rng = np.random.default_rng(0)
    a = rng.standard_normal((3, 12, 14, 16))
    if cplx:
        a = a + 1j * rng.standard_normal(a.shape)
    op = Laplace(gd, -0.5, n=9)
    x = torch.from_numpy(a).cuda()
    y = torch.empty_like(x)
    op.apply(x, y)
    want = restated(a, gd, -0.5)
    got = y.cpu().numpy()
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    if cplx:
        assert np.all(got.imag == 0)


@pytest.mark.gpu
def test_plane_wave():
    import torch
    L, N = 6.0, 16
    gd = GridDescriptor((N, N, N), (L, L, L), True)
    x = (np.arange(N) * L / N)[:, None, None]
    y = (np.arange(N) * L / N)[None, :, None]
    k = 2 * np.pi / L * np.array([2.0, -3.0, 0.0])
    a = np.cos(k[0] * x + k[1] * y + 0 * x * y[..., :1]) * np.ones((N, N, N))
    t = torch.from_numpy(a[None]).cuda()
    out = torch.empty_like(t)
    Laplace(gd, -0.5, n=9).apply(t, out)
    assert np.allclose(out.cpu().numpy()[0], 0.5 * (k @ k) * a, atol=1e-12)
