"""Tensor-core band GEMMs (gb_band_gram_tc / gb_band_rotate_tc) against FP64
products of the same FP32 inputs: the overlap / subspace-Hamiltonian sums
and the subspace rotation of gpaw/eigensolvers/eigensolver.py:174-236 and
gpaw/wavefunctions/fdpw.py:394-424.

Tolerances (FP32 accuracy of the three-product TF32 split, FP32 partial
sums over one CTA's share of the grid, FP64 across shares):
  gram   |C - C64|_ij <= 2e-6 sqrt(C64_ii C64_jj)   (Cauchy-Schwarz scale)
  rotate |Y - Y64|    <= 4e-6 (|U| |X|)              (per element; 160-term sums
                                                      accumulate with truncating
                                                      FP32 additions)
"""
import pytest
import torch

from gpaw_b200.bandops import gram_tc, rotate_tc, tf32_split

pytestmark = pytest.mark.gpu

GRAM_CASES = [(160, 160, 175616), (1, 1, 32), (17, 33, 1000), (300, 270, 5000),
              (160, 160, 100), (5, 7, 36), (129, 16, 4096)]
ROT_CASES = [(160, 160, 175616), (1, 1, 64), (17, 40, 1000), (300, 200, 3000),
             (160, 160, 100), (8, 3, 36), (257, 33, 260)]


def _rand(shape, seed):
    g = torch.Generator(device='cuda').manual_seed(seed)
    return torch.randn(shape, generator=g, device='cuda', dtype=torch.float32)


@pytest.mark.parametrize('na,nb,K', GRAM_CASES)
def test_gram_tc(na, nb, K):
    A = _rand((na, K), 1)
    B = _rand((nb, K), 2)
    C = gram_tc(A, B, alpha=0.5)
    assert C is not None and C.dtype == torch.float64 and C.shape == (na, nb)
    ref = 0.5 * (A.double() @ B.double().T)
    scale = torch.sqrt((A.double() ** 2).sum(1))[:, None] * torch.sqrt((B.double() ** 2).sum(1))[None, :]
    err = ((C - ref).abs() / (0.5 * scale)).max().item()
    assert err < 2e-6, err


def test_gram_tc_overlap_exact_diagonal():
    # S = psi psi^T: the long positive diagonal sums come from FP64 dots
    # (exact to FP64 rounding); off-diagonal errors stay at the FP32 level of
    # the Cauchy-Schwarz scale; symmetric to the same level
    psi = _rand((160, 56 * 56 * 56), 3).reshape(160, 56, 56, 56)
    S = gram_tc(psi, psi, alpha=0.1, exact_diagonal=True)
    ref = 0.1 * (psi.reshape(160, -1).double() @ psi.reshape(160, -1).double().T)
    d = torch.sqrt(torch.diagonal(ref))
    rel = (S - ref).abs() / (d[:, None] * d[None, :])
    assert torch.diagonal(rel).max().item() < 1e-12
    assert rel.max().item() < 2e-6, rel.max().item()
    assert ((S - S.T).abs() / (d[:, None] * d[None, :])).max().item() < 2e-6


def test_gram_tc_bias_of_positive_sums():
    # without the patch the diagonal of an overlap carries the FP32
    # accumulation bias (documented bound 1e-4 relative)
    psi = _rand((32, 175616), 8)
    S = gram_tc(psi, psi)
    ref = psi.double() @ psi.double().T
    diag_rel = ((torch.diagonal(S) - torch.diagonal(ref)).abs() / torch.diagonal(ref)).max().item()
    print('unpatched diagonal relative error', diag_rel)
    assert diag_rel < 1e-4


def test_gram_tc_unaligned_declines():
    A = _rand((4, 1001), 4)       # 1001-float rows: not 16-byte aligned
    assert gram_tc(A, A) is None


@pytest.mark.parametrize('nn,nk,K', ROT_CASES)
def test_rotate_tc(nn, nk, K):
    U = torch.randn((nn, nk), dtype=torch.float64, device='cuda',
                    generator=torch.Generator(device='cuda').manual_seed(5))
    X = _rand((nk, K), 6)
    Y = rotate_tc(U, X)
    assert Y is not None and Y.shape == (nn, K) and Y.dtype == torch.float32
    ref = U @ X.double()
    tol = 4e-6 * (U.abs() @ X.double().abs())
    assert ((Y.double() - ref).abs() <= tol).all(), ((Y.double() - ref).abs() / tol).max().item()


def test_rotate_tc_grid_shaped_orthogonal():
    # psi <- V^T psi for a general orthogonal V, grid-shaped input
    X = _rand((160, 56, 56, 56), 7)
    V = torch.linalg.qr(torch.randn((160, 160), dtype=torch.float64, device='cuda'))[0]
    Y = rotate_tc(V.T, X)
    assert Y.shape == X.shape
    ref = (V.T @ X.reshape(160, -1).double()).reshape(X.shape)
    tol = 4e-6 * (V.T.abs() @ X.reshape(160, -1).double().abs()).reshape(X.shape)
    assert ((Y.double() - ref).abs() <= tol).all()


def test_rotate_tc_identity_split_keeps_norms():
    # a rotation close to the identity (the inverse-Cholesky factor of a
    # nearly orthonormal set): rotating by V - I and adding psi back keeps
    # the norms to ~1e-7 (the plain form loses ~2e-6 to truncation)
    X = _rand((160, 56, 56, 56), 9)
    M = torch.eye(160, dtype=torch.float64, device='cuda') + 0.02 * torch.randn(
        (160, 160), dtype=torch.float64, device='cuda',
        generator=torch.Generator(device='cuda').manual_seed(10))
    Q, R = torch.linalg.qr(M)
    V = Q * torch.sign(torch.diagonal(R))[None, :]
    Xf = X.reshape(160, -1).double()
    ref = V.T @ Xf
    Y = rotate_tc(V.T, X, identity_split=True).reshape(160, -1).double()
    eye = torch.eye(160, dtype=torch.float64, device='cuda')
    tol = 4e-6 * ((V.T - eye).abs() @ Xf.abs()) + 2 ** -23 * ref.abs()
    assert ((Y - ref).abs() <= tol).all()
    n_ref = (ref ** 2).sum()
    assert abs((Y ** 2).sum() - n_ref).item() / n_ref.item() < 2e-7


def test_tf32_split_parts():
    U = torch.randn((37, 45), dtype=torch.float64, device='cuda')
    hi, lo = tf32_split(U)
    assert hi.shape == (37, 48)
    # both parts are TF32 numbers (low 13 mantissa bits clear) ...
    for t in (hi, lo):
        assert ((t.view(torch.int32) & 0x1FFF) == 0).all()
    # ... the padding is zero, and hi + lo carries ~22 bits of U
    assert (hi[:, 45:] == 0).all() and (lo[:, 45:] == 0).all()
    rel = ((hi[:, :45].double() + lo[:, :45].double() - U).abs() / U.abs()).max().item()
    assert rel < 2 ** -20
