"""Band-space helpers of RMM-DIIS on the GPU: per-band inner products, the
per-band DIIS Gram matrix, and batched small dense solves
(gpaw/eigensolvers/rmmdiis.py:133-190), each one launch for all bands and
free of host synchronisation (so they can sit inside a captured CUDA graph).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from gpaw_b200 import _native as nat


def band_dots(a_nG, b_nG):
    """Re <a_n|b_n> per band (without dv), FP64, one gb_band_dots launch."""
    if not (a_nG.is_cuda and b_nG.is_cuda):
        raise nat.GPAWB200Error('band_dots takes CUDA tensors (there is no CPU path)')
    nb = a_nG.shape[0]
    N = int(np.prod(a_nG.shape[1:]))
    if a_nG.dtype != b_nG.dtype:
        raise ValueError('band_dots: operands of different dtypes')
    if not (a_nG[0].is_contiguous() and b_nG[0].is_contiguous()):
        raise ValueError('band_dots: each band must be contiguous')
    out = torch.empty(nb, dtype=torch.float64, device=a_nG.device)
    nat.check(nat.lib().gb_band_dots(
        nb, N, nat.ptr(a_nG), a_nG.stride(0) if nb > 1 else N, nat.ptr(b_nG),
        b_nG.stride(0) if nb > 1 else N, nat.dtype_code(a_nG), nat.ptr(out),
        nat.stream_of(a_nG)), 'gb_band_dots')
    return out


def band_gram(X_niG, k):
    """Re <X_ni|X_nj> for i, j < k per band (without dv): (nb, k, k) FP64."""
    if not X_niG.is_cuda:
        raise nat.GPAWB200Error('band_gram takes CUDA tensors (there is no CPU path)')
    nb = X_niG.shape[0]
    N = int(np.prod(X_niG.shape[2:]))
    if not X_niG[0, 0].is_contiguous():
        raise ValueError('band_gram: each stored vector must be contiguous')
    out = torch.empty((nb, k, k), dtype=torch.float64, device=X_niG.device)
    nat.check(nat.lib().gb_band_gram(
        nb, k, N, nat.ptr(X_niG), X_niG.stride(0), X_niG.stride(1),
        nat.dtype_code(X_niG), nat.ptr(out), nat.stream_of(X_niG)), 'gb_band_gram')
    return out


def small_solve(A, b):
    """x with A[s] x[s] = b[s] for a batch of n x n FP64 systems (n <= 8),
    one gb_small_solve launch; singular systems give x[s] = 0 and info 1.
    Returns (x, info)."""
    if not (A.is_cuda and b.is_cuda):
        raise nat.GPAWB200Error('small_solve takes CUDA tensors (there is no CPU path)')
    n = A.shape[-1]
    A = A.to(torch.float64).contiguous()
    b = b.to(torch.float64).contiguous()
    nb = int(np.prod(A.shape[:-2], dtype=np.int64))
    x = torch.empty_like(b)
    info = torch.empty(A.shape[:-2], dtype=torch.int32, device=A.device)
    nat.check(nat.lib().gb_small_solve(nb, n, nat.ptr(A), nat.ptr(b), nat.ptr(x),
                                       nat.ptr(info), nat.stream_of(A)), 'gb_small_solve')
    return x, info


def band_combine(out, coef, xs):
    """out[n] = sum_i coef[n, i] xs[i][n] for every band n, one launch.

    out and every xs[i]: (nb, ...) tensors of one dtype whose bands are
    contiguous (band stride free, e.g. a column of a DIIS history); coef:
    (nb, k) real tensor (FP64 on the device, rounded to the working
    precision in the kernel); out may be one of xs (in-place update)."""
    k = len(xs)
    nb = out.shape[0]
    N = int(np.prod(out.shape[1:]))
    for x in xs:
        if x.dtype != out.dtype or x.shape[0] != nb or not x[0].is_contiguous():
            raise ValueError('band_combine: operands must share dtype and band count, '
                             'with contiguous bands')
    if not out[0].is_contiguous() or not out.is_cuda:
        raise ValueError('band_combine: out must be a CUDA tensor with contiguous bands')
    coef = coef.to(device=out.device, dtype=torch.float64).reshape(nb, k).contiguous()
    ptrs = (ctypes.c_void_p * k)(*[x.data_ptr() for x in xs])
    lds = (ctypes.c_int64 * k)(*[x.stride(0) if nb > 1 else N for x in xs])
    nat.check(nat.lib().gb_band_combine(
        nb, N, k, nat.ptr(coef), ptrs, lds, out.data_ptr(),
        out.stride(0) if nb > 1 else N, nat.dtype_code(out), nat.stream_of(out)),
        'gb_band_combine')
    return out


# ------------------------------------------------------------------------
# band-space GEMMs on the tensor cores (FP32 wave functions)

def _tc_layout_ok(t):
    return (t.is_cuda and t.dtype == torch.float32 and t.dim() >= 1
            and t.reshape(t.shape[0], -1).stride(1) == 1
            and t.data_ptr() % 16 == 0)


def gram_tc(a_nG, b_nG, alpha=1.0, exact_diagonal=False):
    """alpha a b^T over the grid points, (na, nb) FP64, for FP32 real wave
    functions (gb_band_gram_tc); None when the layout does not qualify
    (unaligned rows, other dtypes): the caller then takes its FP64 GEMM.

    The tensor cores accumulate each CTA's share of the sum in FP32 with
    truncating additions, which biases long sums of same-sign terms by up to
    ~3e-5 relative (the diagonal of an overlap matrix); off-diagonal sums
    wander around zero and keep a tiny absolute error.  exact_diagonal=True
    (na == nb) replaces the diagonal with FP64-accumulated per-band dots
    (gb_band_dots, one more pass over a and b), so norms and band energies
    carry no bias."""
    if not (_tc_layout_ok(a_nG) and _tc_layout_ok(b_nG)):
        return None
    A = a_nG.reshape(a_nG.shape[0], -1)
    B = b_nG.reshape(b_nG.shape[0], -1)
    na, K = A.shape
    nb = B.shape[0]
    lda = A.stride(0) if na > 1 else K
    ldb = B.stride(0) if nb > 1 else K
    if lda % 4 or ldb % 4 or B.shape[1] != K:
        return None
    ws = ctypes.c_int64(0)
    nat.check(nat.lib().gb_band_gram_tc_workspace(na, nb, K, ctypes.byref(ws)),
              'gb_band_gram_tc_workspace')
    work = torch.empty(max(1, ws.value // 8), dtype=torch.float64, device=A.device)
    C = torch.empty((na, nb), dtype=torch.float64, device=A.device)
    nat.check(nat.lib().gb_band_gram_tc(
        na, nb, K, nat.ptr(A), lda, nat.ptr(B), ldb, float(alpha), nat.ptr(C), nb,
        nat.ptr(work), work.numel() * 8, nat.stream_of(A)), 'gb_band_gram_tc')
    if exact_diagonal and na == nb:
        C.diagonal().copy_(band_dots(A, B) * alpha)
    return C


def tf32_split(U):
    """(hi, lo) TF32 parts of a real matrix (FP32 containers, columns padded
    to a multiple of 4), one gb_tf32_split launch."""
    U = U.to(torch.float64).contiguous()
    rows, cols = U.shape
    ldd = (cols + 3) // 4 * 4
    hi = torch.empty((rows, ldd), dtype=torch.float32, device=U.device)
    lo = torch.empty_like(hi)
    nat.check(nat.lib().gb_tf32_split(rows, cols, nat.ptr(U), cols, nat.ptr(hi), nat.ptr(lo),
                                      ldd, nat.stream_of(U)), 'gb_tf32_split')
    return hi, lo


def rotate_tc(U, x_nG, out=None, identity_split=False):
    """y_n = sum_k U[n, k] x_k over FP32 real wave functions on the tensor
    cores (gb_band_rotate_tc); U is any real (nn, nk) matrix (split into TF32
    parts on the device) or a (hi, lo, nk) triple from tf32_split, to share
    one split between rotations (with identity_split, the split of U - I).
    identity_split=True (square U) rotates by
    U - I and adds x back exactly in the epilogue, so the tensor core's
    truncation bias (~1e-6 of a long sum) touches only the correction: the
    form for rotations close to the identity (inverse-Cholesky
    orthonormalisation, subspace rotations near convergence).  None when
    the layout does not qualify."""
    if not _tc_layout_ok(x_nG):
        return None
    X = x_nG.reshape(x_nG.shape[0], -1)
    nk, K = X.shape
    ldx = X.stride(0) if nk > 1 else K
    if isinstance(U, tuple):
        hi, lo, ncols = U
        nn = hi.shape[0]
    else:
        if U.is_complex():
            return None
        nn, ncols = U.shape
        if identity_split:
            if nn != ncols:
                raise ValueError('rotate_tc: identity_split needs a square matrix')
            U = U.to(torch.float64) - torch.eye(nn, dtype=torch.float64, device=U.device)
        hi, lo = tf32_split(U)
    if ldx % 4 or ncols != nk:
        return None
    if out is None:
        out = torch.empty((nn,) + tuple(x_nG.shape[1:]), dtype=torch.float32, device=X.device)
    Y = out.reshape(nn, -1)
    Z = X if identity_split else None
    nat.check(nat.lib().gb_band_rotate_tc(
        nn, nk, K, nat.ptr(hi), nat.ptr(lo), hi.shape[1], nat.ptr(X), ldx,
        1.0, nat.ptr(Z) if Z is not None else None, ldx, nat.ptr(Y),
        Y.stride(0) if nn > 1 else K, nat.stream_of(X)), 'gb_band_rotate_tc')
    return out
