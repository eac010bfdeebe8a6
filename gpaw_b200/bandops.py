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
