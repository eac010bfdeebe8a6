"""ctypes binding of libgpawb200.so (the C ABI declared in include/gpawb200.h).

The library is built in-tree (gpaw_b200/build.py).  There is no fallback:
if the library is missing or a call fails, a GPAWB200Error is raised.
"""
from __future__ import annotations

import ctypes
from ctypes import c_double, c_int, c_int64, c_void_p, c_char_p, POINTER
from pathlib import Path

import numpy as np
import torch

LIBPATH = Path(__file__).resolve().with_name('libgpawb200.so')

GB_DTYPE = {torch.float64: 0, torch.float32: 1,
            torch.complex128: 2, torch.complex64: 3}


class GPAWB200Error(RuntimeError):
    pass


_lib = None

P64 = POINTER(c_int64)
PD = POINTER(c_double)

# name -> (restype, argtypes); mirrors include/gpawb200.h
_SIGNATURES = {
    'gb_last_error': (c_char_p, []),
    'gb_version': (c_char_p, []),
    'gb_device_sm_count': (c_int, [POINTER(c_int)]),
    'gb_operator_new': (c_int, [PD, P64, c_int, P64, c_int, P64, c_int, c_int,
                                POINTER(c_void_p)]),
    'gb_operator_apply': (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int,
                                  PD, c_void_p]),
    'gb_operator_apply_potential': (c_int, [c_void_p, c_void_p, c_void_p, c_int64,
                                            c_int, c_void_p, PD, c_void_p]),
    'gb_operator_relax': (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_int,
                                  c_double, c_void_p]),
    'gb_operator_get_diagonal_element': (c_int, [c_void_p, PD]),
    'gb_operator_free': (c_int, [c_void_p]),
    'gb_set_stencil_path': (c_int, [c_int]),
    'gb_device_errors': (c_int, [c_int, POINTER(c_int)]),
    'gb_transformer_new': (c_int, [P64, P64, c_int, P64, P64, P64, P64, c_int,
                                   c_int, POINTER(c_void_p)]),
    'gb_transformer_apply': (c_int, [c_void_p, c_void_p, c_void_p, c_int64,
                                     c_int, PD, c_void_p]),
    'gb_transformer_apply_axpy': (c_int, [c_void_p, c_void_p, c_void_p, c_int64,
                                          c_int, PD, c_double, c_void_p, c_double,
                                          c_void_p]),
    'gb_transformer_free': (c_int, [c_void_p]),
    'gb_fd_precond_noalloc': (c_int, [c_void_p] * 7 + [c_void_p, c_void_p,
                                                        c_double, c_int64, c_int,
                                                        PD, c_void_p]),
    'gb_lfc_new': (c_int, [c_int, c_void_p, P64, c_void_p, c_void_p, c_int,
                           c_void_p, c_void_p, c_double, c_int, c_void_p,
                           c_int64, c_int, POINTER(c_void_p)]),
    'gb_lfc_add': (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int, c_int,
                           c_void_p]),
    'gb_lfc_integrate': (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int,
                                 c_int, c_void_p]),
    'gb_lfc_free': (c_int, [c_void_p]),
    'gb_lfc_tiled': (c_int, [c_void_p]),
    'gb_add_to_density': (c_int, [c_int64, c_void_p, c_void_p, c_int, c_int64,
                                  c_void_p, c_void_p]),
    'gb_conv3d_forward': (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int,
                                  c_int, P64, POINTER(c_int), c_int, c_void_p]),
    'gb_conv3d_forward_pair': (c_int, [c_void_p, c_void_p, c_void_p, c_void_p,
                                       c_int64, P64, POINTER(c_int), c_void_p]),
    'gb_conv3d_backward_weight': (c_int, [c_void_p, c_void_p, c_void_p, c_int64,
                                          c_int, c_int, P64, POINTER(c_int),
                                          c_void_p]),
    'gb_band_dots': (c_int, [c_int64, c_int64, c_void_p, c_int64, c_void_p,
                             c_int64, c_int, c_void_p, c_void_p]),
    'gb_band_gram': (c_int, [c_int64, c_int, c_int64, c_void_p, c_int64,
                             c_int64, c_int, c_void_p, c_void_p]),
    'gb_band_gram_tc_workspace': (c_int, [c_int64, c_int64, c_int64, POINTER(c_int64)]),
    'gb_band_gram_tc': (c_int, [c_int64, c_int64, c_int64, c_void_p, c_int64, c_void_p,
                                c_int64, c_double, c_void_p, c_int64, c_void_p, c_int64,
                                c_void_p]),
    'gb_tf32_split': (c_int, [c_int64, c_int64, c_void_p, c_int64, c_void_p, c_void_p,
                              c_int64, c_void_p]),
    'gb_band_rotate_tc': (c_int, [c_int64, c_int64, c_int64, c_void_p, c_void_p, c_int64,
                                  c_void_p, c_int64, ctypes.c_float, c_void_p, c_int64,
                                  c_void_p, c_int64, c_void_p]),
    'gb_learned_fold_fine': (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int,
                                     c_void_p, c_int64, c_void_p, c_void_p]),
    'gb_learned_fold_stride': (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_void_p,
                                       c_void_p]),
    'gb_small_solve': (c_int, [c_int64, c_int, c_void_p, c_void_p, c_void_p,
                               c_void_p, c_void_p]),
    'gb_band_combine': (c_int, [c_int64, c_int64, c_int, c_void_p, c_void_p,
                                c_void_p, c_void_p, c_int64, c_int, c_void_p]),
    'gb_spline_new': (c_int, [c_int, c_double, c_int, PD, POINTER(c_void_p)]),
    'gb_spline_free': (c_int, [c_void_p]),
    'gb_spline_get': (c_int, [c_void_p, POINTER(c_int), PD, POINTER(c_int)]),
    'gb_spline_to_grid': (c_int, [c_void_p, P64, P64, PD, PD, P64, P64, c_void_p,
                                  c_void_p, P64, P64, c_void_p]),
    'gb_lfc_derivative': (c_int, [c_void_p, c_void_p, c_void_p, c_int64, PD, P64,
                                  POINTER(c_void_p), P64, PD, c_int, c_int, c_void_p]),
    'gb_operator_apply_k': (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int, c_int,
                                    PD, c_void_p, c_void_p]),
    'gb_transformer_apply_k': (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int, c_int,
                                       PD, c_void_p]),
    'gb_fd_precond_k': (c_int, [c_void_p] * 7 + [c_void_p] * 8 +
                        [c_void_p, c_double, c_int64, c_int, c_int, PD, c_void_p]),
    'gb_lfc_add_k': (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int, c_int, c_void_p]),
    'gb_lfc_integrate_k': (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int, c_int,
                                   c_void_p]),
    'gb_xc_calculate': (c_int, [c_int, c_int, c_int64, c_void_p, c_void_p,
                                c_void_p, c_void_p, c_void_p, c_void_p]),
    'gb_fd_precond': (c_int, [c_void_p] * 7 + [c_void_p] * 8 +
                      [c_void_p, c_void_p, c_double, c_int64, c_int, PD,
                       c_void_p]),
}


def lib():
    """Load (once) and return the ctypes handle of libgpawb200.so."""
    global _lib
    if _lib is None:
        if not LIBPATH.exists():
            raise GPAWB200Error(
                f'{LIBPATH} is missing: build it with `python -m gpaw_b200.build`'
                ' (there is no CPU fallback)')
        h = ctypes.CDLL(str(LIBPATH))
        for name, (res, args) in _SIGNATURES.items():
            f = getattr(h, name)
            f.restype = res
            f.argtypes = args
        _lib = h
    return _lib


def check(status: int, what: str = '') -> None:
    if status != 0:
        msg = lib().gb_last_error().decode(errors='replace')
        raise GPAWB200Error(f'{what}: status {status}: {msg}')


def i64(values) -> ctypes.Array:
    a = np.ascontiguousarray(np.asarray(values, dtype=np.int64).ravel())
    return (c_int64 * len(a))(*a.tolist())


def f64(values) -> ctypes.Array:
    a = np.ascontiguousarray(np.asarray(values, dtype=np.float64).ravel())
    return (c_double * len(a))(*a.tolist())


def phases(phase_cd) -> ctypes.Array | None:
    """3x2 complex Bloch phases -> 12 doubles (re, im) or None."""
    if phase_cd is None:
        return None
    if isinstance(phase_cd, torch.Tensor):
        phase_cd = phase_cd.detach().cpu().numpy()
    p = np.asarray(phase_cd, dtype=complex).reshape(3, 2)
    return f64(np.stack([p.real, p.imag], axis=-1))


def phase_sets(phase_cd):
    """(nk, 3, 2) complex Bloch phases (one set per k-point of a batch) ->
    (nk, ctypes array of nk x 12 doubles), or (1, 12 doubles) for a single
    (3, 2) set."""
    if isinstance(phase_cd, torch.Tensor):
        phase_cd = phase_cd.detach().cpu().numpy()
    p = np.asarray(phase_cd, dtype=complex).reshape(-1, 3, 2)
    return len(p), f64(np.stack([p.real, p.imag], axis=-1))


def is_phase_batch(phase_cd) -> bool:
    """True for (nk, 3, 2) phases with nk > 1 (a k-point batch)."""
    return phase_cd is not None and np.ndim(phase_cd) == 3 and np.shape(phase_cd)[0] > 1


def dtype_code(t: torch.Tensor) -> int:
    try:
        return GB_DTYPE[t.dtype]
    except KeyError:
        raise GPAWB200Error(f'unsupported dtype {t.dtype}') from None


def stream_of(t: torch.Tensor) -> int:
    return torch.cuda.current_stream(t.device).cuda_stream


def require_cuda(*tensors: torch.Tensor) -> None:
    for t in tensors:
        if not isinstance(t, torch.Tensor) or not t.is_cuda:
            raise GPAWB200Error('gpaw_b200 operators take CUDA torch tensors '
                                '(there is no CPU path)')
        if not t.is_contiguous():
            raise GPAWB200Error('arrays must be C-contiguous')


def ptr(t: torch.Tensor) -> int:
    return t.data_ptr()
