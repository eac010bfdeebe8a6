"""Grid restriction / interpolation on the GPU (drop-in for gpaw.transformers).

``Transformer(gdin, gdout, nn, dtype)`` returns an object with
``.apply(input, output=None, phases=None)`` exactly like the reference
(gpaw/transformers.py:18-134); restriction when ``gdin.N_c == 2 gdout.N_c``,
interpolation when ``gdout.N_c == 2 gdin.N_c``.  The pad/skip geometry is the
reference's (gpaw/transformers.py:27-47) and is handed to libgpawb200
(gb_transformer_*), which does all three separable passes in one kernel.
"""
from __future__ import annotations

import numpy as np
import torch

from gpaw_b200 import _native as nat
from gpaw_b200.grid_descriptor import is_real, torch_dtype


class _Transformer:
    def __init__(self, gdin, gdout, nn=1, dtype=float, xp=None):
        self.gdin = gdin
        self.gdout = gdout
        self.nn = nn
        assert 1 <= nn <= 4
        self.dtype = dtype
        self.xp = xp
        pad_cd = np.empty((3, 2), int)
        neighborpad_cd = np.empty((3, 2), int)
        skip_cd = np.zeros((3, 2), int)
        if (gdin.N_c == 2 * gdout.N_c).all():
            pad_cd[:, 0] = 2 * nn - 1 - 2 * gdout.beg_c + gdin.beg_c
            pad_cd[:, 1] = 2 * nn - 2 + 2 * gdout.end_c - gdin.end_c
            neighborpad_cd[:, 0] = 2 * nn - 2 + 2 * gdout.beg_c - gdin.beg_c
            neighborpad_cd[:, 1] = 2 * nn - 1 - 2 * gdout.end_c + gdin.end_c
            self.interpolate = False
        else:
            assert (gdout.N_c == 2 * gdin.N_c).all()
            pad_cd[:, 0] = nn - 1 - gdout.beg_c // 2 + gdin.beg_c
            pad_cd[:, 1] = nn + gdout.end_c // 2 - gdin.end_c
            neighborpad_cd[:, 0] = nn + gdout.beg_c // 2 - gdin.beg_c
            neighborpad_cd[:, 1] = nn - 1 - gdout.end_c // 2 + gdin.end_c
            skip_cd[:, 0] = gdout.beg_c % 2
            skip_cd[:, 1] = gdout.end_c % 2
            self.interpolate = True
            inpoints = (gdin.n_c[0] + 2 * nn - 1) * (gdin.n_c[1] + 2 * nn - 1)
            outpoints = gdout.n_c[0] * gdout.n_c[1]
            if inpoints > outpoints:
                points = ' x '.join([str(N) for N in gdin.N_c])
                raise ValueError('Cannot construct interpolator.  Grid %s '
                                 'may be too small' % points)
        assert (pad_cd.ravel() >= 0).all()
        self.ngpin = tuple(int(x) for x in gdin.n_c)
        self.ngpout = tuple(int(x) for x in gdout.n_c)
        self.pad_cd = pad_cd
        self.neighborpad_cd = neighborpad_cd
        self.skip_cd = skip_cd
        self.real = is_real(dtype)
        h = nat.c_void_p()
        nat.check(nat.lib().gb_transformer_new(
            nat.i64(gdin.n_c), nat.i64(gdout.n_c), 2 * nn, nat.i64(pad_cd),
            nat.i64(neighborpad_cd), nat.i64(skip_cd),
            nat.i64(gdin.neighbor_cd), int(self.real), int(self.interpolate),
            nat.ctypes.byref(h)), 'gb_transformer_new')
        self._handle = h

    def __del__(self):
        h = getattr(self, '_handle', None)
        if h is not None and h.value:
            try:
                nat.lib().gb_transformer_free(h)
            except Exception:
                pass

    @property
    def handle(self):
        return self._handle

    def apply(self, input, output=None, phases=None):
        nat.require_cuda(input)
        if tuple(input.shape[-3:]) != self.ngpin:
            raise ValueError(f'input grid {tuple(input.shape[-3:])} != {self.ngpin}')
        if output is None:
            output = torch.empty(tuple(input.shape[:-3]) + self.ngpout,
                                 dtype=input.dtype, device=input.device)
        nat.require_cuda(output)
        if tuple(output.shape) != tuple(input.shape[:-3]) + self.ngpout:
            raise ValueError('output shape mismatch')
        if output.dtype != input.dtype or input.dtype.is_complex == self.real:
            raise ValueError('dtype mismatch')
        if input.dtype.is_complex and phases is None:
            phases = np.ones((3, 2), complex)
        nin = int(np.prod(input.shape[:-3], dtype=np.int64))
        if input.dtype.is_complex and nat.is_phase_batch(phases):
            # a k-point batch: nk equal groups of grids, phases[k] each
            nk, ph = nat.phase_sets(phases)
            nat.check(nat.lib().gb_transformer_apply_k(
                self._handle, nat.ptr(input), nat.ptr(output), nin, nat.dtype_code(input),
                nk, ph, nat.stream_of(input)), 'gb_transformer_apply_k')
            return output
        nat.check(nat.lib().gb_transformer_apply(
            self._handle, nat.ptr(input), nat.ptr(output), nin,
            nat.dtype_code(input),
            nat.phases(phases) if input.dtype.is_complex else None,
            nat.stream_of(input)), 'gb_transformer_apply')
        return output

    def apply_axpy(self, input, output, alpha=1.0, y=None, gamma=0.0, phases=None):
        """output = alpha * T(input) + gamma * y in one launch (y only for
        interpolation; shaped like output)."""
        nat.require_cuda(input, output)
        if y is not None:
            nat.require_cuda(y)
            if tuple(y.shape) != tuple(output.shape) or y.dtype != output.dtype:
                raise ValueError('y must match the output')
        if tuple(output.shape) != tuple(input.shape[:-3]) + self.ngpout:
            raise ValueError('output shape mismatch')
        if input.dtype.is_complex and phases is None:
            phases = np.ones((3, 2), complex)
        nin = int(np.prod(input.shape[:-3], dtype=np.int64))
        nat.check(nat.lib().gb_transformer_apply_axpy(
            self._handle, nat.ptr(input), nat.ptr(output), nin, nat.dtype_code(input),
            nat.phases(phases) if input.dtype.is_complex else None, float(alpha),
            nat.ptr(y) if y is not None else None, float(gamma), nat.stream_of(input)),
            'gb_transformer_apply_axpy')
        return output

    def get_async_sizes(self):
        return (0, 1, 1)


def Transformer(gdin, gdout, nn=1, dtype=float, xp=None):
    if nn != 9:
        return _Transformer(gdin, gdout, nn, dtype, xp)

    class T:
        nn = 1

        def apply(self, input, output, phases=None):
            output[:] = input

    return T()
