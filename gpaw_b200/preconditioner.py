"""Multigrid preconditioner (drop-in for gpaw.preconditioner.Preconditioner).

``Preconditioner(gd0, kin0, dtype, block)(residuals, kpt, ekin=None,
out=None)`` applies the reference's 3-level V-cycle (gpaw/preconditioner.py
:9-93, c/fd_preconditioner.c:108-353): nn=1 transformers, 7-point coarse
Laplacians with scale -0.5, step = 0.66666666 / kin0.diag.  One
gb_fd_precond call runs the whole cycle for all bands of the block on the
GPU (8 launches with the elementwise passes fused into kernel epilogues).
"""
from __future__ import annotations

import numpy as np
import torch

from gpaw_b200 import _native as nat
from gpaw_b200.fd_operators import Laplace
from gpaw_b200.transformers import Transformer


class Preconditioner:
    def __init__(self, gd0, kin0, dtype=float, block=1, xp=None):
        gd1 = gd0.coarsen()
        gd2 = gd1.coarsen()
        self.gd0, self.gd1, self.gd2 = gd0, gd1, gd2
        self.kin0 = kin0
        self.kin1 = Laplace(gd1, -0.5, 1, dtype, xp=xp)
        self.kin2 = Laplace(gd2, -0.5, 1, dtype, xp=xp)
        self.block = block
        self.dtype = dtype
        self.step = 0.66666666 / kin0.get_diagonal_element()
        self.restrictor_object0 = Transformer(gd0, gd1, 1, dtype, xp=xp)
        self.restrictor_object1 = Transformer(gd1, gd2, 1, dtype, xp=xp)
        self.interpolator_object2 = Transformer(gd2, gd1, 1, dtype, xp=xp)
        self.interpolator_object1 = Transformer(gd1, gd0, 1, dtype, xp=xp)
        self.restrictor0 = self.restrictor_object0.apply
        self.restrictor1 = self.restrictor_object1.apply
        self.interpolator2 = self.interpolator_object2.apply
        self.interpolator1 = self.interpolator_object1.apply
        self.use_c_precond = True
        self.xp = xp
        self._scratch = {}

    def calculate_kinetic_energy(self, psit_xG, kpt):
        return None

    def _work(self, nb, tdtype, device):
        key = (nb, tdtype, device)
        w = self._scratch.get(key)
        if w is None:
            w = (torch.empty((nb,) + tuple(self.gd0.n_c), dtype=tdtype, device=device),
                 torch.empty((3, nb) + tuple(self.gd1.n_c), dtype=tdtype, device=device),
                 torch.empty((3, nb) + tuple(self.gd2.n_c), dtype=tdtype, device=device))
            self._scratch = {key: w}
        return w

    def __call__(self, residuals, kpt=None, ekin=None, out=None):
        """Precondition all bands of `residuals` (nb, n0, n1, n2) in one
        batched call (the reference loops over blocks of `block` bands; the
        GPU path has no reason to)."""
        if residuals.ndim == 3:
            o = None if out is None else out[None]
            return self(residuals[None], kpt, out=o)[0]
        nat.require_cuda(residuals)
        nb = residuals.shape[0]
        if out is None:
            out = torch.empty_like(residuals)
        nat.require_cuda(out)
        phases = getattr(kpt, 'phase_cd', None) if kpt is not None else None
        if residuals.dtype.is_complex and phases is None:
            phases = np.ones((3, 2), complex)
        q0, w1, w2 = self._work(nb, residuals.dtype, residuals.device)
        r1, d1, q1 = w1
        r2, d2, q2 = w2
        P = nat.ptr
        if residuals.dtype.is_complex and nat.is_phase_batch(phases):
            # a k-point batch: nk equal groups of bands, one phase set each
            nk, ph = nat.phase_sets(phases)
            nat.check(nat.lib().gb_fd_precond_k(
                self.restrictor_object0.handle, self.restrictor_object1.handle,
                self.interpolator_object1.handle, self.interpolator_object2.handle,
                self.kin0.handle, self.kin1.handle, self.kin2.handle,
                P(out), P(q0), P(r1), P(d1), P(q1), P(r2), P(d2), P(q2),
                P(residuals), self.step, nb, nat.dtype_code(residuals), nk, ph,
                nat.stream_of(residuals)), 'gb_fd_precond_k')
            return out
        nat.check(nat.lib().gb_fd_precond(
            self.restrictor_object0.handle, self.restrictor_object1.handle,
            self.interpolator_object1.handle, self.interpolator_object2.handle,
            self.kin0.handle, self.kin1.handle, self.kin2.handle,
            P(out), P(q0), P(r1), P(d1), P(q1), P(r2), P(d2), P(q2),
            P(residuals), None, self.step, nb, nat.dtype_code(residuals),
            nat.phases(phases) if residuals.dtype.is_complex else None,
            nat.stream_of(residuals)), 'gb_fd_precond')
        return out
