"""Eigensolver base: residuals and subspace diagonalisation
(gpaw/eigensolvers/eigensolver.py:121-236) on the GPU.

H_nn = dv psi^H (T + v) psi + P dH P^H is one GEMM plus small per-atom
products; it is diagonalised in FP64 (torch.linalg.eigh on the device) and
psi, (T + v) psi and P are rotated with GEMMs in the working precision.
"""
from __future__ import annotations

import numpy as np
import torch


class Eigensolver:
    def __init__(self, keep_htpsit=True, blocksize=None):
        self.keep_htpsit = keep_htpsit
        self.blocksize = blocksize
        self.preconditioner = None
        self.error = np.inf
        self.Htpsit_nG = None

    def initialize(self, wfs, preconditioner):
        self.preconditioner = preconditioner

    def iterate(self, ham, wfs):
        error = 0.0
        for kpt in wfs.kpt_u:
            if not wfs.orthonormalized:
                wfs.orthonormalize(kpt)
            weights = self.weights(kpt)
            error += self.iterate_one_k_point(ham, wfs, kpt, weights)
            wfs.orthonormalize(kpt)
        wfs.orthonormalized = True
        self.error = error
        return error

    @staticmethod
    def weights(kpt):
        """Occupied bands carry the k-point weight in the error sum (the
        reference's default 'occupied' band convergence)."""
        w = np.where(np.asarray(kpt.f_n) > 0, kpt.weight, 0.0)
        return w

    def dH_times(self, wfs, ham, P_ani):
        """C_ani = sum_j P_anj dH_aij (dS = 0 for norm-conserving setups)."""
        return {a: P @ ham.dH_aii[a].to(P.dtype).T for a, P in P_ani.items()}

    def calculate_residuals(self, kpt, wfs, ham, psit_nG, P_ani, eps_n, R_nG):
        """R = (T + v) psi - eps psi + sum_a p^a dH^a P^a
        (gpaw/eigensolvers/eigensolver.py:153-172)."""
        eps = torch.as_tensor(np.asarray(eps_n), dtype=wfs.real_dtype,
                              device=R_nG.device).reshape((-1, 1, 1, 1))
        R_nG -= eps * psit_nG
        C_ani = self.dH_times(wfs, ham, P_ani)
        wfs.pt.add(R_nG, C_ani, kpt.q if wfs.dtype.is_complex else -1)

    def subspace_diagonalize(self, ham, wfs, kpt):
        psit = kpt.psit_nG
        nb = psit.shape[0]
        Htpsit = torch.empty_like(psit)
        wfs.apply_pseudo_hamiltonian(kpt, ham, psit, Htpsit)
        H = wfs.matrix(psit, Htpsit)
        wide = torch.complex128 if wfs.dtype.is_complex else torch.float64
        for a, P in kpt.P_ani.items():
            Pw = P.to(wide)
            H = H + Pw.conj() @ ham.dH_aii[a].to(wide) @ Pw.T
        H64 = H
        H64 = 0.5 * (H64 + H64.conj().T)
        eps, V = torch.linalg.eigh(H64)
        # phi_k = sum_m V[m, k] psi_m
        U = V.T.to(wfs.dtype)
        kpt.psit_nG = (U @ psit.reshape(nb, -1)).reshape(psit.shape)
        self.Htpsit_nG = (U @ Htpsit.reshape(nb, -1)).reshape(psit.shape)
        kpt.P_ani = {a: U @ P for a, P in kpt.P_ani.items()}
        kpt.eps_n = eps.cpu().numpy()
