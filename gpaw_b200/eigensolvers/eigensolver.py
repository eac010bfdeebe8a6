"""Eigensolver base: residuals and subspace diagonalisation
(gpaw/eigensolvers/eigensolver.py:121-236) on the GPU.

Projections are kept concatenated over atoms, P_nM (bands x sum_a ni_a),
and the atomic Hamiltonian corrections as one block-diagonal dH_MM, so that
sum_a p^a dH^a P^a is one GEMM and one LFC launch instead of a loop over
atoms.  H_nn = dv psi^H (T + v) psi + P^* dH P^T is accumulated in FP64 and
diagonalised in FP64 (torch.linalg.eigh on the device); psi, (T + v) psi and
P are rotated with GEMMs in the working precision.  Eigenvalues stay on the
device (kpt.eps_n, FP64), so an iteration needs no host round trip except
the eigensolver of the subspace matrix itself.  FP32 real wave functions take
the tensor-core band GEMMs (gpaw_b200.bandops.gram_tc / rotate_tc).
"""
from __future__ import annotations

import numpy as np
import torch

from gpaw_b200.bandops import band_combine, rotate_tc, tf32_split


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
        """One pass over the k-points; returns the eigenstate error as a
        0-d FP64 device tensor (no host synchronisation)."""
        error = None
        for kpt in wfs.kpt_u:
            if not wfs.orthonormalized:
                wfs.orthonormalize(kpt)
            e = self.iterate_one_k_point(ham, wfs, kpt, self.weights(kpt, wfs))
            error = e if error is None else error + e
            wfs.orthonormalize(kpt)
        wfs.orthonormalized = True
        self.error = error
        return error

    @staticmethod
    def weights(kpt, wfs):
        """Occupied bands carry the k-point weight in the error sum (the
        reference's default 'occupied' band convergence)."""
        w = getattr(kpt, '_w_n', None)
        if w is None:
            # kpt.weight: the k-point weight (an array of one per row for a
            # k-point batch)
            w = torch.as_tensor(np.where(np.asarray(kpt.f_n) > 0, kpt.weight, 0.0),
                                dtype=torch.float64, device=kpt.psit_nG.device)
            kpt._w_n = w
        return w

    @staticmethod
    def dH_times(ham, P_nM):
        """C_nM = P_nM dH_MM^T (dS = 0 for norm-conserving setups)."""
        return P_nM @ ham.dH_MM.to(P_nM.dtype).T

    def calculate_residuals(self, kpt, wfs, ham, psit_nG, P_nM, eps_n, R_nG):
        """R = (T + v) psi - eps psi + sum_a p^a dH^a P^a
        (gpaw/eigensolvers/eigensolver.py:153-172)."""
        eps = eps_n.to(torch.float64)
        band_combine(R_nG, torch.stack([torch.ones_like(eps), -eps], 1), [R_nG, psit_nG])
        wfs.pt.add_M(R_nG, self.dH_times(ham, P_nM),
                     kpt.q if wfs.dtype.is_complex else -1)

    def subspace_matrix(self, ham, wfs, kpt):
        """(H_nn in FP64, (T + v) psi): everything before the eigensolver of
        the subspace problem (no host synchronisation); for a k-point batch
        H is (nk, nbands, nbands), one block per k-point."""
        psit = kpt.psit_nG
        nk = getattr(kpt, 'nk', 1)
        Htpsit = torch.empty_like(psit)
        wfs.apply_pseudo_hamiltonian(kpt, ham, psit, Htpsit)
        H = wfs.matrix(psit, Htpsit, nk)
        wide = torch.complex128 if wfs.dtype.is_complex else torch.float64
        if kpt.P_nM is not None and kpt.P_nM.shape[-1]:
            Pw = kpt.P_nM.to(wide)
            if nk > 1:
                Pw = Pw.reshape(nk, Pw.shape[0] // nk, -1)
            H = H + (Pw.conj() @ ham.dH_MM.to(wide)) @ Pw.transpose(-1, -2)
        H = 0.5 * (H + H.conj().transpose(-1, -2))
        return H, Htpsit

    def subspace_rotate(self, wfs, kpt, eps, V, Htpsit):
        """psi, (T + v) psi and P rotated to the eigenvectors V of H_nn
        (per k-point for a batch: V (nk, nbands, nbands), eps flattened)."""
        psit = kpt.psit_nG
        nb = psit.shape[0]
        nk = getattr(kpt, 'nk', 1)
        if nk > 1:
            U = V.transpose(1, 2).to(wfs.dtype)
            rot = lambda x: torch.bmm(U, x.reshape(nk, nb // nk, -1)).reshape(x.shape)
            kpt.psit_nG = rot(psit)
            self.Htpsit_nG = rot(Htpsit)
            if kpt.P_nM is not None:
                kpt.P_nM = rot(kpt.P_nM)
            kpt.eps_n = eps.reshape(-1)
            return
        # phi_k = sum_m V[m, k] psi_m
        if psit.dtype == torch.float32:
            # FP32 real: tensor-core rotations sharing one TF32 split of
            # V^T - I (psi + (V^T - I) psi: near convergence V is close to
            # the identity, so the FP32 truncation of the tensor core stays
            # in the small correction)
            eye = torch.eye(nb, dtype=V.dtype, device=V.device)
            hi, lo = tf32_split(V.T - eye)
            new = rotate_tc((hi, lo, nb), psit, identity_split=True)
            if new is not None:
                kpt.psit_nG = new
                self.Htpsit_nG = rotate_tc((hi, lo, nb), Htpsit, identity_split=True)
                if kpt.P_nM is not None:
                    kpt.P_nM = V.T.to(kpt.P_nM.dtype) @ kpt.P_nM
                kpt.eps_n = eps
                return
        U = V.T.to(wfs.dtype)
        kpt.psit_nG = (U @ psit.reshape(nb, -1)).reshape(psit.shape)
        self.Htpsit_nG = (U @ Htpsit.reshape(nb, -1)).reshape(psit.shape)
        if kpt.P_nM is not None:
            kpt.P_nM = U @ kpt.P_nM
        kpt.eps_n = eps

    def subspace_diagonalize(self, ham, wfs, kpt):
        H, Htpsit = self.subspace_matrix(ham, wfs, kpt)
        eps, V = torch.linalg.eigh(H)          # batched over k for a batch
        self.subspace_rotate(wfs, kpt, eps, V, Htpsit)
