"""FD wave functions on the GPU (the parts of gpaw.wavefunctions.fd /
fdpw that the RMM-DIIS hot path uses).

* ``apply_pseudo_hamiltonian``: kinetic stencil + local potential, one fused
  launch for all bands (gpaw/wavefunctions/fd.py:82-88).
* ``orthonormalize``: S = dv psi^H psi (+ P dS P^H), inverse Cholesky,
  psi <- L^-1 psi (gpaw/wavefunctions/fdpw.py:394-424).  The band-space
  products are GEMMs in the working precision (FP32 with full-precision
  accumulation, no TF32); the Cholesky factorisation and the triangular
  inverse run in FP64 on the device.
"""
from __future__ import annotations

import numpy as np
import torch

from gpaw_b200.fd_operators import Laplace
from gpaw_b200.lfc import LFC
from gpaw_b200.bandops import band_dots, band_gram, gram_tc, rotate_tc

REAL_OF = {torch.float64: torch.float64, torch.float32: torch.float32,
           torch.complex128: torch.float64, torch.complex64: torch.float32}


def gemm_precision():
    # FP32 band-space products at full FP32 precision (no TF32 rounding)
    torch.backends.cuda.matmul.allow_tf32 = False


class KPoint:
    """The wave functions of one k-point, or of a batch of nk k-points.

    A batch holds nk equal groups of bands in one array (rows k * nbands ..
    (k + 1) * nbands - 1 belong to k-point k), q = range(nk), phase_cd the
    (nk, 3, 2) Bloch phases and weight the k-point weight of every row, so
    that each stencil, preconditioner and LFC launch covers every (k, band);
    the band-space products are batched over k.  f_n includes the k-point
    weight (occupation x weight, as the reference's kpt.f_n)."""

    def __init__(self, psit_nG, q=-1, phase_cd=None, weight=1.0, k_c=None, nk=1):
        self.psit_nG = psit_nG
        self.q = q
        self.phase_cd = phase_cd
        self.weight = weight
        self.k_c = np.zeros(3) if k_c is None else np.asarray(k_c, float)
        self.nk = nk
        self.eps_n = None     # FP64 device tensor after the first subspace step
        self.f_n = None
        self.P_nM = None      # projections <p^a_i|psi_n>, concatenated over atoms


class FDWaveFunctions:
    def __init__(self, gd, nbands, setups, spos_ac, dtype=torch.float64,
                 stencil=3, kd=None):
        self.gd = gd
        self.nbands = nbands
        self.setups = setups
        self.dtype = dtype
        self.real_dtype = REAL_OF[dtype]
        cplx = dtype.is_complex
        self.kin = Laplace(gd, -0.5, stencil, complex if cplx else float)
        self.pt = LFC(gd, [s.pt_j for s in setups], kd=kd, cut=True,
                      dtype=complex if cplx else float)
        self.pt.set_positions(spos_ac)
        self.kpt_u = []
        self.orthonormalized = False
        gemm_precision()

    # ------------------------------------------------------------------
    def apply_pseudo_hamiltonian(self, kpt, ham, psit_xG, Htpsit_xG):
        vt = ham.vt_G if self.real_dtype == torch.float64 else ham.vt_G32
        self.kin.apply_potential(psit_xG, Htpsit_xG, vt, kpt.phase_cd)
        return Htpsit_xG

    def projections(self, psit_xG, kpt):
        """P_xM = <p^a_i|psi_x>, concatenated over atoms (one LFC integrate
        for all bands)."""
        return self.pt.integrate(psit_xG, {}, kpt.q if self.dtype.is_complex else -1)

    def split_M(self, c_xM):
        return {a: c_xM[..., self.pt.M_a[a]:self.pt.M_a[a] + s.ni]
                for a, s in enumerate(self.setups) if s.ni > 0}

    def join_M(self, c_axi, xshape):
        return self.pt._gather(c_axi, xshape, self.dtype, self.gd.device)

    def matrix(self, a_nG, b_nG, nk=1):
        """dv a^H b as an (n, m) FP64 matrix (one GEMM), or (nk, n/nk, m/nk)
        for a k-point batch (one batched GEMM).  The overlap and
        subspace-Hamiltonian matrices feed Cholesky and eigh, which stay FP64,
        so their sums over grid points are accumulated in FP64 even when
        the wave functions are FP32 (the operands are widened on the fly)."""
        if nk > 1:
            wide = torch.complex128 if self.dtype.is_complex else torch.float64
            A = a_nG.reshape(nk, a_nG.shape[0] // nk, -1).to(wide)
            B = b_nG.reshape(nk, b_nG.shape[0] // nk, -1).to(wide)
            return torch.bmm(A.conj(), B.transpose(1, 2)) * self.gd.dv
        if a_nG.dtype == torch.float32 and b_nG.dtype == torch.float32:
            # FP32 real: tensor-core Gram (three-product TF32 split), the
            # diagonal from FP64-accumulated dots
            C = gram_tc(a_nG, b_nG, self.gd.dv,
                        exact_diagonal=a_nG.shape[0] == b_nG.shape[0])
            if C is not None:
                return C
        wide = torch.complex128 if self.dtype.is_complex else torch.float64
        A = a_nG.reshape(a_nG.shape[0], -1).to(wide)
        B = b_nG.reshape(b_nG.shape[0], -1).to(wide)
        return (A.conj() @ B.T) * self.gd.dv

    def orthonormalize(self, kpt, out=None):
        """psi <- L^-1 psi with S = L L^H (gpaw/wavefunctions/fdpw.py:
        394-424); `out` (optional, not aliasing psi) receives the result and
        becomes kpt.psit_nG -- a captured SCF step writes into its static
        buffer this way instead of copying."""
        psit = kpt.psit_nG
        nk = getattr(kpt, 'nk', 1)
        if nk > 1:
            # per k-point: S_k = L_k L_k^H, psi_k <- L_k^-1 psi_k (batched)
            S = self.matrix(psit, psit, nk)
            S = 0.5 * (S + S.conj().transpose(1, 2))
            L = torch.linalg.cholesky_ex(S)[0]
            eye = torch.eye(L.shape[-1], dtype=L.dtype, device=L.device).expand_as(L)
            Linv = torch.linalg.solve_triangular(L, eye, upper=False)
            C = Linv.conj().to(self.dtype)
            y = torch.bmm(C, psit.reshape(nk, psit.shape[0] // nk, -1)).reshape(psit.shape)
            if out is not None:
                y = out.copy_(y)
            kpt.psit_nG = y
            kpt.P_nM = self.projections(kpt.psit_nG, kpt)
            return
        S = self.matrix(psit, psit).to(torch.complex128 if self.dtype.is_complex
                                         else torch.float64)
        S = 0.5 * (S + S.conj().T)
        L = torch.linalg.cholesky_ex(S)[0]
        Linv = torch.linalg.solve_triangular(
            L, torch.eye(L.shape[0], dtype=L.dtype, device=L.device), upper=False)
        # psi_n <- sum_m Linv[n, m]^* psi_m  (S = L L^H, <phi|phi> = 1)
        nb = psit.shape[0]
        y = (rotate_tc(Linv, psit, out=out, identity_split=True)
             if psit.dtype == torch.float32 else None)
        if y is None:
            C = Linv.conj().to(self.dtype)
            y = (C @ psit.reshape(nb, -1)).reshape(psit.shape)
            if out is not None:
                y = out.copy_(y)
        kpt.psit_nG = y
        kpt.P_nM = self.projections(kpt.psit_nG, kpt)

    @staticmethod
    def band_dots(a_nG, b_nG):
        return band_dots(a_nG, b_nG)

    @staticmethod
    def band_gram(X_niG, k):
        return band_gram(X_niG, k)

    def add_to_density(self, nt_G, kpt):
        from gpaw_b200 import _native as nat
        f = getattr(kpt, '_f_t', None)
        if f is None:
            f = kpt._f_t = torch.as_tensor(np.asarray(kpt.f_n, float), device=self.gd.device)
        nb = kpt.psit_nG.shape[0]
        nat.check(nat.lib().gb_add_to_density(
            nb, nat.ptr(f), nat.ptr(kpt.psit_nG), nat.dtype_code(kpt.psit_nG),
            int(np.prod(self.gd.n_c)), nat.ptr(nt_G), nat.stream_of(nt_G)),
            'gb_add_to_density')
