"""RMM-DIIS (drop-in for gpaw.eigensolvers.rmmdiis.RMMDIIS).

The reference's algorithm (gpaw/eigensolvers/rmmdiis.py:63-272): subspace
diagonalisation, residuals, then per band: precondition, line step
lambda = -<R|dR>/<dR|dR>, niter-1 DIIS steps over the stored (psi, R) pairs,
a final preconditioned trial step.  Every band's update uses only its own
vectors, so on the GPU all bands form one block: each stencil,
preconditioner and LFC launch covers every band, the per-band dot products
are batched reductions and the small DIIS systems are one batched solve.
"""
from __future__ import annotations

import numpy as np
import torch

from gpaw_b200.bandops import band_combine, small_solve
from gpaw_b200.eigensolvers.eigensolver import Eigensolver


class RMMDIIS(Eigensolver):
    def __init__(self, keep_htpsit=True, blocksize=None, niter=3, rtol=1e-16,
                 limit_lambda=False, use_rayleigh=False, trial_step=0.1):
        Eigensolver.__init__(self, keep_htpsit, blocksize)
        self.niter = niter
        self.rtol = rtol
        self.limit_lambda = limit_lambda
        self.trial_step = trial_step

    def todict(self):
        return {'name': 'rmm-diis', 'niter': self.niter}

    def iterate_one_k_point(self, ham, wfs, kpt, weights):
        self.subspace_diagonalize(ham, wfs, kpt)
        return self.update_bands(ham, wfs, kpt, weights)

    def update_bands(self, ham, wfs, kpt, weights):
        """Everything of one RMM-DIIS pass after the subspace rotation
        (residuals, preconditioned steps, DIIS); returns the weighted
        residual norm as a 0-d FP64 device tensor."""
        psit = kpt.psit_nG
        R = self.Htpsit_nG
        self.calculate_residuals(kpt, wfs, ham, psit, kpt.P_nM, kpt.eps_n, R)
        dv = wfs.gd.dv
        nb = psit.shape[0]
        B = nb if self.blocksize is None else self.blocksize
        Ht = lambda x, out: wfs.apply_pseudo_hamiltonian(kpt, ham, x, out)

        def dots(a, b):
            # Re <a_n|b_n> per band, FP64 accumulation
            return wfs.band_dots(a, b) * dv

        error = torch.zeros((), dtype=torch.float64, device=psit.device)
        for n1 in range(0, nb, B):
            n2 = min(n1 + B, nb)
            eps_x = kpt.eps_n[n1:n2]
            psitb = psit[n1:n2]
            Rb = R[n1:n2]
            error = error + (weights[n1:n2] * dots(Rb, Rb)).sum()
            nbl = n2 - n1
            # the DIIS history: slot 0 of the wave functions is psitb itself;
            # every later step writes its result straight into its slot (no
            # copies), residual slots live in one slot-major array for the
            # batched Gram kernel
            psi_slots = [psitb]
            R_diis = torch.empty((self.niter, nbl) + psit.shape[1:],
                                 dtype=psit.dtype, device=psit.device)
            R_diis[0].copy_(Rb)
            dpsit = self.preconditioner(R_diis[0], kpt)
            dR = torch.empty_like(dpsit)
            Ht(dpsit, dR)
            P = wfs.projections(dpsit, kpt)
            self.calculate_residuals(kpt, wfs, ham, dpsit, P, eps_x, dR)
            RdR = dots(dR, R_diis[0])
            dRdR = dots(dR, dR)
            lam = -RdR / dRdR
            if self.limit_lambda:
                lo, up = self.limit_lambda['lower'], self.limit_lambda['upper']
                if self.limit_lambda.get('absolute', False):
                    lam = torch.where(lam.abs() < lo, lo * lam.sign(), lam)
                    lam = torch.where(lam.abs() > up, up * lam.sign(), lam)
                else:
                    lam = lam.clamp(lo, up)
            lam2 = torch.stack([torch.ones_like(lam.reshape(-1)).to(torch.float64),
                                lam.reshape(-1).to(torch.float64)], 1)
            if self.niter > 1:
                psi_slots.append(torch.empty_like(psitb))
                band_combine(psi_slots[1], lam2, [psitb, dpsit])
                band_combine(R_diis[1], lam2, [R_diis[0], dR])
                cur_psi, cur_R = psi_slots[1], R_diis[1]
            else:
                cur_psi, cur_R = torch.empty_like(psitb), torch.empty_like(Rb)
                band_combine(cur_psi, lam2, [psitb, dpsit])
                band_combine(cur_R, lam2, [R_diis[0], dR])
            for nit in range(1, self.niter):
                if nit > 1 or self.limit_lambda:
                    # R_ij = <R_i|R_j> over the stored residuals (one batched
                    # Gram kernel), then the bordered DIIS system per band
                    R_nn = wfs.band_gram(R_diis.transpose(0, 1), nit + 1) * dv
                    A = -torch.ones((nbl, nit + 2, nit + 2), dtype=torch.float64,
                                    device=psit.device)
                    A[:, :nit + 1, :nit + 1] = R_nn
                    A[:, -1, -1] = 0.0
                    x = torch.zeros((nbl, nit + 2), dtype=torch.float64, device=psit.device)
                    x[:, -1] = -1.0
                    alpha = small_solve(A, x)[0][:, :-1]
                    cur_psi = torch.empty_like(psitb)
                    cur_R = torch.empty_like(Rb)
                    band_combine(cur_psi, alpha, psi_slots[:nit + 1])
                    band_combine(cur_R, alpha, [R_diis[i] for i in range(nit + 1)])
                if nit < self.niter - 1:
                    dpsit = self.preconditioner(cur_R, kpt)
                    nxt = torch.empty_like(psitb)
                    band_combine(nxt, lam2, [cur_psi, dpsit])
                    psi_slots.append(nxt)
                    Ht(nxt, R_diis[nit + 1])
                    P = wfs.projections(nxt, kpt)
                    self.calculate_residuals(kpt, wfs, ham, nxt, P, eps_x, R_diis[nit + 1])
                    cur_psi, cur_R = nxt, R_diis[nit + 1]
            dpsit = self.preconditioner(cur_R, kpt)
            step = (torch.full_like(lam, self.trial_step) if self.trial_step is not None
                    else lam)
            step2 = torch.stack([torch.ones_like(step.reshape(-1)).to(torch.float64),
                                 step.reshape(-1).to(torch.float64)], 1)
            band_combine(psitb, step2, [cur_psi, dpsit])
        return error
