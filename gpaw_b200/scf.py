"""Minimal FD SCF on the GPU: density -> potential -> RMM-DIIS -> mixing.

The parts of GPAW's old-code SCF that drive the hot path
(gpaw/scf.py:47-155, gpaw/density.py:225-272, 697-740,
gpaw/hamiltonian.py:232-282, 717-786), for norm-conserving HGH setups
(gpaw_b200/hgh.py) at the Gamma point or one k-point:

  density:      nt_G = sum_n f_n |psi_n|^2 (coarse, one launch), Pulay
                mixing on the coarse grid, interpolation to the fine grid
                (Transformer nn=3), rhot_g = nt_g + Gaussian ion charges
  Hamiltonian:  v_H from the FP64 FFT/DST Poisson solver, v_xc (LDA/PBE
                kernels), short-range local part vbar (LFC), vt_g restricted
                to the coarse grid (Transformer nn=3)
  eigensolver:  RMM-DIIS with the batched multigrid preconditioner (or a
                learned one)
  convergence:  energy change per valence electron over the last three
                iterations, density change per electron, eigenstate error
                per electron (gpaw/convergence_criteria.py:154-177)

Precision modes: 'fp64' (everything FP64) and 'fp32' (wave functions,
stencils, LFC, preconditioner and band GEMMs in FP32; Cholesky, eigh,
Poisson, XC and every energy sum in FP64).
Total energies have the zero of the reference's HGH setups: no atomic
reference energy, the ion charges' self-energy removed, ion-ion
interactions included through the Gaussian ion charges.
"""
from __future__ import annotations

import gc
import itertools
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from gpaw_b200.bandops import small_solve
from gpaw_b200.grid_descriptor import GridDescriptor
from gpaw_b200.hgh import HGHSetup
from gpaw_b200.lfc import LFC
from gpaw_b200.poisson import FastPoissonSolver
from gpaw_b200.transformers import Transformer
from gpaw_b200.wavefunctions import FDWaveFunctions, KPoint
from gpaw_b200.xc import XC
from gpaw_b200.eigensolvers import RMMDIIS
from gpaw_b200.preconditioner import Preconditioner

Bohr = 0.52917721067
Hartree = 27.211386024367243


def h2gpts(h, cell_cv, idiv=4):
    """Grid points for spacing h (gpaw/utilities/__init__.py:108-120)."""
    L_c = (np.linalg.inv(cell_cv)**2).sum(0)**-0.5
    return np.maximum(idiv, (L_c / h / idiv + 0.5).astype(int) * idiv)


class PulayMixer:
    """Pulay (DIIS) density mixing on the coarse grid (the role of
    gpaw/mixer.py:35-; plain Euclidean metric).

    The last `nmaxold` input densities and residuals (raw, for the Pulay
    matrix, and Kerker-filtered, for the update) live
    in fixed ring buffers written at a device-side position, so once the
    history is full a mixing step has fixed shapes and addresses and no host
    synchronisation (it can be replayed inside a CUDA graph).  The Pulay
    coefficients do not depend on the order of the history entries."""

    def __init__(self, beta=0.1, nmaxold=5, kerker_q0=None):
        self.beta = beta
        self.nmaxold = nmaxold
        self.kerker_q0 = kerker_q0
        self.gd = None
        self.reset()

    def _precondition(self, r_G):
        """Kerker filter k^2 / (k^2 + q0^2) on the residual (periodic cells):
        damps the long-wavelength charge sloshing of the density update."""
        if not self.kerker_q0 or self.gd is None:
            return r_G
        if self._filter is None:
            gd = self.gd
            ks = [2 * np.pi * np.fft.fftfreq(gd.N_c[c], gd.cell_cv[c, c] / gd.N_c[c])
                  for c in range(3)]
            k2 = (ks[0][:, None, None]**2 + ks[1][None, :, None]**2 +
                  ks[2][None, None, :]**2)
            f = k2 / (k2 + self.kerker_q0**2)
            f[0, 0, 0] = 1.0
            self._filter = torch.from_numpy(f).to(r_G.device)
        return torch.fft.ifftn(torch.fft.fftn(r_G) * self._filter).real

    def reset(self):
        self.count = 0
        self.nin_h = None
        self.res_h = None
        self.pres_h = None
        self.pos = None
        self._filter = None

    def mix(self, nin_G, nout_G, dv):
        if self.nin_h is None:
            shape = (self.nmaxold,) + tuple(nin_G.shape)
            self.nin_h = torch.zeros(shape, dtype=nin_G.dtype, device=nin_G.device)
            self.res_h = torch.zeros_like(self.nin_h)
            self.pres_h = torch.zeros_like(self.nin_h)
            self.pos = torch.zeros(1, dtype=torch.int64, device=nin_G.device)
        self.nin_h.index_copy_(0, self.pos, nin_G[None])
        r_G = nout_G - nin_G
        self.res_h.index_copy_(0, self.pos, r_G[None])
        self.pres_h.index_copy_(0, self.pos, self._precondition(r_G)[None])
        self.pos.add_(1).remainder_(self.nmaxold)
        self.count = min(self.count + 1, self.nmaxold)
        m = self.count
        R = self.res_h[:m].reshape(m, -1)
        M = torch.zeros((m + 1, m + 1), dtype=torch.float64, device=R.device)
        M[:m, :m] = (R @ R.T) * dv
        M[:m, m] = 1.0
        M[m, :m] = 1.0
        rhs = torch.zeros(m + 1, dtype=torch.float64, device=R.device)
        rhs[m:].fill_(1.0)     # slice fill: a device kernel, no host copy
        alpha, info = small_solve(M[None], rhs[None])
        alpha, info = alpha[0, :m], info[0]
        # a singular history falls back to the newest entry (no host check)
        newest = torch.zeros_like(alpha)
        newest.index_fill_(0, (self.pos - 1).remainder(self.nmaxold).clamp_max(m - 1), 1.0)
        alpha = torch.where((info == 0) & torch.isfinite(alpha).all(), alpha, newest)
        N = self.nin_h[:m].reshape(m, -1)
        P = self.pres_h[:m].reshape(m, -1)
        return (alpha.to(N.dtype) @ (N + self.beta * P)).reshape(nin_G.shape)


def _append_log_line(path, it, log, graphed):
    """One JSON object per iteration (JSON Lines): iteration, total energy
    (eV), eigenstate error (eV^2 per electron), density change (electrons
    per electron), wall time since the start (s), whether the iteration was
    a graph replay and the iteration of a learned-preconditioner fallback."""
    import json
    rec = {'iteration': it, 'energy_eV': log.energies[-1], 'eigenstate_error': log.errors[-1],
           'density_change': log.ddens[-1], 'time_s': round(log.times[-1], 6),
           'graphed': bool(graphed), 'fallback_at': log.fallback_at or None}
    with open(path, 'a') as f:
        f.write(json.dumps(rec) + '\n')


@dataclass
class SCFLog:
    energies: list = field(default_factory=list)
    errors: list = field(default_factory=list)
    ddens: list = field(default_factory=list)
    times: list = field(default_factory=list)
    converged: bool = False
    iterations: int = 0
    wall: float = 0.0
    graphed: bool = False
    fallback_at: int = 0


class Calculation:
    """FD-mode calculation of a fixed geometry.

    symbols, positions (Angstrom), cell (Angstrom, 3 or 3x3), pbc;
    h (Angstrom), nbands, xc ('LDA' or 'PBE'), precision 'fp64' | 'fp32',
    preconditioner None (multigrid) or an object with __call__(R, kpt),
    blocksize: RMM-DIIS band block (None = all bands per launch)."""

    def __init__(self, symbols, positions, cell, pbc, h=0.2, nbands=None,
                 xc='LDA', precision='fp64', k_c=None, preconditioner=None,
                 mixer_beta=None, seed=0, device='cuda', stencil=3,
                 r_gauss=0.6, kerker_q0=1.0, blocksize=None, kpts=None,
                 kbatch=True):
        cell = np.array(cell, float)
        cell_cv = np.diag(cell) if cell.ndim == 1 else cell
        self.cell_cv = cell_cv / Bohr
        self.pbc = np.array(pbc, bool) * np.ones(3, bool)
        N_c = h2gpts(h / Bohr, self.cell_cv)
        self.gd = GridDescriptor(N_c, self.cell_cv, self.pbc, device=device)
        self.finegd = self.gd.refine()
        self.spos_ac = np.linalg.solve(self.cell_cv.T, (np.asarray(positions) / Bohr).T).T
        if self.pbc.any():
            self.spos_ac[:, self.pbc] %= 1.0
        self.symbols = list(symbols)
        kinds = {s: HGHSetup(s, r_gauss=r_gauss) for s in set(self.symbols)}
        self.setups = [kinds[s] for s in self.symbols]
        self.nvalence = sum(s.Z for s in self.setups)
        nocc = self.nvalence // 2
        self.nbands = nbands or max(nocc + 4, int(1.2 * nocc))
        self.precision = precision
        # k-points: a Monkhorst-Pack grid reduced by time reversal, one given
        # k-point, or Gamma
        if kpts is not None:
            self.ibz_kc, self.w_k = irreducible_kpoints(monkhorst_pack(kpts))
        elif k_c is not None:
            self.ibz_kc, self.w_k = np.array([k_c], float), np.ones(1)
        else:
            self.ibz_kc, self.w_k = np.zeros((1, 3)), np.ones(1)
        # kbatch: every k-point in each launch (one batched KPoint); else one
        # KPoint per k-point, iterated in turn as the reference does
        self.kbatch = kbatch and len(self.ibz_kc) > 1
        if self.kbatch and blocksize is not None:
            raise ValueError('a k-point batch runs every band in one block (blocksize=None)')
        cplx = bool(np.any(self.ibz_kc))
        if precision == 'fp64':
            dtype = torch.complex128 if cplx else torch.float64
        else:
            dtype = torch.complex64 if cplx else torch.float32
        self.dtype = dtype
        kd = None
        if cplx:
            class _KD:
                pass
            kd = _KD()
            kd.ibzk_qc = self.ibz_kc
            kd.gamma = False
        self.wfs = FDWaveFunctions(self.gd, self.nbands, self.setups, self.spos_ac,
                                   dtype, stencil, kd)
        # fine-grid LFCs: short-range local potential, ion charges, density guess
        self.vbar = LFC(self.finegd, [[s.vbar] for s in self.setups], cut=True)
        self.vbar.set_positions(self.spos_ac)
        self.ghat = LFC(self.finegd, [[s.ghat] for s in self.setups], cut=True,
                        integral=[float(s.Z) for s in self.setups])
        self.ghat.set_positions(self.spos_ac)
        self.vbar_g = self.finegd.zeros()
        self.vbar.add(self.vbar_g, 1.0)
        self.rhoion_g = self.finegd.zeros()
        self.ghat.add(self.rhoion_g, -1.0)
        self.interpolator = Transformer(self.gd, self.finegd, 3)
        self.restrictor = Transformer(self.finegd, self.gd, 3)
        self.poisson = FastPoissonSolver(nn=3)
        self.poisson.set_grid_descriptor(self.finegd)
        self.xc = XC(xc)
        periodic = bool(self.pbc.all())
        self.mixer = PulayMixer(beta=mixer_beta or (0.25 if periodic else 0.25),
                                kerker_q0=kerker_q0 if periodic else None)
        self.mixer.gd = self.gd
        # blocksize None: every band in every launch (the batched form);
        # 10: the reference's default RMM-DIIS band blocks
        self.eigensolver = RMMDIIS(blocksize=blocksize)
        self.preconditioner = preconditioner or Preconditioner(
            self.gd, self.wfs.kin, complex if cplx else float, block=10)
        self.eigensolver.initialize(self.wfs, self.preconditioner)
        self.seed = seed
        self.k_c = self.ibz_kc[0]
        self.vHt_g = self.finegd.zeros()
        self.dH_MM = None
        self.e_constant = self._constant_energy()
        self._init_wavefunctions()
        self._init_density()

    # -------------------------------------------------------------- set-up
    def _init_wavefunctions(self):
        """Seeded pseudo-LCAO start: random combinations of atom-centred
        s and p Gaussians (LFC add), identical for every precision mode."""
        from gpaw_b200.spline import Spline
        r = np.linspace(0, 5.0, 201)
        g = np.exp(-r**2 / (2 * 1.2**2))
        basis = [[Spline.from_data(0, 5.0, g), Spline.from_data(1, 5.0, g)]
                 for _ in self.setups]
        cplx = self.dtype.is_complex
        kd = self.wfs.pt.kd if cplx else None
        lfc = LFC(self.gd, basis, kd=kd, dtype=complex if cplx else float, cut=True)
        lfc.set_positions(self.spos_ac)
        rng = np.random.default_rng(self.seed)
        M = lfc.Mmax
        work = torch.complex128 if cplx else torch.float64
        nk = len(self.ibz_kc)
        psit = self.gd.zeros(nk * self.nbands, dtype=work)
        for k in range(nk):
            c = rng.standard_normal((self.nbands, M))
            if cplx:
                c = c + 0.1j * rng.standard_normal(c.shape)
            c_axi = {a: torch.from_numpy(c[:, lfc.M_a[a]:lfc.M_a[a] + 4].copy()).to(
                self.gd.device, work) for a in range(len(self.setups))}
            part = psit[k * self.nbands:(k + 1) * self.nbands]
            lfc.add(part, c_axi, k if cplx else -1)
        # a little noise so that the start spans more than nbands' worth of LCAO space
        gen = torch.Generator(device=self.gd.device).manual_seed(self.seed)
        noise = torch.randn(psit.shape, generator=gen, device=self.gd.device,
                            dtype=torch.float64)
        psit += 0.01 * noise * psit.abs().max()
        psit = psit.to(self.dtype)
        nocc = self.nvalence // 2
        occ = np.array([2.0] * nocc + [0.0] * (self.nbands - nocc))
        phases = [self.gd.phase_factor_cd(k_c) if cplx else None for k_c in self.ibz_kc]
        if self.kbatch:
            kpt = KPoint(psit, q=range(nk), phase_cd=np.array(phases),
                         weight=np.repeat(self.w_k, self.nbands), k_c=self.ibz_kc, nk=nk)
            kpt.f_n = np.tile(occ, nk) * np.repeat(self.w_k, self.nbands)
            self.wfs.kpt_u = [kpt]
        else:
            self.wfs.kpt_u = []
            for k in range(nk):
                kpt = KPoint(psit[k * self.nbands:(k + 1) * self.nbands].clone(),
                             q=k if cplx else -1, phase_cd=phases[k], weight=self.w_k[k],
                             k_c=self.ibz_kc[k])
                kpt.f_n = occ * self.w_k[k]
                self.wfs.kpt_u.append(kpt)
        for kpt in self.wfs.kpt_u:
            self.wfs.orthonormalize(kpt)
        self.wfs.orthonormalized = True

    def _init_density(self):
        ng = LFC(self.gd, [[s.nguess] for s in self.setups], cut=True,
                 integral=[float(s.Z) for s in self.setups])
        ng.set_positions(self.spos_ac)
        self.nt_G = self.gd.zeros()
        ng.add(self.nt_G, 1.0)
        self.mixer.reset()

    # -------------------------------------------------------------- physics
    def update_hamiltonian(self):
        finegd = self.finegd
        nt_g = self.interpolator.apply(self.nt_G)
        # renormalise the fine density to the electron count (on the device)
        Ntot = nt_g.sum() * finegd.dv
        nt_g *= self.nvalence / Ntot.clamp_min(1e-300)
        rhot_g = nt_g + self.rhoion_g
        # a neutral system: the solver subtracts the mean (the uniform
        # background) and stays on the device
        self.poisson.solve(self.vHt_g, rhot_g, charge=0.0)
        vxc_g = torch.zeros((1,) + tuple(finegd.n_c), dtype=torch.float64,
                            device=finegd.device)
        e_g = finegd.empty()
        if self.xc.gd is not finegd:
            self.xc.set_grid_descriptor(finegd)
        self.xc.calculate_impl(finegd, nt_g[None], vxc_g, e_g)
        Exc = e_g.sum() * finegd.dv
        vt_g = self.vbar_g + self.vHt_g + vxc_g[0]
        vt_G = self.restrictor.apply(vt_g)
        # persistent state is updated in place (fixed addresses for replay)
        if getattr(self, 'vt_G', None) is None:
            self.vt_G = vt_G
            self.vt_G32 = vt_G.to(torch.float32)
        else:
            self.vt_G.copy_(vt_G)
            self.vt_G32.copy_(vt_G)
        if self.dH_MM is None:
            self.dH_MM = self._block_diagonal_dH()
        # energy terms stay FP64 device scalars (read once per iteration)
        e = torch.stack([0.5 * (rhot_g * self.vHt_g).sum() * finegd.dv, Exc,
                         (nt_g * self.vbar_g).sum() * finegd.dv])
        if getattr(self, 'e_terms', None) is None:
            self.e_terms = e
        else:
            self.e_terms.copy_(e)
        self.nt_g = nt_g
        self.vt_g = vt_g

    def _block_diagonal_dH(self):
        """dH^a_ij of every atom on the diagonal of one (Mmax x Mmax) FP64
        matrix, in the projector LFC's M order (the HGH dH_ij are
        density-independent, so this is built once)."""
        pt = self.wfs.pt
        dH = torch.zeros((pt.Mmax, pt.Mmax), dtype=torch.float64)
        for a, s in enumerate(self.setups):
            if s.ni:
                M = pt.M_a[a]
                dH[M:M + s.ni, M:M + s.ni] = torch.from_numpy(np.asarray(s.dH_ii, float))
        return dH.to(self.gd.device)

    def total_energy(self, kpt=None):
        """E = sum f eps - int nt vt + E_H + E_xc + E_vbar + E_0 (Hartree),
        all sums in FP64 (the band energy counts kinetic + nonlocal +
        local parts of the input potential); E_0 is the geometry constant
        of `_constant_energy`."""
        band = 0.0
        for k in (self.wfs.kpt_u if kpt is None or len(self.wfs.kpt_u) > 1 else [kpt]):
            if getattr(k, '_f_t', None) is None:
                k._f_t = torch.as_tensor(np.asarray(k.f_n, float), device=self.gd.device)
            band = band + (k._f_t * k.eps_n).sum()
        nvt = (self.nt_G * self.vt_G).sum() * self.gd.dv
        return band - nvt + self.e_terms.sum() + self.e_constant

    def _constant_energy(self):
        """The energy zero of the reference's HGH setups.  The Hartree term
        0.5 int rhot v_H contains each Gaussian ion charge's self-energy
        Z^2 / (2 sqrt(pi) s), which the reference removes through the setup
        constant M = -Eh_compcharge (gpaw/pseudopotential.py:293,
        gpaw/hgh.py:171-174); and its Gaussian-Gaussian interactions are
        those of widths s, where the reference's compensation charges have
        width r_loc (gpaw/hgh.py:102, 249-258): the difference
        sum_{a != b} Z_a Z_b [erf(R / w_loc) - erf(R / w_s)] / (2 R),
        w = sqrt(2 (s_a^2 + s_b^2)), summed over the neighbouring periodic
        images, is added.  No atomic reference energy is subtracted (the
        reference's HGH setups have E = 0)."""
        from scipy.special import erf
        setups = self.setups
        Z = np.array([s.Z for s in setups], float)
        rl = np.array([s.rloc for s in setups])
        sg = np.array([s.r_gauss for s in setups])
        e = -(Z**2 / (2 * np.sqrt(np.pi) * sg)).sum()
        pos_av = self.spos_ac @ self.cell_cv
        w_loc = np.sqrt(2 * (rl[:, None]**2 + rl[None, :]**2))
        w_s = np.sqrt(2 * (sg[:, None]**2 + sg[None, :]**2))
        ZZ = Z[:, None] * Z[None, :]
        shifts = [(-1, 0, 1) if p else (0,) for p in self.pbc]
        for n_c in itertools.product(*shifts):
            d = pos_av[None, :, :] + np.dot(n_c, self.cell_cv) - pos_av[:, None, :]
            R = np.linalg.norm(d, axis=2)
            if not any(n_c):
                np.fill_diagonal(R, np.inf)
            e += 0.5 * (ZZ * (erf(R / w_loc) - erf(R / w_s)) / R).sum()
        return float(e)

    def update_density(self):
        nt_out = self.gd.zeros()
        for kpt in self.wfs.kpt_u:
            self.wfs.add_to_density(nt_out, kpt)
        ddens = (nt_out - self.nt_G).abs().sum() * (self.gd.dv / self.nvalence)
        self.nt_G.copy_(self.mixer.mix(self.nt_G, nt_out, self.gd.dv))
        self.nt_G.clamp_(min=0.0)
        return ddens

    # -------------------------------------------------------------- driver
    def iteration(self):
        """One SCF iteration, eagerly: RMM-DIIS pass, energy, density mixing,
        new potential.  Returns the FP64 device vector [E (eV), eigenstate
        error, density change]."""
        err = self.eigensolver.iterate(self, self.wfs)
        E = self.total_energy() * Hartree
        ddens = self.update_density()
        self.update_hamiltonian()
        return torch.stack([E, err, ddens, self._judge_flag()])

    def _judge_flag(self):
        """1.0 when a judged (learned) preconditioner has failed its check
        against the multigrid, else 0.0 (a device scalar)."""
        failed = getattr(self.preconditioner, 'failed', None)
        if failed is None:
            return torch.zeros((), dtype=torch.float64, device=self.gd.device)
        return failed.to(torch.float64)

    def use_preconditioner(self, pc):
        self.preconditioner = pc
        self.eigensolver.preconditioner = pc

    def run(self, maxiter=200, energy_tol=1e-5, density_tol=1e-4,
            eigenstates_tol=4e-8, callback=None, graph=False, logfile=None):
        """Iterate to convergence: energy change (eV / valence electron)
        over the last 3 iterations < energy_tol, density change per
        electron < density_tol, eigenstate error (eV^2 / electron) <
        eigenstates_tol.

        graph=True replays each iteration as two captured CUDA graphs (the
        work before and after the subspace eigensolver, which runs eagerly
        between them) once the mixer history is full; the first iterations
        run eagerly.  Either way one iteration reads three scalars from the
        device and nothing else."""
        log = SCFLog()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        self.update_hamiltonian()
        step = None
        # a judged (learned) preconditioner: keep the state each iteration
        # starts from, so that an iteration its failure has made non-finite
        # can be taken back
        snap = (_Snapshot(self) if getattr(self.preconditioner, 'failed', None)
                is not None else None)
        for it in range(1, maxiter + 1):
            if snap is not None:
                snap.take()
            if graph and len(self.wfs.kpt_u) == 1 and self.mixer.count == self.mixer.nmaxold:
                if step is None:
                    step = _GraphedIteration(self)
                out = step.replay()
            else:
                out = self.iteration()
            E, err, ddens, failed = out.tolist()
            if failed > 0.5:
                # the multigrid judged the learned preconditioner off: go on
                # with the multigrid (and capture the step again if graphed)
                self.use_preconditioner(self.preconditioner.fallback)
                log.fallback_at = it
                if step is not None:
                    step.release()
                    step = None
                if not np.all(np.isfinite([E, err, ddens])):
                    # the failed iteration produced NaN / inf: restart it
                    # from the kept state with the multigrid
                    snap.restore()
                    snap = None
                    log.times.append(time.perf_counter() - t0)
                    log.iterations = it
                    continue
                snap = None
            log.energies.append(E)
            log.errors.append(err * Hartree**2 / self.nvalence)
            log.ddens.append(ddens)
            log.times.append(time.perf_counter() - t0)
            log.iterations = it
            if logfile is not None:
                _append_log_line(logfile, it, log, step is not None)
            if callback:
                callback(self, it, log)
            if it >= 3:
                dE = (max(log.energies[-3:]) - min(log.energies[-3:])) / self.nvalence
                if (dE < energy_tol and ddens < density_tol and
                        log.errors[-1] < eigenstates_tol):
                    log.converged = True
                    break
        log.wall = time.perf_counter() - t0
        log.graphed = step is not None
        if step is not None:
            step.release()
        self.log = log
        return log

    def eigenvalues(self):
        """eV: (nbands,) at Gamma / one k-point, (nk, nbands) otherwise."""
        out = []
        for kpt in self.wfs.kpt_u:
            eps = kpt.eps_n
            eps = eps.cpu().numpy() if isinstance(eps, torch.Tensor) else np.asarray(eps)
            out.append(eps.reshape(-1, self.nbands))
        eps = np.concatenate(out) * Hartree
        return eps[0] if len(eps) == 1 else eps

    # -------------------------------------------------------------- forces
    def forces(self):
        """Hellmann-Feynman forces (eV / Angstrom, natoms x 3) of the
        converged state: minus the derivative of the total energy with
        respect to each atom's position at fixed wave functions and density
        (the terms gpaw/forces.py collects from the wave functions, the
        local potential and the compensation charges,
        gpaw/wavefunctions/fdpw.py:426-450, gpaw/hamiltonian.py:408, 803):
          projectors     2 sum_n f_n sum_ij <psi_n|d p^a_i/dr> dH^a_ij P^a_nj
          vbar           int nt d vbar^a/dr
          ion charges    -(derivative of int v_H rhot through the Gaussian
                         ion charge -Z g/I(R), normalised on the grid)
          ion-ion        the geometry constant's gradient
        Evaluated in FP64 (an FP32 run's wave functions are widened first);
        the small per-atom reductions on the host."""
        natoms = len(self.setups)
        F = np.zeros((natoms, 3))
        pt = self.wfs.pt
        if pt.Mmax:
            F_Mv = torch.zeros((pt.Mmax, 3), dtype=torch.float64, device=self.gd.device)
            wide = torch.complex128 if self.dtype.is_complex else torch.float64
            for kpt in self.wfs.kpt_u:
                f_n = torch.as_tensor(np.asarray(kpt.f_n, float), device=self.gd.device)
                nk = getattr(kpt, 'nk', 1)
                nb = kpt.psit_nG.shape[0] // nk
                for k in range(nk):
                    rows = slice(k * nb, (k + 1) * nb)
                    q = (k if nk > 1 else kpt.q) if self.dtype.is_complex else -1
                    # projections and their derivatives from the state widened
                    # to FP64 (FP32 runs: the force sums stay FP64, like the
                    # energy sums)
                    psi = kpt.psit_nG[rows].to(wide).contiguous()
                    D = pt.derivative(psi, {}, q)
                    C = pt.integrate(psi, {}, q) @ self.dH_MM.to(wide).T
                    # 2 Re sum_n f_n conj(D_nMv) C_nM
                    F_Mv += 2 * (f_n[rows, None, None] * (D.conj() * C[:, :, None]).real).sum(0)
            F_Mv = F_Mv.cpu().numpy()
            for a in range(natoms):
                M = pt.M_a[a]
                F[a] += F_Mv[M:M + self.setups[a].ni].sum(0)
        # local potential: d/dR int nt vbar = -int nt dvbar/dr
        Dv = self.vbar.derivative(self.nt_g, {}).cpu().numpy()      # (natoms, 3)
        F += Dv
        # ion charges rho_a = -Z g(r - R) / I(R), I = dv sum_g g:
        # dE/dR = Z [D(v_H) / I - A(v_H) D(1) / I^2] with D(a) = dv sum a dg/dr,
        # A(a) = dv sum a g
        raw = self._ghat_raw()
        one = torch.ones_like(self.vHt_g)
        D_v = raw.derivative(self.vHt_g, {}).cpu().numpy()
        D_1 = raw.derivative(one, {}).cpu().numpy()
        A_v = raw.integrate(self.vHt_g, {}).cpu().numpy()
        I = raw.integrate(one, {}).cpu().numpy()
        Z = np.array([s.Z for s in self.setups], float)
        F -= Z[:, None] * (D_v / I[:, None] - A_v[:, None] * D_1 / I[:, None]**2)
        F -= self._constant_energy_gradient()
        return F * Hartree / Bohr

    def _ghat_raw(self):
        """The ion-charge functions without their grid normalisation."""
        if getattr(self, '_ghat_unnormalised', None) is None:
            g = LFC(self.finegd, [[s.ghat] for s in self.setups], cut=True)
            g.set_positions(self.spos_ac)
            self._ghat_unnormalised = g
        return self._ghat_unnormalised

    def _constant_energy_gradient(self):
        """d E_0 / d R_a (Hartree / Bohr) of `_constant_energy`."""
        from scipy.special import erf
        setups = self.setups
        Z = np.array([s.Z for s in setups], float)
        rl = np.array([s.rloc for s in setups])
        sg = np.array([s.r_gauss for s in setups])
        pos_av = self.spos_ac @ self.cell_cv
        w1 = np.sqrt(2 * (rl[:, None]**2 + rl[None, :]**2))
        w2 = np.sqrt(2 * (sg[:, None]**2 + sg[None, :]**2))
        ZZ = Z[:, None] * Z[None, :]
        G = np.zeros((len(setups), 3))
        shifts = [(-1, 0, 1) if p else (0,) for p in self.pbc]

        def phi_prime(R, w):
            # d/dR [erf(R / w) / R]
            return (2 / np.sqrt(np.pi) * np.exp(-(R / w)**2) / (w * R) -
                    erf(R / w) / R**2)
        for n_c in itertools.product(*shifts):
            d = pos_av[None, :, :] + np.dot(n_c, self.cell_cv) - pos_av[:, None, :]
            R = np.linalg.norm(d, axis=2)
            if not any(n_c):
                np.fill_diagonal(R, np.inf)
            dphi = ZZ * (phi_prime(R, w1) - phi_prime(R, w2))
            # E_0 = 1/2 sum_ab phi(|R_b + n - R_a|): d/dR_a picks both ends
            G -= (dphi[:, :, None] * d / R[:, :, None]).sum(1)
        return G


def monkhorst_pack(size):
    """The Monkhorst-Pack grid of size n1 x n2 x n3 (scaled k-points),
    (i + 1/2) / n - 1/2 along each axis."""
    size = np.asarray(size, int)
    return (np.indices(size).reshape(3, -1).T + 0.5) / size - 0.5


def irreducible_kpoints(k_kc, tol=1e-8):
    """Reduce by time reversal only (psi_-k = psi_k^*, so k and -k give
    the same density and energies): (ibz_kc, weights), weights summing to
    one.  Point-group symmetry is not used."""
    ibz, w = [], []
    for k in k_kc:
        for i, q in enumerate(ibz):
            d = k + q
            if np.all(np.abs(d - np.round(d)) < tol):
                w[i] += 1
                break
        else:
            ibz.append(np.array(k, float))
            w.append(1)
    w = np.array(w, float)
    return np.array(ibz), w / w.sum()


def si_diamond(ncell=1, a=5.43, rattle=0.0, seed=0):
    """Diamond Si, ncell^3 conventional cells (8 atoms each)."""
    base = np.array([[0, 0, 0], [0, 0.5, 0.5], [0.5, 0, 0.5], [0.5, 0.5, 0],
                     [0.25, 0.25, 0.25], [0.25, 0.75, 0.75], [0.75, 0.25, 0.75],
                     [0.75, 0.75, 0.25]])
    pos = []
    for i in range(ncell):
        for j in range(ncell):
            for k in range(ncell):
                pos.extend((base + [i, j, k]) * a)
    pos = np.array(pos)
    if rattle:
        pos += np.random.default_rng(seed).normal(0.0, rattle, pos.shape)
    L = ncell * a
    return ['Si'] * len(pos), pos, [L, L, L]


def h2o_cluster(nx=4, ny=4, nz=2, spacing=3.1, box=15.0, jitter=0.1, seed=0,
                d_oh=0.96, angle=104.5):
    """(H2O)_{nx ny nz} cluster: water molecules (O-H d_oh, H-O-H angle) with
    seeded uniformly random orientations (a random rotation from the QR
    decomposition of a Gaussian matrix, sign-fixed), centred on an
    nx x ny x nz lattice of the given spacing plus seeded Gaussian jitter,
    the lattice centred in a cubic box of side `box` (Angstrom).  The
    32-molecule precision configuration is the default."""
    rng = np.random.default_rng(seed)
    t = np.radians(angle) / 2
    mol = np.array([[0.0, 0.0, 0.0],
                    [d_oh * np.sin(t), 0.0, d_oh * np.cos(t)],
                    [-d_oh * np.sin(t), 0.0, d_oh * np.cos(t)]])
    mol -= mol.mean(0)
    sym, pos = [], []
    lat = np.array([(i, j, k) for i in range(nx) for j in range(ny) for k in range(nz)],
                   float) * spacing
    lat += box / 2 - lat.mean(0)
    for c in lat:
        q, r = np.linalg.qr(rng.standard_normal((3, 3)))
        q = q * np.sign(np.diag(r))
        if np.linalg.det(q) < 0:
            q[:, 0] = -q[:, 0]
        centre = c + rng.normal(0.0, jitter, 3)
        for s, p in zip(('O', 'H', 'H'), mol @ q.T + centre):
            sym.append(s)
            pos.append(p)
    return sym, np.array(pos), [box, box, box]


def h2(vacuum=3.0, d=0.74):
    """H2 along z, `vacuum` on every side (the H2 FD configuration)."""
    cell = [2 * vacuum, 2 * vacuum, 2 * vacuum + d]
    pos = np.array([[vacuum, vacuum, vacuum], [vacuum, vacuum, vacuum + d]])
    return ['H', 'H'], pos, cell


class _Snapshot:
    """The state an SCF iteration starts from (wave functions, projections,
    eigenvalues, density), copied on the device before each iteration while
    a judged preconditioner is in use.  `restore` puts it back, restarts the
    density mixing and rebuilds the potential from the kept density."""

    def __init__(self, calc):
        self.calc = calc
        self.kept = None

    def take(self):
        kpt = self.calc.wfs.kpt_u[0]
        items = [kpt.psit_nG, kpt.P_nM, kpt.eps_n, self.calc.nt_G]
        if self.kept is None or any(
                (a is None) != (b is None) or (a is not None and a.shape != b.shape)
                for a, b in zip(items, self.kept)):
            self.kept = [None if a is None else torch.empty_like(a) for a in items]
        for dst, src in zip(self.kept, items):
            if src is not None:
                dst.copy_(src)

    def restore(self):
        calc = self.calc
        kpt = calc.wfs.kpt_u[0]
        psit, P, eps, nt = self.kept
        kpt.psit_nG.copy_(psit)
        if P is not None:
            kpt.P_nM.copy_(P)
        if eps is not None:
            kpt.eps_n = eps.clone()
        calc.nt_G.copy_(nt)
        calc.mixer.reset()
        calc.update_hamiltonian()


_POOL = None
_POOL_KEEPER = None
_CAPTURE_STREAM = None


def _capture_stream():
    """The one side stream every capture of the process runs on.  The
    caching allocator reuses a free block only for allocations on the stream
    it was allocated on, and torch.cuda.Stream() hands out its pooled
    streams in turn, so a fresh stream per capture found none of the blocks
    the previous captures gave back and allocated new segments every time
    (14-18 per Si64 capture, 5-77 ms)."""
    global _CAPTURE_STREAM
    if _CAPTURE_STREAM is None:
        _CAPTURE_STREAM = torch.cuda.Stream()
    return _CAPTURE_STREAM


def _graph_pool():
    """One private memory pool for every captured SCF step of the process:
    the blocks a released graph gave back are there for the next capture,
    which then allocates (almost) nothing new.  torch retires a pool once no
    graph uses it, so a one-op graph captured into it at creation stays
    alive for the process and keeps the pool."""
    global _POOL, _POOL_KEEPER
    if _POOL is None:
        pool = torch.cuda.graph_pool_handle()
        x = torch.zeros(1, device='cuda')
        keep = torch.cuda.CUDAGraph()
        side = _capture_stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            keep.capture_begin(pool=pool)
            x.add_(1.0)
            keep.capture_end()
        torch.cuda.current_stream().wait_stream(side)
        _POOL, _POOL_KEEPER = pool, (keep, x)
    return _POOL


class _GraphedIteration:
    """One SCF iteration as two CUDA graphs around the subspace eigensolver.

    Graph A: (T + v) psi and the FP64 subspace matrix H.  Then eigh(H) runs
    eagerly (torch's eigh checks its info flag on the host) and writes into
    fixed eigenvalue / eigenvector buffers.  Graph B: rotation, residuals,
    the RMM-DIIS pass with its preconditioner calls, orthonormalisation,
    energy, density and mixing, the new potential, and the copy of the new
    wave functions and projections back into the buffers graph A reads.
    Persistent SCF state (density, potential, energy terms, mixer history)
    is updated in place by the eager code already, so its addresses do not
    change between replays."""

    def __init__(self, calc):
        self.calc = calc
        wfs = calc.wfs
        kpt = wfs.kpt_u[0]
        es = calc.eigensolver
        weights = es.weights(kpt, wfs)
        self.psit = kpt.psit_nG
        self.P = kpt.P_nM
        nb = self.psit.shape[0]
        nk = getattr(kpt, 'nk', 1)
        wide = torch.complex128 if wfs.dtype.is_complex else torch.float64
        self.eps = torch.empty(nb, dtype=torch.float64, device=self.psit.device)
        # one eigenvector block per k-point of a batch
        vshape = (nk, nb // nk, nb // nk) if nk > 1 else (nb, nb)
        self.V = torch.empty(vshape, dtype=wide, device=self.psit.device)
        self.pool = _graph_pool()
        # capture on a side stream with capture_begin/capture_end (the
        # torch.cuda.graph context manager would also run gc.collect() and
        # empty the allocator's cache, whose re-filling costs far more than
        # the capture itself)
        side = _capture_stream()
        side.wait_stream(torch.cuda.current_stream())
        self.gA = torch.cuda.CUDAGraph()
        self.gB = torch.cuda.CUDAGraph()
        # no cyclic garbage collection while capturing: a collection would
        # pause the host for as long as the heap is big and could free
        # device tensors in the middle of the capture
        gc_on = gc.isenabled()
        gc.disable()
        try:
            with torch.cuda.stream(side):
                self.gA.capture_begin(pool=self.pool)
                self.H, self.Htpsit = es.subspace_matrix(calc, wfs, kpt)
                self.gA.capture_end()
                self.gB.capture_begin(pool=self.pool)
                self._capture_b(calc, wfs, kpt, es, weights)
                self.gB.capture_end()
        finally:
            if gc_on:
                gc.enable()
        torch.cuda.current_stream().wait_stream(side)
        kpt.psit_nG = self.psit
        kpt.P_nM = self.P
        kpt.eps_n = self.eps

    def _capture_b(self, calc, wfs, kpt, es, weights):
        es.subspace_rotate(wfs, kpt, self.eps, self.V, self.Htpsit)
        err = es.update_bands(calc, wfs, kpt, weights)
        wfs.orthonormalize(kpt, out=self.psit)
        E = calc.total_energy(kpt) * Hartree
        ddens = calc.update_density()
        calc.update_hamiltonian()
        if kpt.psit_nG.data_ptr() != self.psit.data_ptr():
            self.psit.copy_(kpt.psit_nG)
        if self.P is not None:
            self.P.copy_(kpt.P_nM)
        self.out = torch.stack([E, err, ddens, calc._judge_flag()])

    def replay(self):
        self.gA.replay()
        eps, V = torch.linalg.eigh(self.H)
        self.eps.copy_(eps.reshape(-1))
        self.V.copy_(V)
        self.gB.replay()
        return self.out

    def release(self):
        torch.cuda.synchronize()
        self.gA.reset()
        self.gB.reset()
