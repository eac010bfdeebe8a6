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
Energies exclude the constant ion-ion term (irrelevant for convergence and
for comparing precision modes of one geometry).
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np
import torch

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
    gpaw/mixer.py:35-; plain Euclidean metric)."""

    def __init__(self, beta=0.1, nmaxold=5, kerker_q0=None):
        self.beta = beta
        self.nmaxold = nmaxold
        self.kerker_q0 = kerker_q0
        self.gd = None
        self.nin = []
        self.res = []

    def _precondition(self, r_G):
        """Kerker filter k^2 / (k^2 + q0^2) on the residual (periodic cells):
        damps the long-wavelength charge sloshing of the density update."""
        if not self.kerker_q0 or self.gd is None:
            return r_G
        gd = self.gd
        ks = [2 * np.pi * np.fft.fftfreq(gd.N_c[c], gd.cell_cv[c, c] / gd.N_c[c])
              for c in range(3)]
        k2 = (ks[0][:, None, None]**2 + ks[1][None, :, None]**2 +
              ks[2][None, None, :]**2)
        f = torch.from_numpy(k2 / (k2 + self.kerker_q0**2)).to(r_G.device)
        f[0, 0, 0] = 1.0
        return torch.fft.ifftn(torch.fft.fftn(r_G) * f).real

    def reset(self):
        self.nin, self.res = [], []

    def mix(self, nin_G, nout_G, dv):
        self.nin.append(nin_G.clone())
        self.res.append(nout_G - nin_G)
        if len(self.nin) > self.nmaxold:
            self.nin.pop(0)
            self.res.pop(0)
        m = len(self.res)
        R = torch.stack([r.reshape(-1) for r in self.res])
        A = (R @ R.T) * dv
        M = torch.zeros((m + 1, m + 1), dtype=torch.float64, device=R.device)
        M[:m, :m] = A
        M[:m, m] = 1.0
        M[m, :m] = 1.0
        rhs = torch.zeros(m + 1, dtype=torch.float64, device=R.device)
        rhs[m] = 1.0
        try:
            alpha = torch.linalg.solve(M, rhs)[:m]
        except RuntimeError:
            alpha = torch.zeros(m, dtype=torch.float64, device=R.device)
            alpha[-1] = 1.0
        new = torch.zeros_like(nin_G)
        for a, n, r in zip(alpha, self.nin, self.res):
            new += a * (n + self.beta * self._precondition(r))
        return new


@dataclass
class SCFLog:
    energies: list = field(default_factory=list)
    errors: list = field(default_factory=list)
    ddens: list = field(default_factory=list)
    times: list = field(default_factory=list)
    converged: bool = False
    iterations: int = 0
    wall: float = 0.0


class Calculation:
    """FD-mode calculation of a fixed geometry.

    symbols, positions (Angstrom), cell (Angstrom, 3 or 3x3), pbc;
    h (Angstrom), nbands, xc ('LDA' or 'PBE'), precision 'fp64' | 'fp32',
    preconditioner None (multigrid) or an object with __call__(R, kpt)."""

    def __init__(self, symbols, positions, cell, pbc, h=0.2, nbands=None,
                 xc='LDA', precision='fp64', k_c=None, preconditioner=None,
                 mixer_beta=None, seed=0, device='cuda', stencil=3,
                 r_gauss=0.6, kerker_q0=1.0):
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
        cplx = k_c is not None and np.any(k_c)
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
            kd.ibzk_qc = np.array([k_c], float)
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
        self.eigensolver = RMMDIIS()
        self.preconditioner = preconditioner or Preconditioner(
            self.gd, self.wfs.kin, complex if cplx else float, block=10)
        self.eigensolver.initialize(self.wfs, self.preconditioner)
        self.seed = seed
        self.k_c = np.zeros(3) if k_c is None else np.asarray(k_c, float)
        self.vHt_g = self.finegd.zeros()
        self.dH_aii = None
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
        c = rng.standard_normal((self.nbands, M))
        if cplx:
            c = c + 0.1j * rng.standard_normal(c.shape)
        work = torch.complex128 if cplx else torch.float64
        psit = self.gd.zeros(self.nbands, dtype=work)
        c_axi = {a: torch.from_numpy(c[:, lfc.M_a[a]:lfc.M_a[a] + 4].copy()).to(
            self.gd.device, work) for a in range(len(self.setups))}
        lfc.add(psit, c_axi, 0 if cplx else -1)
        # a little noise so that the start spans more than nbands' worth of LCAO space
        gen = torch.Generator(device=self.gd.device).manual_seed(self.seed)
        noise = torch.randn(psit.shape, generator=gen, device=self.gd.device,
                            dtype=torch.float64)
        psit += 0.01 * noise * psit.abs().max()
        phase = self.gd.phase_factor_cd(self.k_c) if cplx else None
        kpt = KPoint(psit.to(self.dtype), q=0 if cplx else -1, phase_cd=phase,
                     weight=1.0, k_c=self.k_c)
        nocc = self.nvalence // 2
        kpt.f_n = np.array([2.0] * nocc + [0.0] * (self.nbands - nocc))
        self.wfs.kpt_u = [kpt]
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
        # renormalise the fine density to the electron count
        Ntot = float(nt_g.sum()) * finegd.dv
        if Ntot > 0:
            nt_g *= self.nvalence / Ntot
        rhot_g = nt_g + self.rhoion_g
        if self.pbc.all():
            rhot_g = rhot_g - rhot_g.mean()
        self.poisson.solve(self.vHt_g, rhot_g)
        vxc_g = torch.zeros((1,) + tuple(finegd.n_c), dtype=torch.float64,
                            device=finegd.device)
        e_g = finegd.empty()
        Exc = self.xc.calculate(finegd, nt_g[None], vxc_g, e_g)
        vt_g = self.vbar_g + self.vHt_g + vxc_g[0]
        self.vt_G = self.restrictor.apply(vt_g)
        self.vt_G32 = self.vt_G.to(torch.float32)
        self.dH_aii = {a: torch.from_numpy(s.dH_ii).to(self.gd.device)
                       for a, s in enumerate(self.setups) if s.ni > 0}
        self.e_hartree = 0.5 * float((rhot_g * self.vHt_g).sum()) * finegd.dv
        self.e_xc = float(Exc)
        self.e_vbar = float((nt_g * self.vbar_g).sum()) * finegd.dv
        self.nt_g = nt_g
        self.vt_g = vt_g

    def total_energy(self, kpt):
        """E = sum f eps - int nt vt + E_H + E_xc + E_vbar (Hartree),
        all sums in FP64 (the band energy counts kinetic + nonlocal +
        local parts of the input potential)."""
        band = float(np.dot(kpt.f_n, kpt.eps_n))
        nvt = float((self.nt_G * self.vt_G).sum()) * self.gd.dv
        e_kin_nl = band - nvt
        return e_kin_nl + self.e_hartree + self.e_xc + self.e_vbar

    def update_density(self):
        nt_out = self.gd.zeros()
        for kpt in self.wfs.kpt_u:
            self.wfs.add_to_density(nt_out, kpt)
        ddens = float((nt_out - self.nt_G).abs().sum()) * self.gd.dv / self.nvalence
        self.nt_G = self.mixer.mix(self.nt_G, nt_out, self.gd.dv)
        self.nt_G.clamp_(min=0.0)
        return ddens

    # -------------------------------------------------------------- driver
    def run(self, maxiter=200, energy_tol=1e-5, density_tol=1e-4,
            eigenstates_tol=4e-8, callback=None):
        """Iterate to convergence: energy change (eV / valence electron)
        over the last 3 iterations < energy_tol, density change per
        electron < density_tol, eigenstate error (eV^2 / electron) <
        eigenstates_tol."""
        log = SCFLog()
        kpt = self.wfs.kpt_u[0]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        self.update_hamiltonian()
        for it in range(1, maxiter + 1):
            err = self.eigensolver.iterate(self, self.wfs)
            E = self.total_energy(kpt) * Hartree
            ddens = self.update_density()
            self.update_hamiltonian()
            torch.cuda.synchronize()
            log.energies.append(E)
            log.errors.append(err * Hartree**2 / self.nvalence)
            log.ddens.append(ddens)
            log.times.append(time.perf_counter() - t0)
            log.iterations = it
            if callback:
                callback(self, it, log)
            if it >= 3:
                dE = (max(log.energies[-3:]) - min(log.energies[-3:])) / self.nvalence
                if (dE < energy_tol and ddens < density_tol and
                        log.errors[-1] < eigenstates_tol):
                    log.converged = True
                    break
        log.wall = time.perf_counter() - t0
        self.log = log
        return log

    def eigenvalues(self):
        return np.asarray(self.wfs.kpt_u[0].eps_n) * Hartree


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


def h2(vacuum=3.0, d=0.74):
    """H2 along z, `vacuum` on every side (the H2 FD configuration)."""
    cell = [2 * vacuum, 2 * vacuum, 2 * vacuum + d]
    pos = np.array([[vacuum, vacuum, vacuum], [vacuum, vacuum, vacuum + d]])
    return ['H', 'H'], pos, cell
