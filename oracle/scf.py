"""ORACLE (test infrastructure): the FD SCF of the device code on the CPU.

The same algorithm as the device SCF (norm-conserving HGH setups, Gamma
point, FP64), assembled from GPAW's own C kernels built from the reference
sources into oracle/_ref --

  _gpaw.Operator       kinetic stencil (Laplace(-1/2, 3)) and the nn=2
                       gradients of the GGA driver
  _gpaw.Transformer    coarse <-> fine density / potential transfers (nn=3)
                       and the V-cycle's transfers (nn=1)
  _gpaw.fd_precond     the multigrid preconditioner
  _gpaw.Spline, spline_to_grid, LFC    projectors, vbar, ion charges, density
                       guess (boxes and volumes as gpaw/lfc.py:259-374 builds
                       them, sphere normalisation gpaw/lfc.py:125-175)
  _gpaw.XCFunctional   LDA / PBE point kernels
  _gpaw.add_to_density density accumulation

-- and numpy restatements of the reference's Python glue:

  RMM-DIIS                 gpaw/eigensolvers/rmmdiis.py:63-272
  residuals, subspace      gpaw/eigensolvers/eigensolver.py:121-236
  orthonormalisation       gpaw/wavefunctions/fdpw.py:394-424
  boxes                    gpaw/grid_descriptor.py:344-411
  Poisson                  oracle/poisson.py (gpaw/poisson.py:842-1007)
  GGA driver               gpaw/xc/gga.py:106-163, 177-200

plus the device SCF's own density mixing (Pulay over the last five
densities, Kerker filter on periodic cells), density renormalisation and
energy expression, restated in numpy.  Setups, geometry and the starting
wave functions are inputs: `setups` holds per atom the plain radial data
of a setup (valence charge Z, Gaussian width, vbar / ion-charge / density
guess / projector splines as (l, rmax, f_g), and dH_ii).
"""
from __future__ import annotations

from math import pi, sqrt

import numpy as np

from oracle import fd, poisson, ref

HARTREE = 27.211386024367243


# ---------------------------------------------------------------- geometry
class Grid(fd.Grid):
    def __init__(self, N_c, cell_cv, pbc_c):
        super().__init__(N_c, cell_cv, pbc_c)
        self.icell_cv = np.linalg.inv(self.cell_cv).T

    def refine(self):
        return Grid(self.N_c * 2, self.cell_cv, self.pbc_c)

    def coarsen(self):
        return Grid(self.N_c // 2, self.cell_cv, self.pbc_c)


def boxes(g: Grid, spos_c, rcut):
    """(beg_c, end_c, sdisp_c) of every periodic image box a sphere of
    radius rcut at spos_c covers, cut at zero boundaries
    (gpaw/grid_descriptor.py:344-411 with cut=True)."""
    N_c = g.N_c
    ncut = rcut * np.sqrt((g.icell_cv**2).sum(1)) * N_c
    npos = np.asarray(spos_c) * N_c
    beg = np.ceil(npos - ncut).astype(int)
    end = np.ceil(npos + ncut).astype(int)
    for c in range(3):
        if not g.pbc_c[c]:
            beg[c] = max(beg[c], 0)
            end[c] = min(end[c], N_c[c])
    ranges = []
    for c in range(3):
        rc = []
        b = beg[c]
        e = b
        while e < end[c]:
            b0 = b % N_c[c]
            e = min(end[c], b + N_c[c] - b0)
            b1 = b + g.beg_c[c] - b0 if b0 < g.beg_c[c] else b
            e0 = b0 - b + e
            e1 = e - (e0 - g.end_c[c]) if e0 > g.end_c[c] else e
            if e1 > b1:
                rc.append((b1, e1))
            b = e
        ranges.append(rc)
    out = []
    for r0 in ranges[0]:
        for r1 in ranges[1]:
            for r2 in ranges[2]:
                b = np.array([r0[0], r1[0], r2[0]])
                e = np.array([r0[1], r1[1], r2[1]])
                bb = b % N_c
                ee = bb + e - b
                disp = (b - bb) // N_c
                bb = np.maximum(bb, g.beg_c)
                ee = np.minimum(ee, g.end_c)
                if np.all(bb < ee):
                    out.append((bb, ee, disp))
    return out


# ---------------------------------------------------------------- LFC
class LFC:
    """_gpaw.LFC over per-atom spline lists; M order: atom, spline, m."""

    def __init__(self, g: Grid, splines_a, spos_ac, integral=None):
        gp = ref.load()
        self.g = g
        A_W, M_W, G_l, W_l = [], [], [], []
        self.M_a = []
        M = 0
        W = 0
        self.spline_M = []      # _gpaw.Spline per M (LFC.derivative's argument)
        pos_W = []
        for a, spl in enumerate(splines_a):
            self.M_a.append(M)
            A_w, Mw_w = [], []
            Ml = 0
            for (l, rmax, f_g) in spl:
                f = np.array(f_g, float)
                f[-1] = 0.0
                s = gp.Spline(int(l), float(rmax), f)
                self.spline_M.extend([s] * (2 * int(l) + 1))
                for beg, end, sdisp in boxes(g, spos_ac[a], rmax):
                    pos_v = (np.asarray(spos_ac[a]) - sdisp) @ g.cell_cv
                    A_gm, G_b = gp.spline_to_grid(s, beg, end, pos_v,
                                                  np.ascontiguousarray(g.h_cv),
                                                  g.n_c, g.beg_c)
                    if len(G_b) == 0:
                        continue
                    A_w.append(A_gm)
                    Mw_w.append(Ml)
                    G_l.append(G_b)
                    pos_W.append(pos_v)
                    w = np.empty(len(G_b), np.intc)
                    w[0::2] = W
                    w[1::2] = -W - 1
                    W_l.append(w)
                    W += 1
                Ml += 2 * l + 1
            if integral is not None and A_w and integral[a] >= 1e-15:
                # sphere normalisation (gpaw/lfc.py:125-175)
                I_M = np.zeros(Ml)
                for Mw, A_gm in zip(Mw_w, A_w):
                    I_M[Mw:Mw + A_gm.shape[1]] += A_gm.sum(0) * g.dv
                nw = len(A_w) // len(spl)
                for w, (Mw, A_gm) in enumerate(zip(Mw_w, A_w)):
                    if Mw == 0:
                        A_gm *= integral[a] / I_M[0]
                    else:
                        A_gm -= I_M[Mw:Mw + A_gm.shape[1]] / integral[a] * A_w[w % nw]
            A_W.extend(A_w)
            M_W.extend(M + m for m in Mw_w)
            M += Ml
        self.Mmax = M
        self.pos_Wv = np.ascontiguousarray(np.array(pos_W).reshape(-1, 3), float)
        if not A_W:                 # no functions (e.g. H has no projectors)
            self.lfc = None
            return
        G_B = np.concatenate(G_l)
        W_B = np.concatenate(W_l)
        idx = np.argsort(G_B, kind='mergesort')
        # the C object keeps pointers into these arrays: hold them
        self.A_W = A_W
        self.G_B = np.ascontiguousarray(G_B[idx], np.intc)
        self.W_B = np.ascontiguousarray(W_B[idx], np.intc)
        self.phase_qW = np.empty((0, W), complex)
        self.lfc = gp.LFC(A_W, np.array(M_W, np.intc), self.G_B, self.W_B, g.dv,
                          self.phase_qW)

    def add(self, a_xG, c_xM):
        if self.lfc is not None:
            self.lfc.add(np.ascontiguousarray(c_xM), a_xG, -1)

    def integrate(self, a_xG):
        c = np.zeros(a_xG.shape[:-3] + (self.Mmax,))
        if self.lfc is not None:
            self.lfc.integrate(np.ascontiguousarray(a_xG), c, -1)
        return c

    def derivative(self, a_xG):
        """dv sum_G a_xG dPhi_M/dr_v: the reference's LFC.derivative with
        the arguments gpaw/lfc.py:660-682 builds."""
        c = np.zeros(a_xG.shape[:-3] + (self.Mmax, 3))
        if self.lfc is not None:
            g = self.g
            self.lfc.derivative(np.ascontiguousarray(a_xG), c,
                                np.ascontiguousarray(g.h_cv), g.n_c, self.spline_M,
                                g.beg_c, self.pos_Wv, -1)
        return c


def transformer(gin: Grid, gout: Grid, nn):
    restrict = bool((gin.N_c == 2 * gout.N_c).all())
    pad, npad, skip = fd.transformer_geometry(gin.beg_c, gin.end_c, gout.beg_c,
                                              gout.end_c, nn, restrict)
    t = ref.transformer(gin.n_c, gout.n_c, nn, pad, npad, skip, gin.pbc_c, True,
                        not restrict)

    def apply(a):
        a = np.ascontiguousarray(a)
        out = np.zeros(a.shape[:-3] + tuple(gout.n_c))
        t.apply(a, out)
        return out
    return apply


def operator(g: Grid, coef_offset):
    op = ref.operator(*coef_offset, g.n_c, g.pbc_c, True)

    def apply(a):
        a = np.ascontiguousarray(a)
        out = np.zeros_like(a)
        op.apply(a, out)
        return out
    apply.diagonal = op.get_diagonal_element()
    return apply


class Preconditioner:
    """_gpaw.fd_precond with the three levels of gpaw/preconditioner.py:
    Laplace(-1/2, 3) on the finest, Laplace(-1/2, 1) below, nn=1
    transfers, step = 0.66666666 / diagonal."""

    def __init__(self, g0: Grid, kin0_coefs):
        gp = ref.load()
        gs = [g0, g0.coarsen(), g0.coarsen().coarsen()]
        self.gs = gs
        kin = [kin0_coefs] + [fd.guc_laplace(g.h_cv, -0.5, 1) for g in gs[1:]]
        self.ops = [ref.operator(*k, g.n_c, g.pbc_c, True) for k, g in zip(kin, gs)]

        def T(gi, go):
            r = bool((gi.N_c == 2 * go.N_c).all())
            pad, npad, skip = fd.transformer_geometry(gi.beg_c, gi.end_c, go.beg_c,
                                                      go.end_c, 1, r)
            return ref.transformer(gi.n_c, go.n_c, 1, pad, npad, skip, gi.pbc_c,
                                   True, not r)
        self.T = (T(gs[0], gs[1]), T(gs[1], gs[2]), T(gs[1], gs[0]), T(gs[2], gs[1]))
        self.step = 0.66666666 / self.ops[0].get_diagonal_element()
        self.gp = gp

    def __call__(self, R):
        R = np.ascontiguousarray(R)
        B = R.shape[0]
        g0, g1, g2 = self.gs
        d0 = np.zeros_like(R)
        q0 = np.zeros_like(R)
        w1 = [np.zeros((B,) + tuple(g1.n_c)) for _ in range(3)]
        w2 = [np.zeros((B,) + tuple(g2.n_c)) for _ in range(3)]
        rest0, rest1, intp1, intp2 = self.T
        self.gp.fd_precond(rest0, rest1, intp1, intp2, *self.ops, d0, q0, *w1, *w2,
                           R, np.ascontiguousarray(-R), self.step)
        return d0


# ---------------------------------------------------------------- mixing
class PulayMixer:
    """The device SCF's density mixing: Pulay (DIIS) over the last nmaxold
    (input density, residual) pairs with a plain metric, the update built
    from Kerker-filtered residuals k^2 / (k^2 + q0^2) on periodic cells;
    a singular history falls back to the newest entry."""

    def __init__(self, g: Grid, beta, nmaxold=5, kerker_q0=None):
        self.beta = beta
        self.nmaxold = nmaxold
        self.filter = None
        if kerker_q0:
            ks = [2 * pi * np.fft.fftfreq(g.N_c[c], g.cell_cv[c, c] / g.N_c[c])
                  for c in range(3)]
            k2 = (ks[0][:, None, None]**2 + ks[1][None, :, None]**2 +
                  ks[2][None, None, :]**2)
            f = k2 / (k2 + kerker_q0**2)
            f[0, 0, 0] = 1.0
            self.filter = f
        self.reset()

    def reset(self):
        self.hist = []

    def mix(self, nin, nout, dv):
        r = nout - nin
        pr = r if self.filter is None else np.real(np.fft.ifftn(np.fft.fftn(r) * self.filter))
        self.hist.append((nin.copy(), r, pr))
        self.hist = self.hist[-self.nmaxold:]
        m = len(self.hist)
        R = np.array([h[1].ravel() for h in self.hist])
        A = np.zeros((m + 1, m + 1))
        A[:m, :m] = R @ R.T * dv
        A[:m, m] = A[m, :m] = 1.0
        rhs = np.zeros(m + 1)
        rhs[m] = 1.0
        try:
            alpha = np.linalg.solve(A, rhs)[:m]
            if not np.all(np.isfinite(alpha)):
                raise np.linalg.LinAlgError
        except np.linalg.LinAlgError:
            alpha = np.zeros(m)
            alpha[-1] = 1.0
        return sum(a * (h[0] + self.beta * h[2]) for a, h in zip(alpha, self.hist))


# ---------------------------------------------------------------- SCF
def setup_data(s):
    """The plain radial data of a setup object with the attributes Z,
    rloc, r_gauss, vbar / ghat / nguess splines, pt_j and dH_ii (splines
    with l, rmax, f_g)."""
    sp = lambda x: (x.l, x.rmax, np.array(x.f_g))
    return dict(Z=s.Z, rloc=s.rloc, r_gauss=s.r_gauss, vbar=sp(s.vbar),
                ghat=sp(s.ghat), nguess=sp(s.nguess),
                pt=[sp(p) for p in s.pt_j], dH=np.asarray(s.dH_ii, float))


def from_calculation(calc, **kwargs):
    """The oracle on a device calculation's geometry, setups, occupations
    and start (its current wave functions, widened to FP64)."""
    kpt = calc.wfs.kpt_u[0]
    return SCF([setup_data(s) for s in calc.setups], calc.spos_ac, calc.cell_cv,
               calc.pbc, calc.gd.N_c, kpt.psit_nG.double().cpu().numpy(),
               np.asarray(kpt.f_n), mixer_beta=calc.mixer.beta, **kwargs)


def h2gpts(h, cell_cv, idiv=4):
    """gpaw/utilities/__init__.py:108-120."""
    L_c = (np.linalg.inv(cell_cv)**2).sum(0)**-0.5
    return np.maximum(idiv, (L_c / h / idiv + 0.5).astype(int) * idiv)


class SCF:
    """cell_cv and positions in Bohr; psit_nG the starting wave functions
    (orthonormal), f_n the occupations; xc 'LDA' or 'PBE'."""

    def __init__(self, setups, spos_ac, cell_cv, pbc_c, N_c, psit_nG, f_n,
                 xc='LDA', blocksize=None, mixer_beta=0.25, kerker_q0=1.0,
                 niter=3, trial_step=0.1):
        self.g = Grid(N_c, cell_cv, pbc_c)
        self.fine = self.g.refine()
        self.setups = setups
        self.spos_ac = np.asarray(spos_ac, float)
        self.nvalence = sum(s['Z'] for s in setups)
        self.xc = xc
        g, fine = self.g, self.fine
        self.pt = LFC(g, [s['pt'] for s in setups], self.spos_ac)
        self.dH_MM = np.zeros((self.pt.Mmax, self.pt.Mmax))
        for a, s in enumerate(setups):
            ni = len(s['dH'])
            M = self.pt.M_a[a]
            self.dH_MM[M:M + ni, M:M + ni] = s['dH']
        vbar = LFC(fine, [[s['vbar']] for s in setups], self.spos_ac)
        self.vbar = vbar
        self.vbar_g = np.zeros(tuple(fine.n_c))
        vbar.add(self.vbar_g, np.ones((len(setups),)))
        self.ghat_raw = LFC(fine, [[s['ghat']] for s in setups], self.spos_ac)
        ghat = LFC(fine, [[s['ghat']] for s in setups], self.spos_ac,
                   integral=[float(s['Z']) for s in setups])
        self.rhoion_g = np.zeros(tuple(fine.n_c))
        ghat.add(self.rhoion_g, -np.ones((len(setups),)))
        guess = LFC(g, [[s['nguess']] for s in setups], self.spos_ac,
                    integral=[float(s['Z']) for s in setups])
        self.nt_G = np.zeros(tuple(g.n_c))
        guess.add(self.nt_G, np.ones((len(setups),)))
        self.kin = operator(g, fd.guc_laplace(g.h_cv, -0.5, 3))
        self.interpolate = transformer(g, fine, 3)
        self.restrict = transformer(fine, g, 3)
        self.pc = Preconditioner(g, fd.guc_laplace(g.h_cv, -0.5, 3))
        self.grads = [operator(fine, fd.ortho_gradient(fine.h_cv, v, 1.0, 2))
                      for v in range(3)]
        periodic = bool(np.all(pbc_c))
        self.mixer = PulayMixer(g, mixer_beta, 5, kerker_q0 if periodic else None)
        self.psit = np.array(psit_nG, float)
        self.f_n = np.asarray(f_n, float)
        self.weights = np.where(self.f_n > 0, 1.0, 0.0)
        self.P = self.pt.integrate(self.psit)
        self.eps = None
        self.blocksize = blocksize
        self.niter = niter
        self.trial_step = trial_step
        self.constant = self._constant_energy()

    # ---------------------------------------------------------- energy
    def _constant_energy(self):
        """Remove each Gaussian ion charge's self-energy Z^2/(2 sqrt(pi) s)
        from the Hartree term (the role of the setups' M = -Eh_compcharge,
        gpaw/pseudopotential.py:293) and replace the Gaussian-Gaussian
        interaction of widths s by that of widths r_loc (the widths of the
        reference's HGH compensation charges, gpaw/hgh.py:102):
        sum_{a<b} Z_a Z_b [erf(R/sqrt(2(rl_a^2+rl_b^2))) -
        erf(R/sqrt(2(s_a^2+s_b^2)))] / R over the periodic images."""
        from math import erf
        e = -sum(s['Z']**2 / (2 * sqrt(pi) * s['r_gauss']) for s in self.setups)
        pos = self.spos_ac @ self.g.cell_cv
        rng = [(-1, 0, 1) if p else (0,) for p in self.g.pbc_c]
        for a, sa in enumerate(self.setups):
            for b, sb in enumerate(self.setups):
                w1 = sqrt(2 * (sa['rloc']**2 + sb['rloc']**2))
                w2 = sqrt(2 * (sa['r_gauss']**2 + sb['r_gauss']**2))
                for i in rng[0]:
                    for j in rng[1]:
                        for k in rng[2]:
                            if a == b and i == j == k == 0:
                                continue
                            R = float(np.linalg.norm(
                                pos[b] + np.array([i, j, k]) @ self.g.cell_cv - pos[a]))
                            e += 0.5 * sa['Z'] * sb['Z'] * (erf(R / w1) - erf(R / w2)) / R
        return e

    def update_hamiltonian(self):
        fine = self.fine
        nt_g = self.interpolate(self.nt_G)
        nt_g *= self.nvalence / (nt_g.sum() * fine.dv)
        rhot_g = nt_g + self.rhoion_g
        vHt_g = poisson.solve(rhot_g, fine.N_c, fine.pbc_c, fine.cell_cv, 3, charge=0.0)
        e_g = np.zeros(tuple(fine.n_c))
        v_sg = np.zeros((1,) + tuple(fine.n_c))
        gp = ref.load()
        if self.xc == 'LDA':
            gp.XCFunctional(-1).calculate(e_g, nt_g[None].copy(), v_sg)
        else:
            n_sg = nt_g[None].copy()
            grad_vg = [gr(nt_g) for gr in self.grads]
            sigma = sum(x * x for x in grad_vg)[None].copy()
            dedsigma = np.zeros_like(sigma)
            gp.XCFunctional(0).calculate(e_g, n_sg, v_sg, sigma, dedsigma)
            for v in range(3):
                v_sg[0] -= 2.0 * self.grads[v](dedsigma[0] * grad_vg[v])
        self.vHt_g = vHt_g
        self.vt_g = self.vbar_g + vHt_g + v_sg[0]
        self.vt_G = self.restrict(self.vt_g)
        self.e_terms = np.array([0.5 * (rhot_g * vHt_g).sum() * fine.dv,
                                 e_g.sum() * fine.dv,
                                 (nt_g * self.vbar_g).sum() * fine.dv])
        self.nt_g = nt_g

    def total_energy(self):
        band = (self.f_n * self.eps).sum()
        return (band - (self.nt_G * self.vt_G).sum() * self.g.dv +
                self.e_terms.sum() + self.constant)

    # ---------------------------------------------------------- eigensolver
    def apply_H(self, psit):
        return self.kin(psit) + self.vt_G * psit

    def residuals(self, psit, P, eps, R):
        """R <- R - eps psit + sum_a p^a dH^a P^a (eigensolver.py:153-172)."""
        R -= eps[:, None, None, None] * psit
        self.pt.add(R, P @ self.dH_MM.T)

    def dot(self, a, b):
        return (a * b).sum(axis=(-3, -2, -1)) * self.g.dv

    def subspace_diagonalize(self):
        """H_nn = dv psi (H psi)^T + P dH P^T, eigh, rotate psi, H psi and
        P (eigensolver.py:174-236)."""
        Htpsit = self.apply_H(self.psit)
        nb = len(self.psit)
        H = self.psit.reshape(nb, -1) @ Htpsit.reshape(nb, -1).T * self.g.dv
        H += self.P @ self.dH_MM @ self.P.T
        H = 0.5 * (H + H.T)
        eps, V = np.linalg.eigh(H)
        U = V.T
        self.psit = (U @ self.psit.reshape(nb, -1)).reshape(self.psit.shape)
        self.Htpsit = (U @ Htpsit.reshape(nb, -1)).reshape(self.psit.shape)
        self.P = U @ self.P
        self.eps = eps
        return H

    def update_bands(self):
        """The RMM-DIIS pass after the subspace rotation
        (rmmdiis.py:63-272); returns the weighted residual norm."""
        psit = self.psit
        R = self.Htpsit
        self.residuals(psit, self.P, self.eps, R)
        nb = len(psit)
        B = nb if self.blocksize is None else self.blocksize
        error = 0.0
        for n1 in range(0, nb, B):
            n2 = min(n1 + B, nb)
            eps = self.eps[n1:n2]
            psitb = psit[n1:n2]
            Rb = R[n1:n2]
            error += (self.weights[n1:n2] * self.dot(Rb, Rb)).sum()
            psi_diis = [psitb.copy()]
            R_diis = [Rb.copy()]
            dpsit = self.pc(Rb)
            dR = self.apply_H(dpsit)
            self.residuals(dpsit, self.pt.integrate(dpsit), eps, dR)
            lam = -self.dot(dR, Rb) / self.dot(dR, dR)
            psitb += lam[:, None, None, None] * dpsit
            Rb += lam[:, None, None, None] * dR
            for nit in range(1, self.niter):
                psi_diis.append(psitb.copy())
                R_diis.append(Rb.copy())
                if nit > 1:
                    for ib in range(n2 - n1):
                        Rs = np.array([r[ib].ravel() for r in R_diis])
                        A = -np.ones((nit + 2, nit + 2))
                        A[:nit + 1, :nit + 1] = Rs @ Rs.T * self.g.dv
                        A[-1, -1] = 0.0
                        x = np.zeros(nit + 2)
                        x[-1] = -1.0
                        alpha = np.linalg.solve(A, x)[:-1]
                        psitb[ib] = alpha[nit] * psi_diis[nit][ib]
                        Rb[ib] = alpha[nit] * R_diis[nit][ib]
                        for i in range(nit):
                            psitb[ib] += alpha[i] * psi_diis[i][ib]
                            Rb[ib] += alpha[i] * R_diis[i][ib]
                if nit < self.niter - 1:
                    dpsit = self.pc(Rb)
                    psitb += lam[:, None, None, None] * dpsit
                    Rb[:] = self.apply_H(psitb)
                    self.residuals(psitb, self.pt.integrate(psitb), eps, Rb)
            dpsit = self.pc(Rb)
            step = self.trial_step if self.trial_step is not None else lam
            psitb += np.broadcast_to(step, lam.shape)[:, None, None, None] * dpsit
        return error

    def orthonormalize(self):
        """psi <- L^-1 psi with dv psi psi^T = L L^T (fdpw.py:394-424)."""
        nb = len(self.psit)
        A = self.psit.reshape(nb, -1)
        S = A @ A.T * self.g.dv
        L = np.linalg.cholesky(0.5 * (S + S.T))
        self.psit = np.linalg.solve(L, A).reshape(self.psit.shape)
        self.P = self.pt.integrate(self.psit)

    # ---------------------------------------------------------- driver
    def update_density(self):
        gp = ref.load()
        nt = np.zeros(tuple(self.g.n_c))
        for f, p in zip(self.f_n, self.psit):
            gp.add_to_density(float(f), np.ascontiguousarray(p), nt)
        ddens = np.abs(nt - self.nt_G).sum() * self.g.dv / self.nvalence
        self.nt_G = np.maximum(self.mixer.mix(self.nt_G, nt, self.g.dv), 0.0)
        return ddens

    def iteration(self):
        self.subspace_diagonalize()
        err = self.update_bands()
        self.orthonormalize()
        E = self.total_energy() * HARTREE
        ddens = self.update_density()
        self.update_hamiltonian()
        return E, err, ddens

    def run(self, maxiter=200, energy_tol=1e-5, density_tol=1e-4,
            eigenstates_tol=4e-8):
        """The device SCF's convergence test: energy change over the last
        three iterations per valence electron, density change per electron
        and eigenstate error (eV^2 per electron)."""
        self.update_hamiltonian()
        self.energies, self.errors = [], []
        self.converged = False
        for it in range(1, maxiter + 1):
            E, err, ddens = self.iteration()
            self.energies.append(E)
            self.errors.append(err * HARTREE**2 / self.nvalence)
            if it >= 3:
                dE = (max(self.energies[-3:]) - min(self.energies[-3:])) / self.nvalence
                if (dE < energy_tol and ddens < density_tol and
                        self.errors[-1] < eigenstates_tol):
                    self.converged = True
                    break
        self.iterations = it
        return self

    def eigenvalues(self):
        return self.eps * HARTREE

    # ---------------------------------------------------------- forces
    def forces(self):
        """Hellmann-Feynman forces (eV / Angstrom) of the present state:
        projectors 2 sum_n f_n sum_ij <psi|dp_i/dr> dH_ij P_nj (the
        reference's LFC.derivative on the wave functions), vbar
        int nt dvbar/dr, the grid-normalised Gaussian ion charges
        -Z [D(v_H) / I - A(v_H) D(1) / I^2] and the gradient of the
        geometry constant, by central differences of its closed form."""
        natoms = len(self.setups)
        F = np.zeros((natoms, 3))
        if self.pt.Mmax:
            D = self.pt.derivative(self.psit)                  # (nb, M, 3)
            C = self.P @ self.dH_MM.T
            F_Mv = 2 * np.einsum('n,nmv,nm->mv', self.f_n, D, C)
            for a, s in enumerate(self.setups):
                M = self.pt.M_a[a]
                F[a] += F_Mv[M:M + len(s['dH'])].sum(0)
        F += self.vbar.derivative(self.nt_g)
        one = np.ones_like(self.vHt_g)
        D_v = self.ghat_raw.derivative(self.vHt_g)
        D_1 = self.ghat_raw.derivative(one)
        A_v = self.ghat_raw.integrate(self.vHt_g)
        I = self.ghat_raw.integrate(one)
        Z = np.array([s['Z'] for s in self.setups], float)
        F -= Z[:, None] * (D_v / I[:, None] - A_v[:, None] * D_1 / I[:, None]**2)
        h = 1e-5
        for a in range(natoms):
            for v in range(3):
                e = []
                for sgn in (1, -1):
                    spos = self.spos_ac.copy()
                    spos[a] += sgn * h * np.linalg.inv(self.g.cell_cv)[v]
                    saved = self.spos_ac
                    self.spos_ac = spos
                    e.append(self._constant_energy())
                    self.spos_ac = saved
                F[a, v] -= (e[0] - e[1]) / (2 * h)
        return F * HARTREE / 0.52917721067
