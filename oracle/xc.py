"""ORACLE (test infrastructure): LDA / PBE-family exchange-correlation point
kernels in numpy, restating c/xc/xc.c:119-225 (spin-paired and polarised
drivers), c/xc/pbe.c:7-164 (PBE exchange, PW92 + PBE correlation) and
c/xc/rpbe.c:7-27.  Vectorised over grid points, float64.
Pinned against the reference C extension (tests/test_oracle_xc.py) and the
golden vectors in tests/golden/xc.npz.
"""
from __future__ import annotations

import numpy as np

# c/xc/xc_gpaw.h (values derived there from pi)
BETA = 0.066725
GAMMA = 0.031091
MU = BETA * np.pi**2 / 3
C2 = 1 / (18 * np.pi)**(1 / 3)
C0I = 3 / (4 * np.pi)
C1 = -9 / (8 * np.pi) * (2 * np.pi / 3)**(1 / 3)
CC1 = 1 / (2**(4 / 3) - 2)
CC2 = 4 * CC1 / 3
IF2 = 3 / (2 * CC2)
C3 = np.pi * (4 / (9 * np.pi))**(1 / 3) / 16
THIRD = 1 / 3
NMIN = 1e-10

CODES = {'LDA': -1, 'PBE': 0, 'revPBE': 1, 'RPBE': 2}


def _exchange(code, n, rs, a2):
    """pbe_exchange / rpbe_exchange: (e, dedrs, deda2)."""
    e = C1 / rs
    dedrs = -e / rs
    deda2 = np.zeros_like(n)
    if code != -1:
        c = (C2 * rs / n)**2
        s2 = a2 * c
        if code == 2:
            x = np.exp(-MU * s2 / 0.804)
            Fx = 1.0 + 0.804 * (1 - x)
            dFxds2 = MU * x
        else:
            kappa = 1.245 if code == 1 else 0.804
            x = 1.0 + MU * s2 / kappa
            Fx = 1.0 + kappa - kappa / x
            dFxds2 = MU / (x * x)
        ds2drs = 8.0 * c * a2 / rs
        dedrs = dedrs * Fx + e * dFxds2 * ds2drs
        deda2 = e * dFxds2 * c
        e = e * Fx
    return e, dedrs, deda2


def _G(rtrs, A, alpha1, beta1, beta2, beta3, beta4):
    """PW92 interpolation G(r_s) and dG/dr_s (c/xc/pbe.c:30-44)."""
    Q0 = -2.0 * A * (1.0 + alpha1 * rtrs * rtrs)
    Q1 = 2.0 * A * rtrs * (beta1 + rtrs * (beta2 + rtrs * (beta3 + rtrs * beta4)))
    G1 = Q0 * np.log(1.0 + 1.0 / Q1)
    dQ1drs = A * (beta1 / rtrs + 2.0 * beta2 + rtrs * (3.0 * beta3 + 4.0 * beta4 * rtrs))
    dGdrs = -2.0 * A * alpha1 * G1 / Q0 - Q0 * dQ1drs / (Q1 * (Q1 + 1.0))
    return G1, dGdrs


def _correlation(n, rs, zeta, a2, gga, spinpol):
    """pbe_correlation (c/xc/pbe.c:65-164): (e, dedrs, dedzeta, deda2)."""
    rtrs = np.sqrt(rs)
    e0, de0drs = _G(rtrs, GAMMA, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294)
    dedzeta = np.zeros_like(n)
    deda2 = np.zeros_like(n)
    if spinpol:
        e1, de1drs = _G(rtrs, 0.015545, 0.20548, 14.1189, 6.1977, 3.3662, 0.62517)
        alpha, dalphadrs = _G(rtrs, 0.016887, 0.11125, 10.357, 3.6231, 0.88026, 0.49671)
        alpha = -alpha
        dalphadrs = -dalphadrs
        zp = 1.0 + zeta
        zm = 1.0 - zeta
        xp = zp**THIRD
        xm = zm**THIRD
        f = CC1 * (zp * xp + zm * xm - 2.0)
        f1 = CC2 * (xp - xm)
        zeta2 = zeta * zeta
        zeta3 = zeta2 * zeta
        zeta4 = zeta2 * zeta2
        x = 1.0 - zeta4
        dedrs = de0drs * (1.0 - f * zeta4) + de1drs * f * zeta4 + dalphadrs * f * x * IF2
        dedzeta = (4.0 * zeta3 * f * (e1 - e0 - alpha * IF2) +
                   f1 * (zeta4 * e1 - zeta4 * e0 + x * alpha * IF2))
        e = e0 + alpha * IF2 * f * x + (e1 - e0) * f * zeta4
    else:
        dedrs = de0drs
        e = e0
    if gga:
        n2 = n * n
        if spinpol:
            phi = 0.5 * (xp * xp + xm * xm)
            phi2 = phi * phi
            phi3 = phi * phi2
            t2 = C3 * a2 * rs / (n2 * phi2)
            y = -e / (GAMMA * phi3)
        else:
            t2 = C3 * a2 * rs / n2
            y = -e / GAMMA
        x = np.exp(y)
        with np.errstate(divide='ignore', invalid='ignore'):
            A = np.where(x != 1.0, BETA / (GAMMA * (x - 1.0)), BETA / (GAMMA * y))
        At2 = A * t2
        nom = 1.0 + At2
        denom = nom + At2 * At2
        H = GAMMA * np.log(1.0 + BETA * t2 * nom / (denom * GAMMA))
        tmp = GAMMA * BETA / (denom * (BETA * t2 * nom + GAMMA * denom))
        tmp2 = A * A * x / BETA
        dAdrs = tmp2 * dedrs
        if spinpol:
            H = H * phi3
            tmp = tmp * phi3
            dAdrs = dAdrs / phi3
        dHdt2 = (1.0 + 2.0 * At2) * tmp
        dHdA = -At2 * t2 * t2 * (2.0 + At2) * tmp
        dedrs = dedrs + dHdt2 * 7 * t2 / rs + dHdA * dAdrs
        deda2 = dHdt2 * C3 * rs / n2
        if spinpol:
            dphidzeta = (1.0 / xp - 1.0 / xm) / 3.0
            dAdzeta = tmp2 * (dedzeta - 3.0 * e * dphidzeta / phi) / phi3
            dedzeta = dedzeta + ((3.0 * H / phi - dHdt2 * 2.0 * t2 / phi) * dphidzeta +
                                 dHdA * dAdzeta)
            deda2 = deda2 / phi2
        e = e + H
    return e, dedrs, dedzeta, deda2


def calculate(code, e_g, n_sg, v_sg, sigma_xg=None, dedsigma_xg=None):
    """XCFunctional.calculate semantics (c/xc/xc.c:73-227): overwrite e_g and
    dedsigma_xg, ADD to v_sg."""
    gga = code != -1
    nspins = n_sg.shape[0]
    if nspins == 1:
        n = np.maximum(n_sg[0], NMIN)
        rs = (C0I / n)**THIRD
        a2 = sigma_xg[0] if gga else np.zeros_like(n)
        ex, dexdrs, dexda2 = _exchange(code, n, rs, a2)
        ec, decdrs, _, decda2 = _correlation(n, rs, np.zeros_like(n), a2, gga, False)
        if gga:
            dedsigma_xg[0] = n * (dexda2 + decda2)
        e_g[:] = n * (ex + ec)
        v_sg[0] += ex + ec - rs * (dexdrs + decdrs) / 3.0
        return
    na = np.maximum(2.0 * n_sg[0], NMIN)
    rsa = (C0I / na)**THIRD
    nb = np.maximum(2.0 * n_sg[1], NMIN)
    rsb = (C0I / nb)**THIRD
    n = 0.5 * (na + nb)
    rs = (C0I / n)**THIRD
    zeta = 0.5 * (na - nb) / n
    if gga:
        exa, dexadrs, dexada2 = _exchange(code, na, rsa, 4.0 * sigma_xg[0])
        exb, dexbdrs, dexbda2 = _exchange(code, nb, rsb, 4.0 * sigma_xg[2])
        a2 = sigma_xg[0] + 2 * sigma_xg[1] + sigma_xg[2]
        ec, decdrs, decdzeta, decda2 = _correlation(n, rs, zeta, a2, True, True)
        dedsigma_xg[0] = 2 * na * dexada2 + n * decda2
        dedsigma_xg[1] = 2 * n * decda2
        dedsigma_xg[2] = 2 * nb * dexbda2 + n * decda2
    else:
        z = np.zeros_like(n)
        exa, dexadrs, _ = _exchange(code, na, rsa, z)
        exb, dexbdrs, _ = _exchange(code, nb, rsb, z)
        ec, decdrs, decdzeta, _ = _correlation(n, rs, zeta, z, False, True)
    e_g[:] = 0.5 * (na * exa + nb * exb) + n * ec
    v_sg[0] += (exa + ec - (rsa * dexadrs + rs * decdrs) / 3.0 - (zeta - 1.0) * decdzeta)
    v_sg[1] += (exb + ec - (rsb * dexbdrs + rs * decdrs) / 3.0 - (zeta + 1.0) * decdzeta)


def log_uniform_inputs(seed, nspins, ng=10000):
    """Densities / sigmas spread over 5 decades, as in
    gpaw/test/gpu/test_xc_gpu.py:10-13."""
    rng = np.random.default_rng(seed)
    n_sg = np.exp(np.log(10) * 5 * (rng.random((nspins, ng)) - 0.5))
    sigma_xg = np.exp(np.log(10) * 5 * (rng.random((2 * nspins - 1, ng)) - 0.5))
    return n_sg, sigma_xg


def gga_calculate(code, n_sg, h_cv, pbc_c, v_sg, e_g):
    """GGA grid driver (gpaw/xc/gga.py:106-163, 195-200) for orthorhombic
    cells with the nn=2 Gradient stencils; returns nothing, fills e_g and
    adds to v_sg."""
    from oracle.fd import ortho_gradient, fd_apply
    nspins = n_sg.shape[0]
    grads = [ortho_gradient(h_cv, v, 1.0, 2) for v in range(3)]
    gradn_svg = np.empty((nspins, 3) + n_sg.shape[1:])
    sigma_xg = np.zeros((2 * nspins - 1,) + n_sg.shape[1:])
    for v in range(3):
        for s in range(nspins):
            gradn_svg[s, v] = fd_apply(*grads[v], n_sg[s], pbc_c)
            sigma_xg[2 * s] += gradn_svg[s, v]**2
        if nspins == 2:
            sigma_xg[1] += gradn_svg[0, v] * gradn_svg[1, v]
    dedsigma_xg = np.empty_like(sigma_xg)
    calculate(code, e_g, n_sg, v_sg, sigma_xg, dedsigma_xg)
    for v in range(3):
        for s in range(nspins):
            vv = fd_apply(*grads[v], dedsigma_xg[2 * s] * gradn_svg[s, v], pbc_c)
            v_sg[s] -= 2.0 * vv
            if nspins == 2:
                vv = fd_apply(*grads[v], dedsigma_xg[1] * gradn_svg[s, v], pbc_c)
                v_sg[1 - s] -= vv
