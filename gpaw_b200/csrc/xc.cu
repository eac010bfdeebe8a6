// Exchange-correlation on the grid (replaces _gpaw.XCFunctional for LDA and
// the PBE family: c/xc/xc.c:73-227, c/xc/pbe.c, c/xc/rpbe.c).
//
// Written from the published forms:
//   * LDA exchange  e_x = -(3/4)(3/pi)^(1/3) n^(1/3) = C1 / r_s
//   * PW92 correlation (Perdew & Wang, PRB 45, 13244 (1992)): the G(r_s)
//     interpolation with the published (A, alpha1, beta1..beta4) for the
//     paramagnetic, ferromagnetic and spin-stiffness channels, and the
//     f(zeta) spin interpolation
//   * PBE (Perdew, Burke & Ernzerhof, PRL 77, 3865 (1996)): exchange
//     enhancement F_x(s) = 1 + kappa - kappa / (1 + mu s^2 / kappa), gradient
//     correction H(r_s, zeta, t); revPBE (kappa = 1.245) and RPBE
//     (F_x = 1 + kappa (1 - exp(-mu s^2 / kappa)))
// Derivatives are taken w.r.t. r_s at fixed |grad n|^2 (a2), as the reference
// does, and combined into
//   e_g = n (e_x + e_c),  v_g += e_x + e_c - r_s (de_x/dr_s + de_c/dr_s) / 3,
//   dedsigma = n (de_x/da2 + de_c/da2)
// with the reference's spin-scaling for two spins (c/xc/xc.c:149-225).
// Densities below NMIN = 1e-10 are clamped (c/xc/xc_gpaw.h).  FP64 only.
// One thread per grid point; HBM-bound for LDA, FP64-pipe-bound for PBE.
#include <algorithm>
#include <cmath>
#include "internal.cuh"

namespace gb {
namespace xc {

constexpr double PI = 3.14159265358979323846;
constexpr double NMIN = 1.0e-10;
// PBE beta and gamma = (1 - ln 2) / pi^2
constexpr double BETA = 0.066725;
constexpr double GAMMA = 0.031091;

struct Par {
  int gga;      // 0: LDA
  int rpbe;     // RPBE exchange form
  double kappa;
  double mu;    // beta pi^2 / 3
  double C0I;   // 3 / (4 pi)
  double C1;    // LDA exchange: e_x = C1 / r_s
  double C2;    // s^2 = a2 (C2 r_s / n)^2
  double C3;    // t^2 = C3 a2 r_s / (n^2 phi^2)
  double CC1;   // 1 / (2^(4/3) - 2)
  double CC2;   // 4 CC1 / 3
  double IF2;   // 1 / f''(0)
};

// PW92 G(r_s) and dG/dr_s:  G = -2 A (1 + a1 r_s) ln(1 + 1 / (2 A Q)),
// Q = b1 r_s^1/2 + b2 r_s + b3 r_s^3/2 + b4 r_s^2
__device__ __forceinline__ double pw92_G(double rtrs, double A, double a1, double b1, double b2,
                                         double b3, double b4, double* dGdrs) {
  const double rs = rtrs * rtrs;
  const double P = -2.0 * A * (1.0 + a1 * rs);
  const double Q = 2.0 * A * rtrs * (b1 + rtrs * (b2 + rtrs * (b3 + rtrs * b4)));
  const double L = log(1.0 + 1.0 / Q);
  const double G = P * L;
  // dQ/drs = A (b1 / rtrs + 2 b2 + 3 b3 rtrs + 4 b4 rs)
  const double dQ = A * (b1 / rtrs + 2.0 * b2 + rtrs * (3.0 * b3 + 4.0 * b4 * rtrs));
  *dGdrs = -2.0 * A * a1 * L - P * dQ / (Q * (Q + 1.0));
  return G;
}

__device__ __forceinline__ double exchange(const Par& p, double n, double rs, double a2,
                                           double* dedrs, double* deda2) {
  double e = p.C1 / rs;
  *dedrs = -e / rs;
  if (p.gga) {
    double c = p.C2 * rs / n;
    c *= c;
    const double s2 = a2 * c;
    double Fx, dFxds2;
    if (p.rpbe) {
      const double x = exp(-p.mu * s2 / p.kappa);
      Fx = 1.0 + p.kappa * (1.0 - x);
      dFxds2 = p.mu * x;
    } else {
      const double x = 1.0 + p.mu * s2 / p.kappa;
      Fx = 1.0 + p.kappa - p.kappa / x;
      dFxds2 = p.mu / (x * x);
    }
    // s^2 ~ r_s^8 at fixed a2
    *dedrs = *dedrs * Fx + e * dFxds2 * 8.0 * s2 / rs;
    *deda2 = e * dFxds2 * c;
    e *= Fx;
  }
  return e;
}

__device__ __forceinline__ double correlation(const Par& p, double n, double rs, double zeta, double a2,
                                              bool spinpol, double* dedrs, double* dedzeta,
                                              double* deda2) {
  const double rtrs = sqrt(rs);
  double de0;
  const double e0 = pw92_G(rtrs, GAMMA, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294, &de0);
  double e;
  double xp = 1.0, xm = 1.0;
  if (spinpol) {
    double de1, dalpha;
    const double e1 = pw92_G(rtrs, 0.015545, 0.20548, 14.1189, 6.1977, 3.3662, 0.62517, &de1);
    const double alpha = -pw92_G(rtrs, 0.016887, 0.11125, 10.357, 3.6231, 0.88026, 0.49671, &dalpha);
    dalpha = -dalpha;
    const double zp = 1.0 + zeta, zm = 1.0 - zeta;
    xp = cbrt(zp);
    xm = cbrt(zm);
    const double f = p.CC1 * (zp * xp + zm * xm - 2.0);
    const double f1 = p.CC2 * (xp - xm);
    const double z3 = zeta * zeta * zeta, z4 = z3 * zeta;
    const double x = 1.0 - z4;
    *dedrs = de0 * (1.0 - f * z4) + de1 * f * z4 + dalpha * f * x * p.IF2;
    *dedzeta = 4.0 * z3 * f * (e1 - e0 - alpha * p.IF2) + f1 * (z4 * e1 - z4 * e0 + x * alpha * p.IF2);
    e = e0 + alpha * p.IF2 * f * x + (e1 - e0) * f * z4;
  } else {
    *dedrs = de0;
    e = e0;
  }
  if (p.gga) {
    const double n2 = n * n;
    double phi = 1.0, phi2 = 1.0, phi3 = 1.0;
    if (spinpol) {
      phi = 0.5 * (xp * xp + xm * xm);
      phi2 = phi * phi;
      phi3 = phi * phi2;
    }
    const double t2 = p.C3 * a2 * rs / (n2 * phi2);
    const double y = -e / (GAMMA * phi3);
    const double x = exp(y);
    const double A = (x != 1.0) ? BETA / (GAMMA * (x - 1.0)) : BETA / (GAMMA * y);
    const double At2 = A * t2;
    const double nom = 1.0 + At2;
    const double denom = nom + At2 * At2;
    double H = GAMMA * log(1.0 + BETA * t2 * nom / (denom * GAMMA));
    double tmp = GAMMA * BETA / (denom * (BETA * t2 * nom + GAMMA * denom));
    const double tmp2 = A * A * x / BETA;
    double dAdrs = tmp2 * *dedrs;
    if (spinpol) {
      H *= phi3;
      tmp *= phi3;
      dAdrs /= phi3;
    }
    const double dHdt2 = (1.0 + 2.0 * At2) * tmp;
    const double dHdA = -At2 * t2 * t2 * (2.0 + At2) * tmp;
    // t^2 ~ r_s^7 at fixed a2
    *dedrs += dHdt2 * 7.0 * t2 / rs + dHdA * dAdrs;
    *deda2 = dHdt2 * p.C3 * rs / n2;
    if (spinpol) {
      const double dphidzeta = (1.0 / xp - 1.0 / xm) / 3.0;
      const double dAdzeta = tmp2 * (*dedzeta - 3.0 * e * dphidzeta / phi) / phi3;
      *dedzeta += (3.0 * H / phi - dHdt2 * 2.0 * t2 / phi) * dphidzeta + dHdA * dAdzeta;
      *deda2 /= phi2;
    }
    e += H;
  }
  return e;
}

__global__ void xc_unpolarized(const Par p, int64_t ng, double* __restrict__ e_g,
                               const double* __restrict__ n_g, double* __restrict__ v_g,
                               const double* __restrict__ sigma_g, double* __restrict__ dedsigma_g) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < ng;
       g += (int64_t)gridDim.x * blockDim.x) {
    double n = n_g[g];
    if (n < NMIN) n = NMIN;
    const double rs = cbrt(p.C0I / n);
    double dexdrs, dexda2 = 0.0, decdrs, decda2 = 0.0, dz;
    const double a2 = p.gga ? sigma_g[g] : 0.0;
    const double ex = exchange(p, n, rs, a2, &dexdrs, &dexda2);
    const double ec = correlation(p, n, rs, 0.0, a2, false, &decdrs, &dz, &decda2);
    if (p.gga) dedsigma_g[g] = n * (dexda2 + decda2);
    e_g[g] = n * (ex + ec);
    v_g[g] += ex + ec - rs * (dexdrs + decdrs) / 3.0;
  }
}

__global__ void xc_polarized(const Par p, int64_t ng, double* __restrict__ e_g,
                             const double* __restrict__ n_sg, double* __restrict__ v_sg,
                             const double* __restrict__ sigma_xg, double* __restrict__ dedsigma_xg) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < ng;
       g += (int64_t)gridDim.x * blockDim.x) {
    double na = 2.0 * n_sg[g];
    if (na < NMIN) na = NMIN;
    const double rsa = cbrt(p.C0I / na);
    double nb = 2.0 * n_sg[ng + g];
    if (nb < NMIN) nb = NMIN;
    const double rsb = cbrt(p.C0I / nb);
    const double n = 0.5 * (na + nb);
    const double rs = cbrt(p.C0I / n);
    const double zeta = 0.5 * (na - nb) / n;
    double dexadrs, dexada2 = 0.0, dexbdrs, dexbda2 = 0.0, decdrs, decdzeta, decda2 = 0.0;
    double exa, exb, ec;
    if (p.gga) {
      const double s0 = sigma_xg[g], s1 = sigma_xg[ng + g], s2 = sigma_xg[2 * ng + g];
      exa = exchange(p, na, rsa, 4.0 * s0, &dexadrs, &dexada2);
      exb = exchange(p, nb, rsb, 4.0 * s2, &dexbdrs, &dexbda2);
      const double a2 = s0 + 2.0 * s1 + s2;
      ec = correlation(p, n, rs, zeta, a2, true, &decdrs, &decdzeta, &decda2);
      dedsigma_xg[g] = 2.0 * na * dexada2 + n * decda2;
      dedsigma_xg[ng + g] = 2.0 * n * decda2;
      dedsigma_xg[2 * ng + g] = 2.0 * nb * dexbda2 + n * decda2;
    } else {
      exa = exchange(p, na, rsa, 0.0, &dexadrs, &dexada2);
      exb = exchange(p, nb, rsb, 0.0, &dexbdrs, &dexbda2);
      ec = correlation(p, n, rs, zeta, 0.0, true, &decdrs, &decdzeta, &decda2);
    }
    e_g[g] = 0.5 * (na * exa + nb * exb) + n * ec;
    v_sg[g] += exa + ec - (rsa * dexadrs + rs * decdrs) / 3.0 - (zeta - 1.0) * decdzeta;
    v_sg[ng + g] += exb + ec - (rsb * dexbdrs + rs * decdrs) / 3.0 - (zeta + 1.0) * decdzeta;
  }
}

static Par make_par(int code) {
  Par p{};
  p.gga = code != -1;
  p.rpbe = code == 2;
  p.kappa = code == 1 ? 1.245 : 0.804;
  p.mu = BETA * PI * PI / 3.0;
  p.C0I = 3.0 / (4.0 * PI);
  p.C1 = -9.0 / (8.0 * PI) * cbrt(2.0 * PI / 3.0);
  p.C2 = 1.0 / cbrt(18.0 * PI);
  p.C3 = PI * cbrt(4.0 / (9.0 * PI)) / 16.0;
  p.CC1 = 1.0 / (pow(2.0, 4.0 / 3.0) - 2.0);
  p.CC2 = 4.0 * p.CC1 / 3.0;
  // f''(0) = CC1 * (4/9) * 2 = 8 CC1 / 9
  p.IF2 = 9.0 / (8.0 * p.CC1);
  return p;
}

}  // namespace xc
}  // namespace gb

using namespace gb;

extern "C" int gb_xc_calculate(int code, int nspins, int64_t ng, double* e_g, const double* n_sg,
                               double* v_sg, const double* sigma_xg, double* dedsigma_xg,
                               void* stream) {
  GB_REQUIRE(code == -1 || code == 0 || code == 1 || code == 2,
             "gb_xc_calculate: code must be -1 (LDA), 0 (PBE), 1 (revPBE) or 2 (RPBE)");
  GB_REQUIRE(nspins == 1 || nspins == 2, "gb_xc_calculate: nspins must be 1 or 2");
  GB_REQUIRE(ng >= 0, "gb_xc_calculate: negative size");
  if (ng == 0) return GB_OK;
  GB_REQUIRE(e_g && n_sg && v_sg, "gb_xc_calculate: null array");
  GB_REQUIRE(code == -1 || (sigma_xg && dedsigma_xg), "gb_xc_calculate: GGA needs sigma and dedsigma");
  const xc::Par p = xc::make_par(code);
  const int threads = 256;
  const int64_t blocks = std::min<int64_t>((ng + threads - 1) / threads, (int64_t)sm_count() * 16);
  if (nspins == 1)
    xc::xc_unpolarized<<<(unsigned)blocks, threads, 0, (cudaStream_t)stream>>>(p, ng, e_g, n_sg, v_sg, sigma_xg,
                                                                              dedsigma_xg);
  else
    xc::xc_polarized<<<(unsigned)blocks, threads, 0, (cudaStream_t)stream>>>(p, ng, e_g, n_sg, v_sg, sigma_xg,
                                                                            dedsigma_xg);
  return check_launch("xc kernel");
}
