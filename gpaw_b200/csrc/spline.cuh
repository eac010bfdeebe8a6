// Radial splines and real solid harmonics on the device (shared by
// spline.cu -- spline_to_grid -- and the LFC derivative in lfc.cu).
//
// A spline is the per-bin cubic s0 + u (s1 + u (s2 + u s3)), u = r - b dr,
// of the natural-spline construction of c/bmgs/spline.c:11-47 (built on the
// host in spline.cu); values at r >= rmax are 0.  r^l Y_lm are the real
// solid harmonics in the m order of c/bmgs/spherical_harmonics.h (l = 1:
// y, z, x; l = 2: xy, yz, 3z^2 - r^2, xz, x^2 - y^2), with the standard
// normalisations c00 = 1/sqrt(4 pi), c1 = sqrt(3/(4 pi)),
// c2a = sqrt(15/(4 pi)), c20 = sqrt(5/(16 pi)), c22 = sqrt(15/(16 pi)).
//
// Products and sums are written with round-to-nearest intrinsics so that
// nothing is contracted into an FMA: points on a sphere's edge are then
// classified exactly as the reference's (non-FMA) host code classifies them,
// and the tabulated values agree with it to the last bit.
#pragma once
#include <cuda_runtime.h>

// the radial spline object of the C ABI
struct gb_spline {
  int l = 0;
  int nbins = 0;
  double rmax = 0.0;
  double dr = 0.0;
  double* coef = nullptr;   // device [nbins + 1][4]
};

namespace gb {

struct SplineDev {
  const double* coef;   // [nbins + 1][4]
  int nbins;
  int l;
  double dr;
};

constexpr double YC00 = 0.28209479177387814;
constexpr double YC1 = 0.4886025119029199;
constexpr double YC2A = 1.0925484305920792;
constexpr double YC20 = 0.31539156525252005;
constexpr double YC22 = 0.5462742152960396;

__device__ __forceinline__ double mul_(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_(double a, double b) { return __dsub_rn(a, b); }

// f(r) and df/dr
__device__ __forceinline__ void spline_eval(const SplineDev& s, double r, double& f, double& df) {
  const int b = (int)(r / s.dr);
  if (b >= s.nbins) {
    f = 0.0;
    df = 0.0;
    return;
  }
  const double u = sub_(r, mul_((double)b, s.dr));
  const double* c = s.coef + 4 * b;
  f = add_(c[0], mul_(u, add_(c[1], mul_(u, add_(c[2], mul_(u, c[3]))))));
  df = add_(c[1], mul_(u, add_(mul_(2.0, c[2]), mul_(mul_(u, 3.0), c[3]))));
}

__device__ __forceinline__ double spline_value(const SplineDev& s, double r) {
  const int b = (int)(r / s.dr);
  if (b >= s.nbins) return 0.0;
  const double u = sub_(r, mul_((double)b, s.dr));
  const double* c = s.coef + 4 * b;
  return add_(c[0], mul_(u, add_(c[1], mul_(u, add_(c[2], mul_(u, c[3]))))));
}

// p[m] = f r^l Y_lm(x, y, z), l <= 2 (r2 = x^2 + y^2 + z^2)
__device__ __forceinline__ void solid_harmonics(int l, double f, double x, double y, double z, double r2,
                                                double* p) {
  if (l == 0) {
    p[0] = mul_(f, YC00);
  } else if (l == 1) {
    const double g = mul_(f, YC1);
    p[0] = mul_(g, y);
    p[1] = mul_(g, z);
    p[2] = mul_(g, x);
  } else {
    const double g = mul_(f, YC2A);
    p[0] = mul_(mul_(g, x), y);
    p[1] = mul_(mul_(g, y), z);
    p[2] = mul_(mul_(f, YC20), add_(-r2, mul_(mul_(3.0, z), z)));
    p[3] = mul_(mul_(g, x), z);
    p[4] = mul_(mul_(f, YC22), add_(-mul_(y, y), mul_(x, x)));
  }
}

// d/dx, d/dy, d/dz of f r^l Y_lm with f constant: p[3 m + v]
__device__ __forceinline__ void solid_harmonics_gradient(int l, double f, double x, double y, double z,
                                                         double* p) {
  if (l == 0) {
    p[0] = p[1] = p[2] = 0.0;
  } else if (l == 1) {
    const double g = mul_(f, YC1);
    p[0] = 0.0; p[1] = g;   p[2] = 0.0;   // y
    p[3] = 0.0; p[4] = 0.0; p[5] = g;     // z
    p[6] = g;   p[7] = 0.0; p[8] = 0.0;   // x
  } else {
    const double g = mul_(f, YC2A);
    const double h = mul_(f, mul_(2.0, YC20));
    const double k = mul_(f, mul_(2.0, YC22));
    p[0] = mul_(g, y);  p[1] = mul_(g, x);  p[2] = 0.0;                     // xy
    p[3] = 0.0;         p[4] = mul_(g, z);  p[5] = mul_(g, y);              // yz
    p[6] = -mul_(h, x); p[7] = -mul_(h, y); p[8] = mul_(mul_(h, 2.0), z);   // 3z^2 - r^2
    p[9] = mul_(g, z);  p[10] = 0.0;        p[11] = mul_(g, x);             // xz
    p[12] = mul_(k, x); p[13] = -mul_(k, y); p[14] = 0.0;                   // x^2 - y^2
  }
}

}  // namespace gb
