// Restriction / interpolation (replaces _gpaw.Transformer: c/transformers.c,
// c/bmgs/restrict.c, c/bmgs/interpolate.c).
//
// The reference pads each band (c/bc.c), then runs three separable 1-D passes
// with a transpose after each (restrict.c:136-155, interpolate.c:227-257),
// i.e. four trips through memory per band.  Here one persistent kernel does
// all three passes with one read of the input and one write of the output:
// a CTA owns a 2-D tile of the (axis1, axis2) output plane and marches along
// axis 0; each input plane (tile + halo, boundary conditions resolved while
// staging through cp.async) is reduced along axis 2 then axis 1 in shared
// memory, and the axis-0 pass runs on a per-thread register queue of the 2-D
// results.  The pass order (axis 2, 1, 0) and the 0.5 factor per pass follow
// the reference, so real FP64 results agree with it to rounding.
//
// Index conventions (single domain, gpaw/transformers.py:31-47):
//   restriction:   coarse local i  <-> fine local centre 2 i + off,
//                  off = 2 beg_out - beg_in (0 periodic, 1 zero boundary)
//   interpolation: fine local f has global index F = f + skip0; even F copies
//                  coarse global F/2, odd F = 2C+1 mixes coarse C-j, C+1+j;
//                  coarse local = global - cbeg (cbeg = beg_in).

#include <algorithm>
#include <cstring>
#include "internal.cuh"

namespace gb {

struct TrArgs {
  const void* in;
  void* out;
  const void* y;      // optional epilogue operand (interpolation)
  int64_t nbatch;
  int ni[3], no[3];   // input / output local sizes
  int pbc[3];
  int off[3];         // restriction centre offsets
  int skip0[3];       // interpolation parity offsets
  int cbeg[3];        // interpolation coarse begin
  int tiles1, tiles2;
  int nsteps;         // marching steps along axis 0 per column
  double alpha, gamma;
  PhaseSets phs;      // Bloch phases per k-point group of bands
  double w[4];        // midpoint weights for pairs at distance 1/2, 3/2, ...
};

__device__ __forceinline__ int tr_mod(int i, int n) {
  int r = i % n;
  return r < 0 ? r + n : r;
}

__device__ __forceinline__ int floor_div(int a, int b) {
  return (a >= 0) ? a / b : -((-a + b - 1) / b);
}

// Stage one input plane (rows [ry0, ry0+NR), cols [cx0, cx0+NC)) of `S` into
// smem (row pitch PITCH), resolving zero / periodic boundaries.  cx0 must be a
// multiple of VEC so 16-byte chunks line up.
template <typename T, int NR, int NC, int PITCH, int NT>
__device__ __forceinline__ void stage_plane(T* P, const T* S, int ry0, int cx0, int n1, int n2,
                                            int pbc1, int pbc2, int tid) {
  constexpr int VEC = 16 / sizeof(T);
  constexpr int KC = NC / VEC;
  static_assert(NC % VEC == 0, "");
  for (int e = tid; e < NR * KC; e += NT) {
    const int r = e / KC, k = e % KC;
    T* sd = P + r * PITCH + k * VEC;
    int y = ry0 + r;
    if (y < 0 || y >= n1) {
      if (!pbc1) {
#pragma unroll
        for (int v = 0; v < VEC; ++v) sd[v] = zero<T>();
        continue;
      }
      y = tr_mod(y, n1);
    }
    const T* row = S + (int64_t)y * n2;
    const int zs = cx0 + k * VEC;
    if (zs >= 0 && zs + VEC <= n2 && ((reinterpret_cast<uintptr_t>(row + zs) & 15) == 0)) {
      cp_async16(sd, row + zs);
    } else {
#pragma unroll
      for (int v = 0; v < VEC; ++v) {
        int z = zs + v;
        if (z < 0 || z >= n2) {
          if (!pbc2) { sd[v] = zero<T>(); continue; }
          z = tr_mod(z, n2);
        }
        cp_async_elem(sd + v, row + z);
      }
    }
  }
}

// multiply wrapped cells of a staged plane by the Bloch phase
template <typename T, int NR, int NC, int PITCH, int NT>
__device__ __forceinline__ void phase_fixup(T* P, int ry0, int cx0, int n1, int n2,
                                            const TrArgs& a, const double (&PH)[3][2][2], int tid) {
  for (int e = tid; e < NR * NC; e += NT) {
    const int r = e / NC, c = e % NC;
    const int y = ry0 + r, z = cx0 + c;
    double pr = 1.0, pi = 0.0;
    bool w = false;
    if (a.pbc[1] && (y < 0 || y >= n1)) { const int s = y < 0; pr = PH[1][s][0]; pi = PH[1][s][1]; w = true; }
    if (a.pbc[2] && (z < 0 || z >= n2)) {
      const int s = z < 0;
      const double qr = PH[2][s][0], qi = PH[2][s][1];
      const double tr = pr * qr - pi * qi, ti = pr * qi + pi * qr;
      pr = tr; pi = ti; w = true;
    }
    if (w) P[r * PITCH + c] = phase_mul(P[r * PITCH + c], pr, pi);
  }
}

// ---------------------------------------------------------------- restriction
template <typename T_, int K_, int CY_, int CZ_, int D_>
struct RCfg {
  using T = T_;
  static constexpr int K = K_, CY = CY_, CZ = CZ_, D = D_;
  static constexpr int NT = CY * CZ;
  static constexpr int VEC = 16 / (int)sizeof(T);
  static constexpr int FR = 2 * CY + 2 * K - 3;
  static constexpr int FC = 2 * CZ + 2 * K - 3;
  static constexpr int FCW = ((FC + VEC - 1 + VEC - 1) / VEC) * VEC;   // room for the alignment shift
  static constexpr int PITCH = FCW;
  static constexpr int PLANE = FR * PITCH;
  static constexpr int NS = D + 1;
  static constexpr int TB = FR * CZ;                                  // pass-A buffer
  static constexpr size_t SMEM = ((size_t)NS * PLANE + TB) * sizeof(T);
  static constexpr int NQ = 2 * K - 1;
};

template <class C>
__global__ void __launch_bounds__(C::NT) restrict_kernel(const TrArgs a) {
  using T = typename C::T;
  using R = typename Elem<T>::R;
  constexpr int K = C::K, CY = C::CY, CZ = C::CZ, D = C::D, NT = C::NT, VEC = C::VEC;
  constexpr int FR = C::FR, PITCH = C::PITCH, PLANE = C::PLANE, NS = C::NS, NQ = C::NQ;
  constexpr bool CPLX = Elem<T>::cplx;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ring = reinterpret_cast<T*>(smem_raw);
  T* tbuf = ring + NS * PLANE;

  const int tid = threadIdx.x, ty = tid / CZ, tz = tid % CZ;
  const int nf0 = a.ni[0], nf1 = a.ni[1], nf2 = a.ni[2];
  const int nc0 = a.no[0], nc1 = a.no[1], nc2 = a.no[2];
  const int64_t nf12 = (int64_t)nf1 * nf2, nc12 = (int64_t)nc1 * nc2;
  const int64_t ntiles = (int64_t)a.tiles1 * a.tiles2;
  const int64_t total = a.nbatch * ntiles * nc0;
  int64_t s = total * blockIdx.x / gridDim.x;
  const int64_t s_end = total * (blockIdx.x + 1) / gridDim.x;
  R w[K / 2];
#pragma unroll
  for (int m = 0; m < K / 2; ++m) w[m] = (R)a.w[m];
  const R half = (R)0.5, alpha = (R)a.alpha;

  while (s < s_end) {
    const int64_t col = s / nc0;
    const int Is = (int)(s % nc0);
    const int Ie = (int)((s_end - s) < (int64_t)(nc0 - Is) ? Is + (s_end - s) : nc0);
    s += Ie - Is;
    const int64_t band = col / ntiles;
    const int t = (int)(col % ntiles);
    const int Y0 = (t / a.tiles2) * CY, Z0 = (t % a.tiles2) * CZ;
    const T* src = reinterpret_cast<const T*>(a.in) + band * nf12 * nf0;
    T* dst = reinterpret_cast<T*>(a.out) + band * nc12 * nc0;
    const auto& PH = a.phs.ph[phase_set_of(a.phs, band)];
    const int ry0 = 2 * Y0 + a.off[1] - (K - 1);
    const int s0 = 2 * Z0 + a.off[2] - (K - 1);
    const int cx0 = floor_div(s0, VEC) * VEC;
    const int sh = s0 - cx0;
    const bool edge = ry0 < 0 || ry0 + FR > nf1 || cx0 < 0 || cx0 + PITCH > nf2;
    const int j0 = 2 * Is + a.off[0] - (K - 1);
    const int j1 = 2 * (Ie - 1) + a.off[0] + K;   // exclusive

    auto src_plane = [&](int j, double& pr, double& pi) -> int {
      pr = 1.0; pi = 0.0;
      if (j >= 0 && j < nf0) return j;
      if (!a.pbc[0]) return -1;
      const int sd = j < 0;
      pr = PH[0][sd][0]; pi = PH[0][sd][1];
      return tr_mod(j, nf0);
    };
    auto issue = [&](int j) {
      double pr, pi;
      const int sp = src_plane(j, pr, pi);
      if (sp < 0) return;
      stage_plane<T, FR, PITCH, PITCH, NT>(ring + ((j - j0) % NS) * PLANE, src + (int64_t)sp * nf12,
                                           ry0, cx0, nf1, nf2, a.pbc[1], a.pbc[2], tid);
    };

    T q[NQ];
#pragma unroll
    for (int m = 0; m < NQ; ++m) q[m] = zero<T>();
#pragma unroll
    for (int d = 0; d < D; ++d) {
      if (j0 + d < j1) issue(j0 + d);
      cp_async_commit();
    }
    for (int j = j0; j < j1; ++j) {
      cp_async_wait<D - 1>();
      __syncthreads();
      double pr, pi;
      const int sp = src_plane(j, pr, pi);
      T* P = ring + ((j - j0) % NS) * PLANE;
      T u = zero<T>();
      if (sp >= 0) {
        if (CPLX && a.phs.any && edge) {
          phase_fixup<T, FR, PITCH, PITCH, NT>(P, ry0, cx0, nf1, nf2, a, PH, tid);
          __syncthreads();
        }
        if constexpr (K == 2) {
          // k = 2: the 3 x 3 in-plane stencil straight from the staged plane
          // (the same operations, in the same order, as the two separable
          // passes below; no intermediate buffer, no barrier)
          const T* f = P + (2 * ty + 1) * PITCH + sh + 2 * tz + 1;
          T g[3];
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            const T* fr = f + (d - 1) * PITCH;
            g[d] = scale(half, fmadd(fr[0], w[0], add(fr[1], fr[-1])));
          }
          u = scale(half, fmadd(g[1], w[0], add(g[2], g[0])));
          if (CPLX) u = phase_mul(u, pr, pi);
        } else {
          // pass A: along axis 2 for every staged row
          for (int e = tid; e < FR * CZ; e += NT) {
            const int r = e / CZ, jz = e % CZ;
            const T* f = P + r * PITCH + sh + 2 * jz + (K - 1);
            T x = f[0];
#pragma unroll
            for (int m = 0; m < K / 2; ++m) x = fmadd(x, w[m], add(f[2 * m + 1], f[-(2 * m + 1)]));
            tbuf[r * CZ + jz] = scale(half, x);
          }
          __syncthreads();
          // pass B: along axis 1 for the own coarse point
          const T* tcol = tbuf + (2 * ty + (K - 1)) * CZ + tz;
          T x = tcol[0];
#pragma unroll
          for (int m = 0; m < K / 2; ++m)
            x = fmadd(x, w[m], add(tcol[(2 * m + 1) * CZ], tcol[-(2 * m + 1) * CZ]));
          u = scale(half, x);
          if (CPLX) u = phase_mul(u, pr, pi);
        }
      }
#pragma unroll
      for (int m = 0; m < NQ - 1; ++m) q[m] = q[m + 1];
      q[NQ - 1] = u;
      // axis 0: coarse plane whose last fine contribution just arrived
      const int tI = j - a.off[0] - (K - 1);
      if (tI >= 2 * Is && (tI & 1) == 0) {
        const int I = tI >> 1;
        T x = q[K - 1];
#pragma unroll
        for (int m = 0; m < K / 2; ++m) x = fmadd(x, w[m], add(q[K - 1 + 2 * m + 1], q[K - 1 - (2 * m + 1)]));
        x = scale(half, x);
        const int yi = Y0 + ty, zi = Z0 + tz;
        if (yi < nc1 && zi < nc2) dst[(int64_t)I * nc12 + (int64_t)yi * nc2 + zi] = scale(alpha, x);
      }
      // the separable passes reuse tbuf next step; the k = 2 path needs no
      // barrier here: the slot refilled below was last read in step j - 1,
      // which every thread finished before the barrier at the top of step j
      if constexpr (K != 2) __syncthreads();
      if (j + D < j1) issue(j + D);
      cp_async_commit();
    }
    cp_async_wait<0>();
    __syncthreads();
  }
}

// ---------------------------------------------------------------- interpolation
template <typename T_, int K_, int FY_, int FZ_, int RY_, int RZ_, int D_>
struct ICfg {
  using T = T_;
  static constexpr int K = K_, FY = FY_, FZ = FZ_, RY = RY_, RZ = RZ_, D = D_;
  static constexpr int TY = FY / RY, TZ = FZ / RZ, NT = TY * TZ;
  static constexpr int VEC = 16 / (int)sizeof(T);
  static constexpr int CR = FY / 2 + K + 1;                     // coarse rows staged
  static constexpr int CC = FZ / 2 + K + 1;                     // coarse cols needed
  static constexpr int PITCH = ((CC + VEC - 1 + VEC - 1) / VEC) * VEC;
  static constexpr int PLANE = CR * PITCH;
  static constexpr int NS = D + 1;
  static constexpr int TB = CR * FZ;
  static constexpr size_t SMEM = ((size_t)NS * PLANE + TB) * sizeof(T);
};

template <class C>
__global__ void __launch_bounds__(C::NT) interpolate_kernel(const TrArgs a) {
  using T = typename C::T;
  using R = typename Elem<T>::R;
  constexpr int K = C::K, FY = C::FY, FZ = C::FZ, RY = C::RY, RZ = C::RZ, D = C::D;
  constexpr int TZ = C::TZ, NT = C::NT, VEC = C::VEC, CR = C::CR, PITCH = C::PITCH;
  constexpr int PLANE = C::PLANE, NS = C::NS, KH = K / 2;
  constexpr bool CPLX = Elem<T>::cplx;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ring = reinterpret_cast<T*>(smem_raw);
  T* tbuf = ring + NS * PLANE;

  const int tid = threadIdx.x, ty = tid / TZ, tz = tid % TZ;
  const int nc0 = a.ni[0], nc1 = a.ni[1], nc2 = a.ni[2];
  const int nf0 = a.no[0], nf1 = a.no[1], nf2 = a.no[2];
  const int64_t nc12 = (int64_t)nc1 * nc2, nf12 = (int64_t)nf1 * nf2;
  const int64_t ntiles = (int64_t)a.tiles1 * a.tiles2;
  // output pairs along axis 0: global coarse C from cmin to cmin + nsteps
  const int cmin = floor_div(a.skip0[0], 2);
  const int64_t total = a.nbatch * ntiles * a.nsteps;
  int64_t s = total * blockIdx.x / gridDim.x;
  const int64_t s_end = total * (blockIdx.x + 1) / gridDim.x;
  R w[KH];
#pragma unroll
  for (int m = 0; m < KH; ++m) w[m] = (R)a.w[m];
  const R alpha = (R)a.alpha, gamma = (R)a.gamma;

  while (s < s_end) {
    const int64_t col = s / a.nsteps;
    const int Ps = (int)(s % a.nsteps);
    const int Pe = (int)((s_end - s) < (int64_t)(a.nsteps - Ps) ? Ps + (s_end - s) : a.nsteps);
    s += Pe - Ps;
    const int64_t band = col / ntiles;
    const int t = (int)(col % ntiles);
    const int Y0 = (t / a.tiles2) * FY, Z0 = (t % a.tiles2) * FZ;
    const T* src = reinterpret_cast<const T*>(a.in) + band * nc12 * nc0;
    T* dst = reinterpret_cast<T*>(a.out) + band * nf12 * nf0;
    const auto& PH = a.phs.ph[phase_set_of(a.phs, band)];
    const T* ysrc = a.y ? reinterpret_cast<const T*>(a.y) + band * nf12 * nf0 : nullptr;
    // coarse rows / cols staged: global coarse index base, local = global - cbeg
    const int crow0 = floor_div(Y0 + a.skip0[1], 2) - (KH - 1);          // global coarse row of staged row 0
    const int ry0 = crow0 - a.cbeg[1];                                    // local
    const int ccol0 = floor_div(Z0 + a.skip0[2], 2) - (KH - 1);
    const int cl = ccol0 - a.cbeg[2];
    const int cx0 = floor_div(cl, VEC) * VEC;
    const int sh = cl - cx0;
    const bool edge = ry0 < 0 || ry0 + CR > nc1 || cx0 < 0 || cx0 + PITCH > nc2;
    // coarse planes (global) needed for output pairs [cmin+Ps, cmin+Pe)
    const int g0 = cmin + Ps - (KH - 1), g1 = cmin + Pe + KH;   // [g0, g1)

    auto src_plane = [&](int g, double& pr, double& pi) -> int {
      pr = 1.0; pi = 0.0;
      const int l = g - a.cbeg[0];
      if (l >= 0 && l < nc0) return l;
      if (!a.pbc[0]) return -1;
      const int sd = l < 0;
      pr = PH[0][sd][0]; pi = PH[0][sd][1];
      return tr_mod(l, nc0);
    };
    auto issue = [&](int g) {
      double pr, pi;
      const int sp = src_plane(g, pr, pi);
      if (sp < 0) return;
      stage_plane<T, CR, PITCH, PITCH, NT>(ring + ((g - g0) % NS) * PLANE, src + (int64_t)sp * nc12,
                                           ry0, cx0, nc1, nc2, a.pbc[1], a.pbc[2], tid);
    };

    T q[K][RY][RZ];
#pragma unroll
    for (int m = 0; m < K; ++m)
#pragma unroll
      for (int r = 0; r < RY; ++r)
#pragma unroll
        for (int c = 0; c < RZ; ++c) q[m][r][c] = zero<T>();
#pragma unroll
    for (int d = 0; d < D; ++d) {
      if (g0 + d < g1) issue(g0 + d);
      cp_async_commit();
    }
    for (int g = g0; g < g1; ++g) {
      cp_async_wait<D - 1>();
      __syncthreads();
      double pr, pi;
      const int sp = src_plane(g, pr, pi);
      T* P = ring + ((g - g0) % NS) * PLANE;
      T u[RY][RZ];
      if (sp >= 0) {
        if (CPLX && a.phs.any && edge) {
          phase_fixup<T, CR, PITCH, PITCH, NT>(P, ry0, cx0, nc1, nc2, a, PH, tid);
          __syncthreads();
        }
        // pass A: along axis 2, every staged coarse row -> FZ fine columns
        for (int e = tid; e < CR * FZ; e += NT) {
          const int r = e / FZ, fc = e % FZ;
          const int F = Z0 + fc + a.skip0[2];
          const T* row = P + r * PITCH + sh;
          T x;
          if ((F & 1) == 0) {
            x = row[(F >> 1) - ccol0];
          } else {
            const int cc = ((F - 1) >> 1) - ccol0;
            x = scale(w[0], add(row[cc], row[cc + 1]));
#pragma unroll
            for (int m = 1; m < KH; ++m) x = fmadd(x, w[m], add(row[cc - m], row[cc + 1 + m]));
          }
          tbuf[r * FZ + fc] = x;
        }
        __syncthreads();
        // pass B: along axis 1 for the own fine points
#pragma unroll
        for (int r = 0; r < RY; ++r) {
          const int F = Y0 + ty * RY + r + a.skip0[1];
#pragma unroll
          for (int c = 0; c < RZ; ++c) {
            const T* tc = tbuf + tz * RZ + c;
            T x;
            if ((F & 1) == 0) {
              x = tc[((F >> 1) - crow0) * FZ];
            } else {
              const int cr = ((F - 1) >> 1) - crow0;
              x = scale(w[0], add(tc[cr * FZ], tc[(cr + 1) * FZ]));
#pragma unroll
              for (int m = 1; m < KH; ++m) x = fmadd(x, w[m], add(tc[(cr - m) * FZ], tc[(cr + 1 + m) * FZ]));
            }
            u[r][c] = CPLX ? phase_mul(x, pr, pi) : x;
          }
        }
      } else {
#pragma unroll
        for (int r = 0; r < RY; ++r)
#pragma unroll
          for (int c = 0; c < RZ; ++c) u[r][c] = zero<T>();
      }
#pragma unroll
      for (int m = 0; m < K - 1; ++m)
#pragma unroll
        for (int r = 0; r < RY; ++r)
#pragma unroll
          for (int c = 0; c < RZ; ++c) q[m][r][c] = q[m + 1][r][c];
#pragma unroll
      for (int r = 0; r < RY; ++r)
#pragma unroll
        for (int c = 0; c < RZ; ++c) q[K - 1][r][c] = u[r][c];
      // output fine planes 2C and 2C+1 for C = g - KH once coarse C+KH is in
      const int Cg = g - KH;
      if (Cg >= cmin + Ps) {
#pragma unroll
        for (int par = 0; par < 2; ++par) {
          const int f = 2 * Cg + par - a.skip0[0];
          if (f < 0 || f >= nf0) continue;
          T* op = dst + (int64_t)f * nf12;
          const T* yp = ysrc ? ysrc + (int64_t)f * nf12 : nullptr;
#pragma unroll
          for (int r = 0; r < RY; ++r) {
            const int yi = Y0 + ty * RY + r;
            if (yi >= nf1) continue;
#pragma unroll
            for (int c = 0; c < RZ; ++c) {
              const int zi = Z0 + tz * RZ + c;
              if (zi >= nf2) continue;
              T x;
              if (par == 0) {
                x = q[KH - 1][r][c];
              } else {
                x = scale(w[0], add(q[KH - 1][r][c], q[KH][r][c]));
#pragma unroll
                for (int m = 1; m < KH; ++m) x = fmadd(x, w[m], add(q[KH - 1 - m][r][c], q[KH + m][r][c]));
              }
              x = scale(alpha, x);
              const int64_t o = (int64_t)yi * nf2 + zi;
              if (yp) x = fmadd(x, gamma, yp[o]);
              op[o] = x;
            }
          }
        }
      }
      __syncthreads();
      if (g + D < g1) issue(g + D);
      cp_async_commit();
    }
    cp_async_wait<0>();
    __syncthreads();
  }
}

// ---------------------------------------------------------------- host side
static void midpoint_weights(int k, double* w) {
  // Lagrange weights of the degree-(k-1) interpolant through +-1/2, +-3/2, ...
  // at 0, for the pairs at distance (2j+1)/2 (the k = 2, 4, 6, 8 weights of
  // c/bmgs/restrict.c:36-56 and c/bmgs/interpolate.c:184-197).
  for (int j = 0; j < k / 2; ++j) {
    const double xj = (2 * j + 1) / 2.0;
    double num = 1.0, den = 1.0;
    for (int i = 0; i < k; ++i) {
      const double xi = (2 * i - k + 1) / 2.0;
      if (xi == xj) continue;
      num *= -xi;
      den *= xj - xi;
    }
    w[j] = num / den;
  }
}

static void fill_common(const gb_transformer* t, TrArgs& a, const double* ph, int nk, int64_t nbatch) {
  memset(&a, 0, sizeof(a));
  for (int c = 0; c < 3; ++c) {
    a.ni[c] = (int)t->nin_c[c];
    a.no[c] = (int)t->nout_c[c];
    a.pbc[c] = t->pbc[c];
    a.off[c] = t->off[c];
    a.skip0[c] = t->skip0[c];
    a.cbeg[c] = t->cbeg[c];
  }
  midpoint_weights(t->k, a.w);
  fill_phase_sets(a.phs, ph, nk, nbatch);
}

template <class C, typename KernelT>
static int launch_persistent(KernelT kernel, const TrArgs& a, int64_t total, cudaStream_t st, int min_steps) {
  static int occ = -1;
  if (occ < 0) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, C::NT, C::SMEM);
    if (occ < 1) occ = 1;
  }
  int64_t blocks = (int64_t)sm_count() * occ;
  // at least min_steps planes per CTA amortise its (2K-1)-plane prologue --
  // unless that would leave SMs idle (one small grid, e.g. the density's
  // 112^3 -> 56^3): then the prologue's L2 re-reads cost less than idle SMs
  const int64_t by_steps = total / min_steps;
  blocks = std::min<int64_t>(blocks, by_steps >= sm_count() ? by_steps : std::max<int64_t>(1, total));
  kernel<<<(unsigned)blocks, C::NT, C::SMEM, st>>>(a);
  return check_launch("transformer kernel");
}

template <typename T, int K, int CY, int CZ>
static int restrict_cfg(const gb_transformer* t, const void* in, void* out, int64_t nin,
                        const double* ph, cudaStream_t st, double alpha, int nk) {
  using C = RCfg<T, K, CY, CZ, 2>;
  TrArgs a;
  fill_common(t, a, ph, nk, nin);
  a.in = in; a.out = out; a.nbatch = nin; a.alpha = alpha;
  a.tiles1 = ceil_div(a.no[1], C::CY);
  a.tiles2 = ceil_div(a.no[2], C::CZ);
  const int64_t total = nin * (int64_t)a.tiles1 * a.tiles2 * a.no[0];
  return launch_persistent<C>(restrict_kernel<C>, a, total, st, 4 + K);
}

// k = 2 restriction of real data on a grid periodic on every axis (the
// preconditioner's and the learned network's first transfer), marching
// along axis 0: a CTA owns TYC coarse rows of one band over a chunk of
// coarse planes; each fine plane it needs (rows 2 J0 - 1 .. 2 J0 + 2 TYC - 1
// plus the wrap-around columns) is staged once with cp.async into a two-slot
// ring, every thread restricts it in-plane for two neighbouring coarse
// points (axis 2, then axis 1: the general kernel's arithmetic, in its
// order) and the axis-0 step takes the last three fine planes from a
// register queue.  Rows must be 16-byte aligned.
// four consecutive values from a 16-byte aligned shared-memory address
__device__ __forceinline__ void load4(const float* f, float (&v)[4]) {
  const float4 q = *reinterpret_cast<const float4*>(f);
  v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void load4(const double* f, double (&v)[4]) {
  const double2 q0 = reinterpret_cast<const double2*>(f)[0], q1 = reinterpret_cast<const double2*>(f)[1];
  v[0] = q0.x; v[1] = q0.y; v[2] = q1.x; v[3] = q1.y;
}

template <typename T, int TYC>
__global__ void __launch_bounds__(256) restrict2_march_kernel(const TrArgs a, int nch) {
  extern __shared__ __align__(16) unsigned char r2m_smem[];
  T* slot = reinterpret_cast<T*>(r2m_smem);
  constexpr int VEC = 16 / (int)sizeof(T);
  const int nf0 = a.ni[0], nf1 = a.ni[1], nf2 = a.ni[2];
  const int nc0 = a.no[0], nc1 = a.no[1], nc2 = a.no[2];
  const int FR = 2 * TYC + 1, FP = nf2 + 2 * VEC + 8;   // fine column c at VEC + c
  const int tid = threadIdx.x, nt = blockDim.x;
  const int ngx = (nc2 + 1) >> 1;
  const int gx = tid % ngx, ty = tid / ngx;
  const int J0 = blockIdx.y * TYC, J = J0 + ty, K0 = 2 * gx;
  const int64_t b = blockIdx.z;
  const int I_beg = (int)((int64_t)blockIdx.x * nc0 / nch), I_end = (int)((int64_t)(blockIdx.x + 1) * nc0 / nch);
  const T* src = reinterpret_cast<const T*>(a.in) + b * (int64_t)nf0 * nf1 * nf2;
  T* dst = reinterpret_cast<T*>(a.out) + b * (int64_t)nc0 * nc1 * nc2;
  const T w0 = (T)a.w[0], half = (T)0.5, alpha = (T)a.alpha;
  const int r0 = 2 * J0 + a.off[1] - 1;                 // first staged fine row
  auto wrap = [](int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); };
  // the copies of a staged plane: element e = (row r, piece c) is a 16-byte
  // chunk (c < chunks), column -1 or column nf2; a thread's first MAXU
  // elements have their offsets worked out once (no index divisions per plane)
  const int chunks = nf2 / VEC, ne = FR * (chunks + 2);
  constexpr int MAXU = 4;
  int s_off[MAXU], d_off[MAXU];
  unsigned wide = 0u;
#pragma unroll
  for (int u = 0; u < MAXU; ++u) {
    const int e = tid + u * nt;
    s_off[u] = 0;
    d_off[u] = -1;
    if (e < ne) {
      const int r = e / (chunks + 2), c = e % (chunks + 2);
      const int row = wrap(r0 + r, nf1) * nf2;
      if (c < chunks) {
        s_off[u] = row + c * VEC;
        d_off[u] = r * FP + VEC + c * VEC;
        wide |= 1u << u;
      } else if (c == chunks) {
        s_off[u] = row + nf2 - 1;                 // column -1
        d_off[u] = r * FP + VEC - 1;
      } else {
        s_off[u] = row;                           // column nf2
        d_off[u] = r * FP + VEC + nf2;
      }
    }
  }
  auto stage = [&](int p, T* d) {
    const T* pl = src + (int64_t)wrap(p, nf0) * nf1 * nf2;
#pragma unroll
    for (int u = 0; u < MAXU; ++u) {
      if (d_off[u] < 0) continue;
      if (wide & (1u << u)) cp_async16(d + d_off[u], pl + s_off[u]);
      else cp_async_elem(d + d_off[u], pl + s_off[u]);
    }
    for (int e = tid + MAXU * nt; e < ne; e += nt) {
      const int r = e / (chunks + 2), c = e % (chunks + 2);
      const T* row = pl + (int64_t)wrap(r0 + r, nf1) * nf2;
      T* dr = d + r * FP;
      if (c < chunks) cp_async16(dr + VEC + c * VEC, row + c * VEC);
      else if (c == chunks) cp_async_elem(dr + VEC - 1, row + nf2 - 1);   // column -1
      else cp_async_elem(dr + VEC + nf2, row);                          // column nf2
    }
  };
  // the five fine columns 2K - 1 .. 2K + 3 a thread reads per row: one
  // 16-byte load and one scalar when the window start is 16-byte aligned
  const bool vec4 = (a.off[2] % VEC) == 0;
  const int p_beg = 2 * I_beg + a.off[0] - 1, p_end = 2 * (I_end - 1) + a.off[0] + 1;
  stage(p_beg, slot);
  cp_async_commit();
  T q0[2] = {0, 0}, q1[2] = {0, 0}, q2[2] = {0, 0};
  const bool act = ty < TYC && J < nc1;
  for (int p = p_beg; p <= p_end; ++p) {
    const int s = (p - p_beg) & 1;
    if (p + 1 <= p_end) stage(p + 1, slot + (s ^ 1) * FR * FP);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    if (act) {
      const T* P = slot + s * FR * FP + 2 * ty * FP + VEC + 2 * K0 + a.off[2];
      T g[3][2];
#pragma unroll
      for (int dy = 0; dy < 3; ++dy) {
        const T* f = P + dy * FP;
        T v[4];
        if (vec4) {
          load4(f, v);
        } else {
#pragma unroll
          for (int i = 0; i < 4; ++i) v[i] = f[i];
        }
        const T fm = f[-1];
        g[dy][0] = half * fmadd(v[0], w0, add(v[1], fm));
        g[dy][1] = half * fmadd(v[2], w0, add(v[3], v[1]));
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        q0[h] = q1[h];
        q1[h] = q2[h];
        q2[h] = half * fmadd(g[1][h], w0, add(g[2][h], g[0][h]));
      }
      const int tI = p - a.off[0] - 1;                  // fine plane 2I + off + 1 just arrived
      if (tI >= 2 * I_beg && (tI & 1) == 0) {
        const int I = tI >> 1;
        T* o = dst + ((int64_t)I * nc1 + J) * nc2 + K0;
#pragma unroll
        for (int h = 0; h < 2; ++h)
          if (K0 + h < nc2) o[h] = alpha * (half * fmadd(q1[h], w0, add(q2[h], q0[h])));
      }
    }
    __syncthreads();
  }
  cp_async_wait<0>();
}

template <typename T>
static int restrict2_march_launch(const gb_transformer* t, const void* in, void* out, int64_t nin,
                                  cudaStream_t st, double alpha) {
  constexpr int VEC = 16 / (int)sizeof(T);
  TrArgs a;
  fill_common(t, a, nullptr, 1, nin);
  a.in = in; a.out = out; a.nbatch = nin; a.alpha = alpha;
  const int ngx = (a.no[2] + 1) / 2;
  const int TYC = ngx * 8 <= 256 ? 8 : (ngx * 4 <= 256 ? 4 : 2);
  const int nch = std::max(1, std::min(a.no[0], a.no[0] / 8));
  const size_t smem = (size_t)2 * (2 * TYC + 1) * (a.ni[2] + 2 * VEC + 8) * sizeof(T);
  const dim3 grid((unsigned)nch, (unsigned)((a.no[1] + TYC - 1) / TYC), (unsigned)nin);
  const unsigned threads = (unsigned)(ngx * TYC);
  if (TYC == 8) restrict2_march_kernel<T, 8><<<grid, threads, smem, st>>>(a, nch);
  else if (TYC == 4) restrict2_march_kernel<T, 4><<<grid, threads, smem, st>>>(a, nch);
  else restrict2_march_kernel<T, 2><<<grid, threads, smem, st>>>(a, nch);
  return check_launch("restrict2_march_kernel");
}

template <typename T>
static bool restrict2_march_ok(const gb_transformer* t, int64_t nin, const double* ph) {
  if (!t->pbc[0] || !t->pbc[1] || !t->pbc[2] || nin > 65535 || nin < 1) return false;
  if (ph)
    for (int i = 0; i < 12; ++i)
      if (ph[i] != ((i % 2) ? 0.0 : 1.0)) return false;
  const int64_t nf2 = t->nin_c[2];
  const int64_t ngx = (t->nout_c[2] + 1) / 2;
  const int64_t tyc = ngx * 8 <= 256 ? 8 : (ngx * 4 <= 256 ? 4 : 2);
  // single-wrap periodic indices: at least 2 * TYC fine rows, 2 planes
  return (nf2 * (int64_t)sizeof(T)) % 16 == 0 && ngx * 2 <= 256 && t->nin_c[0] >= 2 &&
         t->nin_c[1] >= 2 * tyc && nf2 >= 2 * (16 / (int)sizeof(T)) && t->nout_c[1] >= 1;
}

// k = 2 interpolation of real data on a grid periodic on every axis (fine
// point 2C on coarse point C), marching along axis 0 over coarse planes: a
// CTA owns TYF fine rows of one band over a chunk of coarse planes; each
// coarse plane (rows F0/2 .. F0/2 + TYF/2 plus the wrap-around column) is
// staged once into a two-slot ring; every thread interpolates it for four
// neighbouring fine columns of its row (axis 2, then axis 1: the general
// kernel's arithmetic, in its order) and, once coarse plane C + 1 is in,
// writes fine planes 2C and 2C + 1 with the alpha / gamma * y epilogue as
// 16-byte vectors.  Rows must be 16-byte aligned.
template <typename T, int TYF>
__global__ void __launch_bounds__(256) interp2_march_kernel(const TrArgs a, int nch) {
  extern __shared__ __align__(16) unsigned char i2m_smem[];
  T* slot = reinterpret_cast<T*>(i2m_smem);
  constexpr int VEC = 16 / (int)sizeof(T);
  constexpr int CRR = TYF / 2 + 1;
  const int nc0 = a.ni[0], nc1 = a.ni[1], nc2 = a.ni[2];
  const int nf1 = a.no[1], nf2 = a.no[2];
  const int CP = nc2 + 2 * VEC + 8;                    // coarse column c at VEC + c
  const int tid = threadIdx.x, nt = blockDim.x;
  const int ngx = nf2 >> 2;
  const int gx = tid % ngx, ty = tid / ngx;
  const int F0 = blockIdx.y * TYF, F = F0 + ty, k = 4 * gx;
  const int64_t b = blockIdx.z;
  const int C_beg = (int)((int64_t)blockIdx.x * nc0 / nch), C_end = (int)((int64_t)(blockIdx.x + 1) * nc0 / nch);
  const T* src = reinterpret_cast<const T*>(a.in) + b * (int64_t)nc0 * nc1 * nc2;
  const int64_t fplane = (int64_t)nf1 * nf2;
  T* dst = reinterpret_cast<T*>(a.out) + b * 2 * (int64_t)nc0 * fplane;
  const T* ysrc = a.y ? reinterpret_cast<const T*>(a.y) + b * 2 * (int64_t)nc0 * fplane : nullptr;
  const T w0 = (T)a.w[0], alpha = (T)a.alpha, gamma = (T)a.gamma;
  auto wrap = [](int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); };
  // rows of a whole number of 16-byte chunks are copied in chunks, others
  // (a 14-point FP32 row, say) element by element
  const bool rows16 = (nc2 * (int)sizeof(T)) % 16 == 0;
  auto stage = [&](int g, T* d) {
    const T* pl = src + (int64_t)wrap(g, nc0) * nc1 * nc2;
    if (rows16) {
      const int chunks = nc2 / VEC;
      for (int e = tid; e < CRR * (chunks + 1); e += nt) {
        const int r = e / (chunks + 1), c = e % (chunks + 1);
        const T* row = pl + (int64_t)wrap((F0 >> 1) + r, nc1) * nc2;
        T* dr = d + r * CP;
        if (c < chunks) cp_async16(dr + VEC + c * VEC, row + c * VEC);
        else cp_async_elem(dr + VEC + nc2, row);                 // column nc2
      }
    } else {
      for (int e = tid; e < CRR * (nc2 + 1); e += nt) {
        const int r = e / (nc2 + 1), c = e % (nc2 + 1);
        const T* row = pl + (int64_t)wrap((F0 >> 1) + r, nc1) * nc2;
        cp_async_elem(d + r * CP + VEC + c, row + (c < nc2 ? c : 0));   // column nc2 = column 0
      }
    }
  };
  stage(C_beg, slot);
  cp_async_commit();
  T qp[4];                                             // u of the previous coarse plane
  const bool act = ty < TYF && F < nf1;
  for (int g = C_beg; g <= C_end; ++g) {
    const int s = (g - C_beg) & 1;
    if (g + 1 <= C_end) stage(g + 1, slot + (s ^ 1) * CRR * CP);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    if (act) {
      const T* P = slot + s * CRR * CP + VEC + (k >> 1);
      const int rl = (F >> 1) - (F0 >> 1);
      T A[2][4];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const T* row = P + (rl + h) * CP;
        const T c0 = row[0], c1 = row[1], c2 = row[2];
        A[h][0] = c0;
        A[h][1] = w0 * add(c0, c1);
        A[h][2] = c1;
        A[h][3] = w0 * add(c1, c2);
      }
      T u[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) u[q] = (F & 1) ? w0 * add(A[0][q], A[1][q]) : A[0][q];
      if (g > C_beg) {
        const int C = g - 1;
#pragma unroll
        for (int par = 0; par < 2; ++par) {
          const int64_t o = (int64_t)(2 * C + par) * fplane + (int64_t)F * nf2 + k;
          T x[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            T v = par == 0 ? qp[q] : w0 * add(qp[q], u[q]);
            v = alpha * v;
            if (ysrc) v = fmadd(v, gamma, ysrc[o + q]);
            x[q] = v;
          }
          if constexpr (sizeof(T) == 4) {
            *reinterpret_cast<float4*>(dst + o) = make_float4(x[0], x[1], x[2], x[3]);
          } else {
            reinterpret_cast<double2*>(dst + o)[0] = make_double2(x[0], x[1]);
            reinterpret_cast<double2*>(dst + o)[1] = make_double2(x[2], x[3]);
          }
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) qp[q] = u[q];
    }
    __syncthreads();
  }
  cp_async_wait<0>();
}

template <typename T>
static bool interp2_march_ok(const gb_transformer* t, int64_t nin, const double* ph, const void* y) {
  if (!t->pbc[0] || !t->pbc[1] || !t->pbc[2] || nin > 65535 || nin < 1) return false;
  if (ph)
    for (int i = 0; i < 12; ++i)
      if (ph[i] != ((i % 2) ? 0.0 : 1.0)) return false;
  for (int c = 0; c < 3; ++c)
    if (t->skip0[c] != 0 || t->cbeg[c] != 0 || t->nout_c[c] != 2 * t->nin_c[c]) return false;
  const int64_t nc2 = t->nin_c[2], nf2 = t->nout_c[2];
  const int64_t ngx = nf2 / 4;
  const int64_t tyf = ngx * 8 <= 256 ? 8 : (ngx * 4 <= 256 ? 4 : 2);
  (void)y;
  return nf2 % 4 == 0 && ngx * 2 <= 256 && t->nin_c[0] >= 1 && t->nin_c[1] >= tyf / 2 + 1 &&
         nc2 >= 16 / (int)sizeof(T);
}

template <typename T>
static int interp2_march_launch(const gb_transformer* t, const void* in, void* out, int64_t nin,
                                cudaStream_t st, double alpha, const void* y, double gamma) {
  constexpr int VEC = 16 / (int)sizeof(T);
  TrArgs a;
  fill_common(t, a, nullptr, 1, nin);
  a.in = in; a.out = out; a.nbatch = nin; a.alpha = alpha; a.y = y; a.gamma = gamma;
  const int ngx = a.no[2] / 4;
  const int TYF = ngx * 8 <= 256 ? 8 : (ngx * 4 <= 256 ? 4 : 2);
  const int nch = std::max(1, std::min(a.ni[0], a.ni[0] / 7));
  const size_t smem = (size_t)2 * (TYF / 2 + 1) * (a.ni[2] + 2 * VEC + 8) * sizeof(T);
  const dim3 grid((unsigned)nch, (unsigned)((a.no[1] + TYF - 1) / TYF), (unsigned)nin);
  const unsigned threads = (unsigned)(ngx * TYF);
  if (TYF == 8) interp2_march_kernel<T, 8><<<grid, threads, smem, st>>>(a, nch);
  else if (TYF == 4) interp2_march_kernel<T, 4><<<grid, threads, smem, st>>>(a, nch);
  else interp2_march_kernel<T, 2><<<grid, threads, smem, st>>>(a, nch);
  return check_launch("interp2_march_kernel");
}

// coarse rows of at most 16 points (the coarse levels of small grids) use a
// 16 x 16 tile, wider ones 8 x 32: no more than half a warp idles on a row
// k = 6 restriction of real data on a grid periodic on every axis (the
// density / potential transfers between the coarse and the fine grid),
// marching along axis 0 like restrict2_march_kernel: a CTA owns TYC coarse
// rows of one band over a chunk of coarse planes and stages every fine
// plane it needs once (rows 2 J0 + off - 5 .. 2 (J0 + TYC - 1) + off + 5,
// five wrap-around columns on each side) with cp.async into a two-slot
// ring.  A thread restricts the plane in-plane for two neighbouring coarse
// points -- axis 2 on each of its seven fine rows, then axis 1 -- and the
// axis-0 step takes the last eleven fine planes from a register queue; the
// arithmetic of the general kernel (x = f0, x += w_m (f_{2m+1} + f_{-2m-1}),
// m = 0, 1, 2, then x / 2, axis by axis), in its order.  Rows must be
// 16-byte aligned.
template <typename T, int TYC>
__global__ void __launch_bounds__(256) restrict6_march_kernel(const TrArgs a, int nch) {
  extern __shared__ __align__(16) unsigned char r6m_smem[];
  T* slot = reinterpret_cast<T*>(r6m_smem);
  constexpr int VEC = 16 / (int)sizeof(T);
  constexpr int CO = ((5 + VEC - 1) / VEC) * VEC;        // fine column c at CO + c
  const int nf0 = a.ni[0], nf1 = a.ni[1], nf2 = a.ni[2];
  const int nc0 = a.no[0], nc1 = a.no[1], nc2 = a.no[2];
  const int FR = 2 * TYC + 9, FP = nf2 + 2 * CO + 2 * VEC;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int ngx = (nc2 + 1) >> 1;
  const int gx = tid % ngx, ty = tid / ngx;
  const int J0 = blockIdx.y * TYC, J = J0 + ty, K0 = 2 * gx;
  const int64_t b = blockIdx.z;
  const int I_beg = (int)((int64_t)blockIdx.x * nc0 / nch), I_end = (int)((int64_t)(blockIdx.x + 1) * nc0 / nch);
  const T* src = reinterpret_cast<const T*>(a.in) + b * (int64_t)nf0 * nf1 * nf2;
  T* dst = reinterpret_cast<T*>(a.out) + b * (int64_t)nc0 * nc1 * nc2;
  const T w0 = (T)a.w[0], w1 = (T)a.w[1], w2 = (T)a.w[2], half = (T)0.5, alpha = (T)a.alpha;
  const int r0 = 2 * J0 + a.off[1] - 5;                 // first staged fine row
  auto wrap = [](int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); };
  // element e = (row r, piece c): 16-byte chunks c < chunks, then the five
  // columns -5 .. -1 and the five columns nf2 .. nf2 + 4
  const int chunks = nf2 / VEC, per = chunks + 10, ne = FR * per;
  constexpr int MAXU = 8;
  int s_off[MAXU], d_off[MAXU];
  unsigned wide = 0u;
#pragma unroll
  for (int u = 0; u < MAXU; ++u) {
    const int e = tid + u * nt;
    s_off[u] = 0;
    d_off[u] = -1;
    if (e < ne) {
      const int r = e / per, c = e % per;
      const int row = wrap(r0 + r, nf1) * nf2;
      if (c < chunks) {
        s_off[u] = row + c * VEC;
        d_off[u] = r * FP + CO + c * VEC;
        wide |= 1u << u;
      } else if (c < chunks + 5) {
        const int h = c - chunks;                   // column h - 5
        s_off[u] = row + nf2 - 5 + h;
        d_off[u] = r * FP + CO - 5 + h;
      } else {
        const int h = c - chunks - 5;               // column nf2 + h
        s_off[u] = row + h;
        d_off[u] = r * FP + CO + nf2 + h;
      }
    }
  }
  auto stage = [&](int p, T* d) {
    const T* pl = src + (int64_t)wrap(p, nf0) * nf1 * nf2;
#pragma unroll
    for (int u = 0; u < MAXU; ++u) {
      if (d_off[u] < 0) continue;
      if (wide & (1u << u)) cp_async16(d + d_off[u], pl + s_off[u]);
      else cp_async_elem(d + d_off[u], pl + s_off[u]);
    }
    for (int e = tid + MAXU * nt; e < ne; e += nt) {
      const int r = e / per, c = e % per;
      const T* row = pl + (int64_t)wrap(r0 + r, nf1) * nf2;
      T* dr = d + r * FP + CO;
      if (c < chunks) cp_async16(dr + c * VEC, row + c * VEC);
      else if (c < chunks + 5) cp_async_elem(dr - 5 + (c - chunks), row + nf2 - 5 + (c - chunks));
      else cp_async_elem(dr + nf2 + (c - chunks - 5), row + (c - chunks - 5));
    }
  };
  // one axis: x = f0; x += w_m (f_{2m+1} + f_{-(2m+1)}); x / 2
  auto axis = [&](T c0, T p1, T m1, T p3, T m3, T p5, T m5) {
    T x = c0;
    x = fmadd(x, w0, add(p1, m1));
    x = fmadd(x, w1, add(p3, m3));
    x = fmadd(x, w2, add(p5, m5));
    return half * x;
  };
  const int p_beg = 2 * I_beg + a.off[0] - 5, p_end = 2 * (I_end - 1) + a.off[0] + 5;
  stage(p_beg, slot);
  cp_async_commit();
  T q[2][11];
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int m = 0; m < 11; ++m) q[h][m] = (T)0;
  const bool act = ty < TYC && J < nc1;
  for (int p = p_beg; p <= p_end; ++p) {
    const int s = (p - p_beg) & 1;
    if (p + 1 <= p_end) stage(p + 1, slot + (s ^ 1) * FR * FP);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    if (act) {
      // centre fine row 2J + off of this thread: staged row 2 ty + 5
      const T* P = slot + s * FR * FP + (2 * ty + 5) * FP + CO + 2 * K0 + a.off[2];
      T g[2][11];                                      // [h][fine row offset + 5]
#pragma unroll
      for (int dy = -5; dy <= 5; ++dy) {
        if (dy != 0 && (dy & 1) == 0) continue;        // even offsets carry no weight
        const T* f = P + dy * FP;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const T* c = f + 2 * h;
          g[h][dy + 5] = axis(c[0], c[1], c[-1], c[3], c[-3], c[5], c[-5]);
        }
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
#pragma unroll
        for (int m = 0; m < 10; ++m) q[h][m] = q[h][m + 1];
        q[h][10] = axis(g[h][5], g[h][6], g[h][4], g[h][8], g[h][2], g[h][10], g[h][0]);
      }
      const int tI = p - a.off[0] - 5;                  // fine plane 2I + off + 5 just arrived
      if (tI >= 2 * I_beg && (tI & 1) == 0) {
        const int I = tI >> 1;
        T* o = dst + ((int64_t)I * nc1 + J) * nc2 + K0;
#pragma unroll
        for (int h = 0; h < 2; ++h)
          if (K0 + h < nc2) o[h] = alpha * axis(q[h][5], q[h][6], q[h][4], q[h][8], q[h][2], q[h][10], q[h][0]);
      }
    }
    __syncthreads();
  }
  cp_async_wait<0>();
}

template <typename T>
static bool restrict6_march_ok(const gb_transformer* t, int64_t nin, const double* ph) {
  if (!t->pbc[0] || !t->pbc[1] || !t->pbc[2] || nin > 65535 || nin < 1) return false;
  if (ph)
    for (int i = 0; i < 12; ++i)
      if (ph[i] != ((i % 2) ? 0.0 : 1.0)) return false;
  const int64_t nf2 = t->nin_c[2];
  const int64_t ngx = (t->nout_c[2] + 1) / 2;
  const int64_t tyc = ngx * 8 <= 256 ? 8 : (ngx * 4 <= 256 ? 4 : 2);
  // single-wrap periodic indices: at least 6 fine planes and columns, and
  // rows enough that the last tile's staged rows (up to nf1 + 2 TYC + 2)
  // stay below 2 nf1
  return (nf2 * (int64_t)sizeof(T)) % 16 == 0 && ngx * 2 <= 256 && t->nin_c[0] >= 6 &&
         t->nin_c[1] >= 2 * tyc + 3 && nf2 >= 6 && t->nout_c[1] >= 1 && t->nout_c[0] >= 1;
}

template <typename T>
static int restrict6_march_launch(const gb_transformer* t, const void* in, void* out, int64_t nin,
                                  cudaStream_t st, double alpha) {
  constexpr int VEC = 16 / (int)sizeof(T);
  constexpr int CO = ((5 + VEC - 1) / VEC) * VEC;
  TrArgs a;
  fill_common(t, a, nullptr, 1, nin);
  a.in = in; a.out = out; a.nbatch = nin; a.alpha = alpha;
  const int ngx = (a.no[2] + 1) / 2;
  const int TYC = ngx * 8 <= 256 ? 8 : (ngx * 4 <= 256 ? 4 : 2);
  // plane chunks: enough CTAs for every SM (a single grid is cut into
  // short chunks, each re-staging its ten halo planes from L2)
  const int64_t tiles = (int64_t)((a.no[1] + TYC - 1) / TYC) * nin;
  const int nch = (int)std::max<int64_t>(1, std::min<int64_t>(a.no[0], (sm_count() + tiles - 1) / tiles));
  const size_t smem = (size_t)2 * (2 * TYC + 9) * (a.ni[2] + 2 * CO + 2 * VEC) * sizeof(T);
  static size_t attr = 0;
  if (smem > 48 * 1024 && smem > attr) {
    cudaFuncSetAttribute(restrict6_march_kernel<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(restrict6_march_kernel<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(restrict6_march_kernel<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr = smem;
  }
  const dim3 grid((unsigned)nch, (unsigned)((a.no[1] + TYC - 1) / TYC), (unsigned)nin);
  const unsigned threads = (unsigned)(ngx * TYC);
  if (TYC == 8) restrict6_march_kernel<T, 8><<<grid, threads, smem, st>>>(a, nch);
  else if (TYC == 4) restrict6_march_kernel<T, 4><<<grid, threads, smem, st>>>(a, nch);
  else restrict6_march_kernel<T, 2><<<grid, threads, smem, st>>>(a, nch);
  return check_launch("restrict6_march_kernel");
}

template <typename T, int K>
static int restrict_k(const gb_transformer* t, const void* in, void* out, int64_t nin,
                      const double* ph, cudaStream_t st, double alpha, int nk) {
  if constexpr (K == 2 && !Elem<T>::cplx) {
    if (restrict2_march_ok<T>(t, nin, ph)) return restrict2_march_launch<T>(t, in, out, nin, st, alpha);
  }
  if constexpr (K == 6 && !Elem<T>::cplx) {
    if (restrict6_march_ok<T>(t, nin, ph)) return restrict6_march_launch<T>(t, in, out, nin, st, alpha);
  }
  if (t->nout_c[2] <= 16) return restrict_cfg<T, K, 16, 16>(t, in, out, nin, ph, st, alpha, nk);
  return restrict_cfg<T, K, 8, 32>(t, in, out, nin, ph, st, alpha, nk);
}

template <typename T, int K>
static int interpolate_k(const gb_transformer* t, const void* in, void* out, int64_t nin,
                         const double* ph, cudaStream_t st, double alpha, const void* y, double gamma,
                         int nk) {
  if constexpr (K == 2 && !Elem<T>::cplx) {
    if (interp2_march_ok<T>(t, nin, ph, y)) return interp2_march_launch<T>(t, in, out, nin, st, alpha, y, gamma);
  }
  constexpr int RZ = sizeof(T) == 4 ? 4 : (sizeof(T) == 8 ? 2 : 1);
  using C = ICfg<T, K, 16, 32, 2, RZ, 2>;
  TrArgs a;
  fill_common(t, a, ph, nk, nin);
  a.in = in; a.out = out; a.nbatch = nin; a.alpha = alpha; a.y = y; a.gamma = gamma;
  a.tiles1 = ceil_div(a.no[1], C::FY);
  a.tiles2 = ceil_div(a.no[2], C::FZ);
  // output pairs C with 2C - skip0 or 2C + 1 - skip0 in [0, nf0)
  const int cmin = a.skip0[0] >= 0 ? a.skip0[0] / 2 : -((-a.skip0[0] + 1) / 2);
  const int cmax = (a.no[0] - 1 + a.skip0[0]) / 2;
  a.nsteps = cmax - cmin + 1;
  const int64_t total = nin * (int64_t)a.tiles1 * a.tiles2 * a.nsteps;
  return launch_persistent<C>(interpolate_kernel<C>, a, total, st, 4 + K);
}

template <typename T>
static int tr_dispatch(const gb_transformer* t, const void* in, void* out, int64_t nin,
                       const double* ph, cudaStream_t st, double alpha, const void* y, double gamma,
                       int nk) {
  if (t->interpolate) {
    switch (t->k) {
      case 2: return interpolate_k<T, 2>(t, in, out, nin, ph, st, alpha, y, gamma, nk);
      case 4: return interpolate_k<T, 4>(t, in, out, nin, ph, st, alpha, y, gamma, nk);
      case 6: return interpolate_k<T, 6>(t, in, out, nin, ph, st, alpha, y, gamma, nk);
      default: return interpolate_k<T, 8>(t, in, out, nin, ph, st, alpha, y, gamma, nk);
    }
  }
  if (y) return fail(GB_E_UNSUPPORTED, "restriction has no y epilogue");
  switch (t->k) {
    case 2: return restrict_k<T, 2>(t, in, out, nin, ph, st, alpha, nk);
    case 4: return restrict_k<T, 4>(t, in, out, nin, ph, st, alpha, nk);
    case 6: return restrict_k<T, 6>(t, in, out, nin, ph, st, alpha, nk);
    default: return restrict_k<T, 8>(t, in, out, nin, ph, st, alpha, nk);
  }
}

int tr_apply(const gb_transformer* t, const void* in, void* out, int64_t nin, int dtype,
             const double* ph, cudaStream_t st, double alpha, const void* y, double gamma, int nk) {
  if (nk > KMAX) return fail(GB_E_UNSUPPORTED, "more k-point phase sets than one launch takes");
  if (nk > 1 && nin % nk) return fail(GB_E_INVALID, "batch not divisible by the number of phase sets");
  switch (dtype) {
    case GB_DTYPE_F64: return tr_dispatch<double>(t, in, out, nin, ph, st, alpha, y, gamma, nk);
    case GB_DTYPE_F32: return tr_dispatch<float>(t, in, out, nin, ph, st, alpha, y, gamma, nk);
    case GB_DTYPE_C128: return tr_dispatch<double2>(t, in, out, nin, ph, st, alpha, y, gamma, nk);
    default: return tr_dispatch<float2>(t, in, out, nin, ph, st, alpha, y, gamma, nk);
  }
}

}  // namespace gb

using namespace gb;

extern "C" {

int gb_transformer_new(const int64_t size_in[3], const int64_t size_out[3], int k,
                       const int64_t pad_cd[6], const int64_t npad_cd[6], const int64_t skip_cd[6],
                       const int64_t neighbor_cd[6], int real, int interpolate, gb_transformer** out) {
  GB_REQUIRE(out && size_in && size_out && pad_cd && npad_cd && skip_cd && neighbor_cd,
             "gb_transformer_new: null pointer");
  GB_REQUIRE(k == 2 || k == 4 || k == 6 || k == 8, "gb_transformer_new: k must be 2, 4, 6 or 8");
  const int nn = k / 2;
  auto* t = new (std::nothrow) gb_transformer();
  if (!t) return fail(GB_E_NOMEM, "gb_transformer_new: out of host memory");
  t->k = k;
  t->interpolate = interpolate ? 1 : 0;
  t->real = real;
  for (int c = 0; c < 3; ++c) {
    t->nin_c[c] = size_in[c];
    t->nout_c[c] = size_out[c];
    t->pbc[c] = (neighbor_cd[2 * c] >= 0 || neighbor_cd[2 * c + 1] >= 0) ? 1 : 0;
    const int64_t p0 = pad_cd[2 * c], p1 = pad_cd[2 * c + 1];
    if (size_in[c] <= 0 || size_out[c] <= 0 || p0 < 0 || p1 < 0) {
      delete t;
      return fail(GB_E_INVALID, "gb_transformer_new: bad sizes or padding");
    }
    if (!interpolate) {
      // pad0 = 2nn - 1 - (2 beg_out - beg_in)  (gpaw/transformers.py:33)
      t->off[c] = (int)(2 * nn - 1 - p0);
      // output count of the reference: (n_in + pad0 + pad1 - 2k + 3) / 2
      const int64_t nout = (size_in[c] + p0 + p1 - 2 * k + 3) / 2;
      if (nout != size_out[c] || t->off[c] < 0 || t->off[c] > 1) {
        delete t;
        return fail(GB_E_INVALID, "gb_transformer_new: restriction sizes/padding inconsistent");
      }
    } else {
      // pad0 = nn - 1 - beg_out // 2 + beg_in, skip0 = beg_out % 2  (transformers.py:41-46)
      t->skip0[c] = (int)skip_cd[2 * c];
      t->skip1[c] = (int)skip_cd[2 * c + 1];
      t->cbeg[c] = (int)(p0 - nn + 1);
      const int64_t npairs = size_in[c] + p0 + p1 - (k - 1) + t->skip1[c];
      const int64_t nout = 2 * npairs - t->skip0[c] - t->skip1[c];
      if (nout != size_out[c] || t->cbeg[c] < 0 || t->cbeg[c] > 1) {
        delete t;
        return fail(GB_E_INVALID, "gb_transformer_new: interpolation sizes/padding inconsistent");
      }
    }
    (void)npad_cd;
  }
  *out = t;
  return GB_OK;
}

int gb_transformer_apply(const gb_transformer* t, const void* in, void* out, int64_t nin, int dtype,
                         const double* phase_cd, void* stream) {
  GB_REQUIRE(t, "gb_transformer_apply: null transformer");
  GB_REQUIRE(dtype_valid(dtype), "gb_transformer_apply: unknown dtype");
  GB_REQUIRE(nin >= 0, "gb_transformer_apply: negative batch");
  GB_REQUIRE(dtype_complex(dtype) == !t->real,
             "gb_transformer_apply: dtype does not match the transformer's real/complex flag");
  if (nin == 0) return GB_OK;
  GB_REQUIRE(in && out && in != out, "gb_transformer_apply: bad data pointers");
  GB_REQUIRE(!dtype_complex(dtype) || phase_cd, "gb_transformer_apply: complex data needs phase_cd");
  return tr_apply(t, in, out, nin, dtype, dtype_complex(dtype) ? phase_cd : nullptr,
                  (cudaStream_t)stream, 1.0, nullptr, 0.0);
}

int gb_transformer_apply_axpy(const gb_transformer* t, const void* in, void* out, int64_t nin, int dtype,
                              const double* phase_cd, double alpha, const void* y, double gamma, void* stream) {
  GB_REQUIRE(t, "gb_transformer_apply_axpy: null transformer");
  GB_REQUIRE(dtype_valid(dtype), "gb_transformer_apply_axpy: unknown dtype");
  GB_REQUIRE(nin >= 0, "gb_transformer_apply_axpy: negative batch");
  GB_REQUIRE(dtype_complex(dtype) == !t->real,
             "gb_transformer_apply_axpy: dtype does not match the transformer's real/complex flag");
  if (nin == 0) return GB_OK;
  GB_REQUIRE(in && out && in != out, "gb_transformer_apply_axpy: bad data pointers");
  GB_REQUIRE(t->interpolate || !y, "gb_transformer_apply_axpy: restriction has no y term");
  GB_REQUIRE(!dtype_complex(dtype) || phase_cd, "gb_transformer_apply_axpy: complex data needs phase_cd");
  return tr_apply(t, in, out, nin, dtype, dtype_complex(dtype) ? phase_cd : nullptr, (cudaStream_t)stream, alpha,
                  y, gamma);
}

int gb_transformer_free(gb_transformer* t) {
  delete t;
  return GB_OK;
}

int gb_transformer_apply_k(const gb_transformer* t, const void* in, void* out, int64_t nin, int dtype, int nk,
                           const double* phase_kcd, void* stream) {
  GB_REQUIRE(t && dtype_valid(dtype) && nin >= 0, "gb_transformer_apply_k: bad arguments");
  GB_REQUIRE(dtype_complex(dtype) == !t->real, "gb_transformer_apply_k: dtype does not match the transformer");
  GB_REQUIRE(nk >= 1 && nk <= KMAX && nin % nk == 0, "gb_transformer_apply_k: bad number of phase sets");
  if (nin == 0) return GB_OK;
  GB_REQUIRE(in && out && in != out, "gb_transformer_apply_k: bad data pointers");
  GB_REQUIRE(!dtype_complex(dtype) || phase_kcd, "gb_transformer_apply_k: complex data needs phases");
  return tr_apply(t, in, out, nin, dtype, dtype_complex(dtype) ? phase_kcd : nullptr, (cudaStream_t)stream, 1.0,
                  nullptr, 0.0, nk);
}

}  // extern "C"
