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
  int has_phase;
  double alpha, gamma;
  double ph[3][2][2];
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
                                            const TrArgs& a, int tid) {
  for (int e = tid; e < NR * NC; e += NT) {
    const int r = e / NC, c = e % NC;
    const int y = ry0 + r, z = cx0 + c;
    double pr = 1.0, pi = 0.0;
    bool w = false;
    if (a.pbc[1] && (y < 0 || y >= n1)) { const int s = y < 0; pr = a.ph[1][s][0]; pi = a.ph[1][s][1]; w = true; }
    if (a.pbc[2] && (z < 0 || z >= n2)) {
      const int s = z < 0;
      const double qr = a.ph[2][s][0], qi = a.ph[2][s][1];
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
      pr = a.ph[0][sd][0]; pi = a.ph[0][sd][1];
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
        if (CPLX && a.has_phase && edge) {
          phase_fixup<T, FR, PITCH, PITCH, NT>(P, ry0, cx0, nf1, nf2, a, tid);
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
      pr = a.ph[0][sd][0]; pi = a.ph[0][sd][1];
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
        if (CPLX && a.has_phase && edge) {
          phase_fixup<T, CR, PITCH, PITCH, NT>(P, ry0, cx0, nc1, nc2, a, tid);
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

static void fill_common(const gb_transformer* t, TrArgs& a, const double* ph) {
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
  for (int c = 0; c < 3; ++c)
    for (int d = 0; d < 2; ++d) {
      a.ph[c][d][0] = ph ? ph[(c * 2 + d) * 2] : 1.0;
      a.ph[c][d][1] = ph ? ph[(c * 2 + d) * 2 + 1] : 0.0;
      if (a.ph[c][d][0] != 1.0 || a.ph[c][d][1] != 0.0) a.has_phase = 1;
    }
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
  blocks = std::min<int64_t>(blocks, std::max<int64_t>(1, total / min_steps));
  kernel<<<(unsigned)blocks, C::NT, C::SMEM, st>>>(a);
  return check_launch("transformer kernel");
}

template <typename T, int K, int CY, int CZ>
static int restrict_cfg(const gb_transformer* t, const void* in, void* out, int64_t nin,
                        const double* ph, cudaStream_t st, double alpha) {
  using C = RCfg<T, K, CY, CZ, 2>;
  TrArgs a;
  fill_common(t, a, ph);
  a.in = in; a.out = out; a.nbatch = nin; a.alpha = alpha;
  a.tiles1 = ceil_div(a.no[1], C::CY);
  a.tiles2 = ceil_div(a.no[2], C::CZ);
  const int64_t total = nin * (int64_t)a.tiles1 * a.tiles2 * a.no[0];
  return launch_persistent<C>(restrict_kernel<C>, a, total, st, 4 + K);
}

// coarse rows of at most 16 points (the coarse levels of small grids) use a
// 16 x 16 tile, wider ones 8 x 32: no more than half a warp idles on a row
template <typename T, int K>
static int restrict_k(const gb_transformer* t, const void* in, void* out, int64_t nin,
                      const double* ph, cudaStream_t st, double alpha) {
  if (t->nout_c[2] <= 16) return restrict_cfg<T, K, 16, 16>(t, in, out, nin, ph, st, alpha);
  return restrict_cfg<T, K, 8, 32>(t, in, out, nin, ph, st, alpha);
}

template <typename T, int K>
static int interpolate_k(const gb_transformer* t, const void* in, void* out, int64_t nin,
                         const double* ph, cudaStream_t st, double alpha, const void* y, double gamma) {
  constexpr int RZ = sizeof(T) == 4 ? 4 : (sizeof(T) == 8 ? 2 : 1);
  using C = ICfg<T, K, 16, 32, 2, RZ, 2>;
  TrArgs a;
  fill_common(t, a, ph);
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
                       const double* ph, cudaStream_t st, double alpha, const void* y, double gamma) {
  if (t->interpolate) {
    switch (t->k) {
      case 2: return interpolate_k<T, 2>(t, in, out, nin, ph, st, alpha, y, gamma);
      case 4: return interpolate_k<T, 4>(t, in, out, nin, ph, st, alpha, y, gamma);
      case 6: return interpolate_k<T, 6>(t, in, out, nin, ph, st, alpha, y, gamma);
      default: return interpolate_k<T, 8>(t, in, out, nin, ph, st, alpha, y, gamma);
    }
  }
  if (y) return fail(GB_E_UNSUPPORTED, "restriction has no y epilogue");
  switch (t->k) {
    case 2: return restrict_k<T, 2>(t, in, out, nin, ph, st, alpha);
    case 4: return restrict_k<T, 4>(t, in, out, nin, ph, st, alpha);
    case 6: return restrict_k<T, 6>(t, in, out, nin, ph, st, alpha);
    default: return restrict_k<T, 8>(t, in, out, nin, ph, st, alpha);
  }
}

int tr_apply(const gb_transformer* t, const void* in, void* out, int64_t nin, int dtype,
             const double* ph, cudaStream_t st, double alpha, const void* y, double gamma) {
  switch (dtype) {
    case GB_DTYPE_F64: return tr_dispatch<double>(t, in, out, nin, ph, st, alpha, y, gamma);
    case GB_DTYPE_F32: return tr_dispatch<float>(t, in, out, nin, ph, st, alpha, y, gamma);
    case GB_DTYPE_C128: return tr_dispatch<double2>(t, in, out, nin, ph, st, alpha, y, gamma);
    default: return tr_dispatch<float2>(t, in, out, nin, ph, st, alpha, y, gamma);
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

}  // extern "C"
