// FD stencil operator (replaces _gpaw.Operator: c/operators.c, c/bmgs/fd.c,
// c/bc.c).  Two kernels:
//
//  * star_kernel  -- stencils whose points all lie on the three axes (the
//    reference's "cfd" case: Laplace on orthorhombic cells, Gradient).  A
//    persistent CTA owns a (T1 x T2) tile of the (axis1, axis2) plane of one
//    grid and marches along axis 0.  Planes (tile + halo) stream through a
//    ring of NS shared-memory slots filled by cp.async (LDGSTS, no register
//    staging, D planes in flight); every thread keeps a register queue of
//    2H+1 values of its own R1 x R2 points along axis 0, so each input
//    element is read from HBM once and from shared memory ~5-7 times.
//    Zero and periodic boundaries (with Bloch phases) are resolved while
//    filling the tile: out-of-range cells become zeros or wrapped copies,
//    wrapped copies of complex data are multiplied by the phase in a short
//    fix-up pass (only tiles that touch a periodic face pay it).
//
//  * box_kernel   -- any stencil (off-axis points of GUC Laplacians /
//    non-orthogonal gradients, c/bmgs/fd.c generic loop).  3-D tile with a
//    full halo cube in shared memory; correctness path.
//
// Boundary semantics follow c/bc.c:146-258: a halo cell beyond the upper end
// of a periodic axis c holds in[... m ...] * phase_cd[c][0], below the lower
// end in[... n-1-m ...] * phase_cd[c][1]; zero boundaries give zeros.

#include <vector>
#include <cmath>
#include <cstring>
#include <algorithm>
#include "internal.cuh"

namespace gb {


struct StarArgs {
  const void* in;
  void* out;
  int64_t nbatch;
  int n0, n1, n2;
  int pbc0, pbc1, pbc2;
  int tiles1, tiles2;
  double c0;
  double c0diff;              // c0 + sum of the neighbour coefficients (difference form)
  double a[3][2 * HMAX + 1];  // a[axis][m + HMAX]: coefficient of offset m (m != 0)
  PhaseSets phs;              // Bloch phases per k-point group of bands
  // epilogue: out = alpha * S(in) + beta * in + gamma * y   (y may be null)
  double alpha, beta, gamma;
  const void* y;
  const void* vpot;
};

template <typename T_, int H_, int R1_, int R2_, int TY_, int TZ_, int D_>
struct StarCfg {
  using T = T_;
  static constexpr int H = H_, R1 = R1_, R2 = R2_, TY = TY_, TZ = TZ_, D = D_;
  static constexpr int VEC = 16 / (int)sizeof(T);
  static constexpr int HZ = ((H + VEC - 1) / VEC) * VEC;
  static constexpr int T1 = TY * R1, T2 = TZ * R2;
  static constexpr int W = T2 + 2 * HZ;
  static constexpr int ROWS = T1 + 2 * H;
  static constexpr int PLANE = ROWS * W;
  static constexpr int NS = H + D;
  static constexpr int NT = TY * TZ;
  static constexpr int KH = T2 / VEC;       // chunks in a halo row
  static constexpr int KC = W / VEC;        // chunks in a centre row
  static constexpr int NCHUNK = 2 * H * KH + T1 * KC;
  static constexpr size_t SMEM = (size_t)NS * PLANE * sizeof(T);
  static_assert(R2 % VEC == 0, "R2 must be a multiple of the 16-byte vector");
  static_assert((W * sizeof(T)) % 16 == 0, "row pitch must keep 16-byte alignment");
};

// true modulo: partial tiles of small grids can reach several periods away
// (those cells feed no valid output, but their loads must stay in bounds)
__device__ __forceinline__ int wrap_index(int i, int n) {
  int r = i % n;
  return r < 0 ? r + n : r;
}

template <class C>
__global__ void __launch_bounds__(C::NT, 2) star_kernel(const StarArgs args) {
  using T = typename C::T;
  using R = typename Elem<T>::R;
  constexpr int H = C::H, R1 = C::R1, R2 = C::R2, TZ = C::TZ, VEC = C::VEC, HZ = C::HZ;
  constexpr int T1 = C::T1, T2 = C::T2, W = C::W, PLANE = C::PLANE, NS = C::NS, D = C::D;
  constexpr bool CPLX = Elem<T>::cplx;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* planes = reinterpret_cast<T*>(smem_raw);

  const int tid = threadIdx.x;
  const int ty = tid / TZ, tz = tid % TZ;
  const int n0 = args.n0, n1 = args.n1, n2 = args.n2;
  const int64_t n12 = (int64_t)n1 * n2;
  const int64_t n012 = n12 * n0;
  const int64_t ntiles = (int64_t)args.tiles1 * args.tiles2;
  const int64_t total = args.nbatch * ntiles * n0;
  int64_t s = total * blockIdx.x / gridDim.x;
  const int64_t s_end = total * (blockIdx.x + 1) / gridDim.x;

  const bool epi = args.alpha != 1.0 || args.beta != 0.0 || args.y != nullptr || args.vpot != nullptr;
  const R* __restrict__ vpot = reinterpret_cast<const R*>(args.vpot);
  const R ealpha = (R)args.alpha, ebeta = (R)args.beta, egamma = (R)args.gamma;
  // FP32: the difference form sum_p c_p (x_p - x_c) + (sum c) x_c keeps the
  // operator exactly constant-annihilating after the coefficients are rounded
  constexpr bool DIFF = sizeof(R) == 4;
  R c0 = DIFF ? (R)args.c0diff : (R)args.c0;
  R a0[2 * H + 1], a1[2 * H + 1], a2[2 * H + 1];
#pragma unroll
  for (int m = 0; m <= 2 * H; ++m) {
    a0[m] = (R)args.a[0][m - H + HMAX];
    a1[m] = (R)args.a[1][m - H + HMAX];
    a2[m] = (R)args.a[2][m - H + HMAX];
  }

  while (s < s_end) {
    const int64_t col = s / n0;
    const int p_start = (int)(s % n0);
    const int p_end = (int)(s_end - s < (int64_t)(n0 - p_start) ? p_start + (s_end - s) : n0);
    s += p_end - p_start;
    const int64_t band = col / ntiles;
    const int t = (int)(col % ntiles);
    const int y0 = (t / args.tiles2) * T1;
    const int z0 = (t % args.tiles2) * T2;
    const T* __restrict__ src = reinterpret_cast<const T*>(args.in) + band * n012;
    T* __restrict__ dst = reinterpret_cast<T*>(args.out) + band * n012;
    const T* __restrict__ ybase = args.y ? reinterpret_cast<const T*>(args.y) + band * n012 : nullptr;
    const auto& PH = args.phs.ph[phase_set_of(args.phs, band)];
    const bool edge = (y0 - H < 0) || (y0 + T1 + H > n1) || (z0 - HZ < 0) || (z0 + T2 + HZ > n2);

    const int j0 = p_start - H, j1 = p_end + H;   // planes pushed: [j0, j1)

    // plane j -> source plane (or -1 for an all-zero plane) and its phase
    auto plane_src = [&](int j, double& pr, double& pi) -> int {
      pr = 1.0; pi = 0.0;
      if (j >= 0 && j < n0) return j;
      if (!args.pbc0) return -1;
      const int side = j < 0 ? 1 : 0;
      pr = PH[0][side][0]; pi = PH[0][side][1];
      return wrap_index(j, n0);
    };

    auto issue = [&](int j) {
      double pr, pi;
      const int sp = plane_src(j, pr, pi);
      if (sp < 0) return;
      T* P = planes + ((j - j0) % NS) * PLANE;
      const T* S = src + (int64_t)sp * n12;
      for (int e = tid; e < C::NCHUNK; e += C::NT) {
        int Rw, k;
        if (e < 2 * H * C::KH) {
          const int hr = e / C::KH;
          Rw = hr < H ? hr : hr + T1;
          k = HZ / VEC + e % C::KH;
        } else {
          const int e2 = e - 2 * H * C::KH;
          Rw = H + e2 / C::KC;
          k = e2 % C::KC;
        }
        T* sd = P + Rw * W + k * VEC;
        int y = y0 - H + Rw;
        if (y < 0 || y >= n1) {
          if (!args.pbc1) {
#pragma unroll
            for (int v = 0; v < VEC; ++v) sd[v] = zero<T>();
            continue;
          }
          y = wrap_index(y, n1);
        }
        const T* row = S + (int64_t)y * n2;
        const int zs = z0 - HZ + k * VEC;
        if (zs >= 0 && zs + VEC <= n2 && ((reinterpret_cast<uintptr_t>(row + zs) & 15) == 0)) {
          cp_async16(sd, row + zs);
        } else {
#pragma unroll
          for (int v = 0; v < VEC; ++v) {
            int z = zs + v;
            if (z < 0 || z >= n2) {
              if (!args.pbc2) { sd[v] = zero<T>(); continue; }
              z = wrap_index(z, n2);
            }
            cp_async_elem(sd + v, row + z);
          }
        }
      }
    };

    // Bloch phase of wrapped in-plane cells (complex data only)
    auto fixup = [&](T* P) {
      for (int e = tid; e < C::NCHUNK * VEC; e += C::NT) {
        const int ec = e / VEC, v = e % VEC;
        int Rw, k;
        if (ec < 2 * H * C::KH) {
          const int hr = ec / C::KH;
          Rw = hr < H ? hr : hr + T1;
          k = HZ / VEC + ec % C::KH;
        } else {
          const int e2 = ec - 2 * H * C::KH;
          Rw = H + e2 / C::KC;
          k = e2 % C::KC;
        }
        const int y = y0 - H + Rw, z = z0 - HZ + k * VEC + v;
        double pr = 1.0, pi = 0.0;
        bool w = false;
        if (args.pbc1 && (y < 0 || y >= n1)) { const int sd = y < 0; pr = PH[1][sd][0]; pi = PH[1][sd][1]; w = true; }
        if (args.pbc2 && (z < 0 || z >= n2)) {
          const int sd = z < 0;
          const double qr = PH[2][sd][0], qi = PH[2][sd][1];
          const double tr = pr * qr - pi * qi, ti = pr * qi + pi * qr;
          pr = tr; pi = ti; w = true;
        }
        if (w) { T* c = P + Rw * W + k * VEC + v; *c = phase_mul(*c, pr, pi); }
      }
    };

    T q[2 * H + 1][R1][R2];
#pragma unroll
    for (int m = 0; m <= 2 * H; ++m)
#pragma unroll
      for (int r = 0; r < R1; ++r)
#pragma unroll
        for (int c = 0; c < R2; ++c) q[m][r][c] = zero<T>();

#pragma unroll
    for (int d = 0; d < D; ++d) {
      if (j0 + d < j1) issue(j0 + d);
      cp_async_commit();
    }

    for (int j = j0; j < j1; ++j) {
      cp_async_wait<D - 1>();
      __syncthreads();
      double pr, pi;
      const int sp = plane_src(j, pr, pi);
      T* P = planes + ((j - j0) % NS) * PLANE;
      if (CPLX && args.phs.any && edge && sp >= 0) {
        fixup(P);
        __syncthreads();
      }
      // push own values of plane j into the axis-0 queue
#pragma unroll
      for (int m = 0; m < 2 * H; ++m)
#pragma unroll
        for (int r = 0; r < R1; ++r)
#pragma unroll
          for (int c = 0; c < R2; ++c) q[m][r][c] = q[m + 1][r][c];
      if (sp >= 0) {
#pragma unroll
        for (int r = 0; r < R1; ++r) {
          T v[R2];
          lds_vec<T, R2>(P + (H + ty * R1 + r) * W + HZ + tz * R2, v);
#pragma unroll
          for (int c = 0; c < R2; ++c) q[2 * H][r][c] = CPLX ? phase_mul(v[c], pr, pi) : v[c];
        }
      } else {
#pragma unroll
        for (int r = 0; r < R1; ++r)
#pragma unroll
          for (int c = 0; c < R2; ++c) q[2 * H][r][c] = zero<T>();
      }

      const int cpl = j - H;   // centre plane computed this iteration
      if (cpl >= p_start) {
        const T* Pc = planes + ((cpl - j0) % NS) * PLANE;
        T acc[R1][R2];
        // axis 0 (register queue) and axis 2 (row windows)
#pragma unroll
        for (int r = 0; r < R1; ++r) {
          const T* rowp = Pc + (H + ty * R1 + r) * W + tz * R2;
          T wl[HZ], wr[HZ];
          lds_vec<T, HZ>(rowp, wl);
          lds_vec<T, HZ>(rowp + HZ + R2, wr);
#pragma unroll
          for (int c = 0; c < R2; ++c) {
            T x = scale(c0, q[H][r][c]);
#pragma unroll
            for (int m = 0; m <= 2 * H; ++m)
              if (m != H) x = fmadd(x, a0[m], DIFF ? sub(q[m][r][c], q[H][r][c]) : q[m][r][c]);
#pragma unroll
            for (int m = 0; m <= 2 * H; ++m) {
              if (m == H) continue;
              const int cc = c + m - H;
              T v;
              if (cc < 0) v = wl[HZ + cc];
              else if (cc >= R2) v = wr[cc - R2];
              else v = q[H][r][cc];
              x = fmadd(x, a2[m], DIFF ? sub(v, q[H][r][c]) : v);
            }
            acc[r][c] = x;
          }
        }
        // axis 1: rows of the own block come from the queue, others from smem
#pragma unroll
        for (int rr = -H; rr < R1 + H; ++rr) {
          T v[R2];
          if (rr >= 0 && rr < R1) {
#pragma unroll
            for (int c = 0; c < R2; ++c) v[c] = q[H][rr][c];
          } else {
            lds_vec<T, R2>(Pc + (H + ty * R1 + rr) * W + HZ + tz * R2, v);
          }
#pragma unroll
          for (int r = 0; r < R1; ++r) {
            const int m = rr - r + H;
            if (m < 0 || m > 2 * H || m == H) continue;
#pragma unroll
            for (int c = 0; c < R2; ++c)
              acc[r][c] = fmadd(acc[r][c], a1[m], DIFF ? sub(v[c], q[H][r][c]) : v[c]);
          }
        }
        // epilogue (fused axpy passes of the multigrid V-cycle)
        if (epi) {
          const T* yp = ybase ? ybase + (int64_t)cpl * n12 : nullptr;
#pragma unroll
          for (int r = 0; r < R1; ++r) {
            const int y = y0 + ty * R1 + r;
#pragma unroll
            for (int c = 0; c < R2; ++c) {
              const int z = z0 + tz * R2 + c;
              T v = fmadd(scale(ealpha, acc[r][c]), ebeta, q[H][r][c]);
              if (yp && y < n1 && z < n2) v = fmadd(v, egamma, yp[(int64_t)y * n2 + z]);
              if (vpot && y < n1 && z < n2) v = fmadd(v, vpot[(int64_t)cpl * n12 + (int64_t)y * n2 + z], q[H][r][c]);
              acc[r][c] = v;
            }
          }
        }
        // store
        T* outp = dst + (int64_t)cpl * n12;
#pragma unroll
        for (int r = 0; r < R1; ++r) {
          const int y = y0 + ty * R1 + r;
          if (y >= n1) continue;
          T* o = outp + (int64_t)y * n2;
          const int z = z0 + tz * R2;
          if (z + R2 <= n2 && ((reinterpret_cast<uintptr_t>(o + z) & 15) == 0)) {
#pragma unroll
            for (int c = 0; c < R2; c += VEC) {
              float4 w4;
              T* e = reinterpret_cast<T*>(&w4);
#pragma unroll
              for (int k = 0; k < VEC; ++k) e[k] = acc[r][c + k];
              __stcs(reinterpret_cast<float4*>(o + z + c), w4);
            }
          } else {
#pragma unroll
            for (int c = 0; c < R2; ++c)
              if (z + c < n2) st_cs(o + z + c, acc[r][c]);
          }
        }
      }
      __syncthreads();
      if (j + D < j1) issue(j + D);
      cp_async_commit();
    }
    cp_async_wait<0>();
    __syncthreads();
  }
}

// --------------------------------------------------------------------------
// Generic stencil: arbitrary offsets within a cube of radius M (<= 6).
struct BoxArgs {
  const void* in;
  void* out;
  int64_t nbatch;
  int n0, n1, n2;
  int pbc0, pbc1, pbc2;
  int M;                  // halo radius
  int np;
  int b0, b1, b2;         // tile extents
  int tiles0, tiles1, tiles2;
  double coef[64];
  int off[64][3];
  PhaseSets phs;
  double alpha, beta, gamma;
  const void* y;
  const void* vpot;
  double csum;   // sum of all coefficients (difference form in FP32)
};

template <typename T>
__global__ void __launch_bounds__(256) box_kernel(const BoxArgs args) {
  using R = typename Elem<T>::R;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* tile = reinterpret_cast<T*>(smem_raw);
  const int M = args.M;
  const int E0 = args.b0 + 2 * M, E1 = args.b1 + 2 * M, E2 = args.b2 + 2 * M;
  const int64_t ntile = (int64_t)args.tiles0 * args.tiles1 * args.tiles2;
  const int64_t n12 = (int64_t)args.n1 * args.n2, n012 = n12 * args.n0;
  for (int64_t w = blockIdx.x; w < args.nbatch * ntile; w += gridDim.x) {
    const int64_t band = w / ntile;
    int t = (int)(w % ntile);
    const int x0 = (t / (args.tiles1 * args.tiles2)) * args.b0;
    t %= args.tiles1 * args.tiles2;
    const int y0 = (t / args.tiles2) * args.b1;
    const int z0 = (t % args.tiles2) * args.b2;
    const T* src = reinterpret_cast<const T*>(args.in) + band * n012;
    T* dst = reinterpret_cast<T*>(args.out) + band * n012;
    const auto& PH = args.phs.ph[phase_set_of(args.phs, band)];
    __syncthreads();
    for (int e = threadIdx.x; e < E0 * E1 * E2; e += blockDim.x) {
      const int i2 = e % E2, i1 = (e / E2) % E1, i0 = e / (E1 * E2);
      int g[3] = {x0 - M + i0, y0 - M + i1, z0 - M + i2};
      const int n[3] = {args.n0, args.n1, args.n2};
      const int pbc[3] = {args.pbc0, args.pbc1, args.pbc2};
      double pr = 1.0, pi = 0.0;
      bool zero_cell = false;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if (g[c] < 0 || g[c] >= n[c]) {
          if (!pbc[c]) { zero_cell = true; break; }
          const int sd = g[c] < 0;
          const double qr = PH[c][sd][0], qi = PH[c][sd][1];
          const double tr = pr * qr - pi * qi, ti = pr * qi + pi * qr;
          pr = tr; pi = ti;
          g[c] = wrap_index(g[c], n[c]);
        }
      }
      T v = zero<T>();
      if (!zero_cell) {
        v = src[(int64_t)g[0] * n12 + (int64_t)g[1] * args.n2 + g[2]];
        if (args.phs.any) v = phase_mul(v, pr, pi);
      }
      tile[e] = v;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < args.b0 * args.b1 * args.b2; e += blockDim.x) {
      const int i2 = e % args.b2, i1 = (e / args.b2) % args.b1, i0 = e / (args.b1 * args.b2);
      const int gx = x0 + i0, gy = y0 + i1, gz = z0 + i2;
      if (gx >= args.n0 || gy >= args.n1 || gz >= args.n2) continue;
      constexpr bool DIFF = sizeof(R) == 4;
      const T xc0 = tile[((i0 + M) * E1 + (i1 + M)) * E2 + (i2 + M)];
      T x = DIFF ? scale((R)args.csum, xc0) : zero<T>();
      for (int p = 0; p < args.np; ++p) {
        const int j = ((i0 + M + args.off[p][0]) * E1 + (i1 + M + args.off[p][1])) * E2 + (i2 + M + args.off[p][2]);
        x = fmadd(x, (R)args.coef[p], DIFF ? sub(tile[j], xc0) : tile[j]);
      }
      const int64_t gidx = (int64_t)gx * n12 + (int64_t)gy * args.n2 + gz;
      if (args.alpha != 1.0 || args.beta != 0.0 || args.y || args.vpot) {
        const T xc = tile[((i0 + M) * E1 + (i1 + M)) * E2 + (i2 + M)];
        x = fmadd(scale((R)args.alpha, x), (R)args.beta, xc);
        if (args.y) x = fmadd(x, (R)args.gamma, reinterpret_cast<const T*>(args.y)[band * n012 + gidx]);
        if (args.vpot) x = fmadd(x, reinterpret_cast<const R*>(args.vpot)[gidx], xc);
      }
      dst[gidx] = x;
    }
  }
}

// --------------------------------------------------------------------------
// Jacobi relaxation (relax_method 2 of c/bmgs/relax.c:40-66) for real FP64:
//   f <- (1-w) f + w (s - sum_{p != 0} c_p f[. + o_p]) / c_0
// One sweep per launch; the halo is resolved like box_kernel.
__global__ void jacobi_kernel(const BoxArgs args, const double* f_in, double* f_out,
                              const double* s, double w, double c_center) {
  const int64_t n12 = (int64_t)args.n1 * args.n2, N = n12 * args.n0;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < N; g += (int64_t)gridDim.x * blockDim.x) {
    const int i0 = (int)(g / n12), i1 = (int)((g / args.n2) % args.n1), i2 = (int)(g % args.n2);
    double x = 0.0;
    for (int p = 0; p < args.np; ++p) {
      if (args.off[p][0] == 0 && args.off[p][1] == 0 && args.off[p][2] == 0) continue;
      int c3[3] = {i0 + args.off[p][0], i1 + args.off[p][1], i2 + args.off[p][2]};
      const int n[3] = {args.n0, args.n1, args.n2};
      const int pbc[3] = {args.pbc0, args.pbc1, args.pbc2};
      bool z = false;
      for (int c = 0; c < 3; ++c)
        if (c3[c] < 0 || c3[c] >= n[c]) {
          if (!pbc[c]) { z = true; break; }
          c3[c] = wrap_index(c3[c], n[c]);
        }
      if (!z) x += args.coef[p] * f_in[(int64_t)c3[0] * n12 + (int64_t)c3[1] * args.n2 + c3[2]];
    }
    f_out[g] = (1.0 - w) * f_in[g] + w * (s[g] - x) / c_center;
  }
}

}  // namespace gb

namespace gb {


template <class C>
static int launch_star(const gb_operator* op, const void* in, void* out, int64_t nin,
                       const double* phase_cd, cudaStream_t stream, const Epilogue& ep, int nk) {
  static int occ = -1;
  static size_t smem_set = 0;
  if (smem_set != C::SMEM) {
    cudaFuncSetAttribute(star_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
    smem_set = C::SMEM;
  }
  if (occ < 0) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, star_kernel<C>, C::NT, C::SMEM);
    if (occ < 1) occ = 1;
  }
  StarArgs a{};
  a.in = in; a.out = out; a.nbatch = nin;
  a.n0 = (int)op->n[0]; a.n1 = (int)op->n[1]; a.n2 = (int)op->n[2];
  a.pbc0 = op->pbc[0]; a.pbc1 = op->pbc[1]; a.pbc2 = op->pbc[2];
  a.tiles1 = ceil_div(a.n1, C::T1);
  a.tiles2 = ceil_div(a.n2, C::T2);
  a.c0 = op->center;
  a.c0diff = op->center;
  for (int c = 0; c < 3; ++c)
    for (int m = 0; m < 2 * HMAX + 1; ++m) a.c0diff += op->a[c][m];
  memcpy(a.a, op->a, sizeof(a.a));
  a.alpha = ep.alpha; a.beta = ep.beta; a.gamma = ep.gamma; a.y = ep.y; a.vpot = ep.vpot;
  fill_phase_sets(a.phs, phase_cd, nk, nin);
  const int64_t total = nin * (int64_t)a.tiles1 * a.tiles2 * a.n0;
  int64_t blocks = (int64_t)sm_count() * occ;
  // keep at least a few planes per CTA so the prologue (2H planes) stays small
  blocks = std::min<int64_t>(blocks, std::max<int64_t>(1, total / (4 * C::H + 4)));
  star_kernel<C><<<(unsigned)blocks, C::NT, C::SMEM, stream>>>(a);
  return check_launch("star_kernel");
}

// Small real grids (the coarsest multigrid level, 14^3 for a 56^3 grid):
// the tiles of star_kernel would leave most threads idle and march a few
// planes per CTA through its staging pipeline, so one thread per point reads
// its 6H neighbours straight from global memory (the grid stays in L1/L2).
// Same terms in the same order as star_kernel (axis 0, axis 2, axis 1, m
// ascending; the FP32 difference form), so both give identical results.
template <typename T, int H>
__global__ void __launch_bounds__(256) star_direct_kernel(const StarArgs args) {
  constexpr bool DIFF = sizeof(T) == 4;
  const int n0 = args.n0, n1 = args.n1, n2 = args.n2;
  const int64_t n12 = (int64_t)n1 * n2, n012 = n12 * n0;
  const int64_t total = args.nbatch * n012;
  const bool epi = args.alpha != 1.0 || args.beta != 0.0 || args.y != nullptr || args.vpot != nullptr;
  const T* __restrict__ vpot = reinterpret_cast<const T*>(args.vpot);
  const T c0 = DIFF ? (T)args.c0diff : (T)args.c0;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t band = e / n012;
    const int64_t g = e - band * n012;
    const int i0 = (int)(g / n12);
    const int i1 = (int)((g - (int64_t)i0 * n12) / n2);
    const int i2 = (int)(g - (int64_t)i0 * n12 - (int64_t)i1 * n2);
    const T* __restrict__ src = reinterpret_cast<const T*>(args.in) + band * n012;
    const T xc = src[g];
    T x = scale(c0, xc);
    // axis 0
#pragma unroll
    for (int m = 0; m <= 2 * H; ++m) {
      if (m == H) continue;
      int j = i0 + m - H;
      T v = (T)0;
      if (j >= 0 && j < n0) v = src[g + (int64_t)(m - H) * n12];
      else if (args.pbc0) v = src[(int64_t)wrap_index(j, n0) * n12 + (g - (int64_t)i0 * n12)];
      x = fmadd(x, (T)args.a[0][m - H + HMAX], DIFF ? v - xc : v);
    }
    // axis 2
#pragma unroll
    for (int m = 0; m <= 2 * H; ++m) {
      if (m == H) continue;
      int j = i2 + m - H;
      T v = (T)0;
      if (j >= 0 && j < n2) v = src[g + (m - H)];
      else if (args.pbc2) v = src[g - i2 + wrap_index(j, n2)];
      x = fmadd(x, (T)args.a[2][m - H + HMAX], DIFF ? v - xc : v);
    }
    // axis 1
#pragma unroll
    for (int m = 0; m <= 2 * H; ++m) {
      if (m == H) continue;
      int j = i1 + m - H;
      T v = (T)0;
      if (j >= 0 && j < n1) v = src[g + (int64_t)(m - H) * n2];
      else if (args.pbc1) v = src[g + (int64_t)(wrap_index(j, n1) - i1) * n2];
      x = fmadd(x, (T)args.a[1][m - H + HMAX], DIFF ? v - xc : v);
    }
    if (epi) {
      T v = fmadd(scale((T)args.alpha, x), (T)args.beta, xc);
      if (args.y) v = fmadd(v, (T)args.gamma, reinterpret_cast<const T*>(args.y)[e]);
      if (vpot) v = fmadd(v, vpot[g], xc);
      x = v;
    }
    reinterpret_cast<T*>(args.out)[e] = x;
  }
}

template <typename T, int H>
static int launch_star_direct(const gb_operator* op, const void* in, void* out, int64_t nin,
                              cudaStream_t stream, const Epilogue& ep) {
  StarArgs a{};
  a.in = in; a.out = out; a.nbatch = nin;
  a.n0 = (int)op->n[0]; a.n1 = (int)op->n[1]; a.n2 = (int)op->n[2];
  a.pbc0 = op->pbc[0]; a.pbc1 = op->pbc[1]; a.pbc2 = op->pbc[2];
  a.c0 = op->center;
  a.c0diff = op->center;
  for (int c = 0; c < 3; ++c)
    for (int m = 0; m < 2 * HMAX + 1; ++m) a.c0diff += op->a[c][m];
  memcpy(a.a, op->a, sizeof(a.a));
  a.alpha = ep.alpha; a.beta = ep.beta; a.gamma = ep.gamma; a.y = ep.y; a.vpot = ep.vpot;
  const int64_t total = nin * op->n[0] * op->n[1] * op->n[2];
  const int64_t blocks = std::min<int64_t>((total + 255) / 256, (int64_t)sm_count() * 8);
  star_direct_kernel<T, H><<<(unsigned)std::max<int64_t>(blocks, 1), 256, 0, stream>>>(a);
  return check_launch("star_direct_kernel");
}

// Per-element-size tile shapes.  (R1 x R2) points per thread, (TY x TZ)
// threads; R2 * sizeof(T) = 16 bytes so row windows are single LDS.128s and a
// warp's 16 lanes along axis 2 read 256 contiguous bytes (no bank conflicts).
template <typename T, int H>
struct StarTile;
template <int H> struct StarTile<float, H>   { using C = StarCfg<float, H, (H <= 3 ? 4 : 2), 4, 8, 8, 2>; };
template <int H> struct StarTile<double, H>  { using C = StarCfg<double, H, (H <= 3 ? 4 : 2), 2, 8, 16, 2>; };
template <int H> struct StarTile<float2, H>  { using C = StarCfg<float2, H, (H <= 3 ? 4 : 2), 2, 8, 16, 2>; };
template <int H> struct StarTile<double2, H> { using C = StarCfg<double2, H, (H <= 3 ? 4 : 2), 1, 8, 16, 2>; };

template <typename T>
static int dispatch_star(const gb_operator* op, const void* in, void* out, int64_t nin,
                         const double* ph, cudaStream_t st, const Epilogue& ep, int nk) {
  if constexpr (!Elem<T>::cplx) {
    // tiles of star_kernel less than a quarter used: one thread per point
    using C1 = typename StarTile<T, 1>::C;
    const int64_t n1 = op->n[1], n2 = op->n[2];
    const int64_t tiled = (int64_t)ceil_div((int)n1, C1::T1) * C1::T1 * ceil_div((int)n2, C1::T2) * C1::T2;
    if (op->H <= 3 && 4 * n1 * n2 < tiled) {
      switch (op->H) {
        case 1: return launch_star_direct<T, 1>(op, in, out, nin, st, ep);
        case 2: return launch_star_direct<T, 2>(op, in, out, nin, st, ep);
        default: return launch_star_direct<T, 3>(op, in, out, nin, st, ep);
      }
    }
  }
  switch (op->H) {
    case 1: return launch_star<typename StarTile<T, 1>::C>(op, in, out, nin, ph, st, ep, nk);
    case 2: return launch_star<typename StarTile<T, 2>::C>(op, in, out, nin, ph, st, ep, nk);
    case 3: return launch_star<typename StarTile<T, 3>::C>(op, in, out, nin, ph, st, ep, nk);
    case 4: return launch_star<typename StarTile<T, 4>::C>(op, in, out, nin, ph, st, ep, nk);
    case 5:
    case 6: return launch_star<typename StarTile<T, 6>::C>(op, in, out, nin, ph, st, ep, nk);
    default: return fail(GB_E_UNSUPPORTED, "star stencil radius > 6");
  }
}

static void fill_box_args(const gb_operator* op, BoxArgs& a, const double* phase_cd, int nk = 1,
                          int64_t nbatch = 1) {
  memset(&a, 0, sizeof(a));
  a.alpha = 1.0;
  a.n0 = (int)op->n[0]; a.n1 = (int)op->n[1]; a.n2 = (int)op->n[2];
  a.pbc0 = op->pbc[0]; a.pbc1 = op->pbc[1]; a.pbc2 = op->pbc[2];
  a.M = op->range;
  a.np = op->np;
  a.csum = 0.0;
  for (int p = 0; p < op->np; ++p) {
    a.coef[p] = op->coef[p];
    a.csum += op->coef[p];
    for (int c = 0; c < 3; ++c) a.off[p][c] = op->off[p * 3 + c];
  }
  fill_phase_sets(a.phs, phase_cd, nk, nbatch);
}

template <typename T>
static int launch_box(const gb_operator* op, const void* in, void* out, int64_t nin,
                      const double* phase_cd, cudaStream_t stream, const Epilogue& ep, int nk) {
  BoxArgs a;
  fill_box_args(op, a, phase_cd, nk, nin);
  a.alpha = ep.alpha; a.beta = ep.beta; a.gamma = ep.gamma; a.y = ep.y;
  a.in = in; a.out = out; a.nbatch = nin;
  a.b0 = 4; a.b1 = 8; a.b2 = 32;
  const int M = a.M;
  size_t smem = (size_t)(a.b0 + 2 * M) * (a.b1 + 2 * M) * (a.b2 + 2 * M) * sizeof(T);
  while (smem > 200 * 1024 && a.b2 > 8) {
    a.b2 /= 2;
    smem = (size_t)(a.b0 + 2 * M) * (a.b1 + 2 * M) * (a.b2 + 2 * M) * sizeof(T);
  }
  a.tiles0 = ceil_div(a.n0, a.b0); a.tiles1 = ceil_div(a.n1, a.b1); a.tiles2 = ceil_div(a.n2, a.b2);
  cudaFuncSetAttribute(box_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int64_t work = nin * (int64_t)a.tiles0 * a.tiles1 * a.tiles2;
  const int64_t blocks = std::min<int64_t>(work, (int64_t)sm_count() * 8);
  box_kernel<T><<<(unsigned)std::max<int64_t>(blocks, 1), 256, smem, stream>>>(a);
  return check_launch("box_kernel");
}

// internal entry used by gb_operator_apply and the preconditioner chain
int op_apply(const gb_operator* op, const void* in, void* out, int64_t nin, int dtype,
             const double* ph, cudaStream_t st, const Epilogue& ep, int nk) {
  if (nk > KMAX) return fail(GB_E_UNSUPPORTED, "more k-point phase sets than one launch takes");
  if (nk > 1 && nin % nk) return fail(GB_E_INVALID, "batch not divisible by the number of phase sets");
  if (op->cfd) {
    const int rc = star_tma_apply(op, in, out, nin, dtype, ph, st, ep, nk);
    if (rc != 1) return rc;
    if (stencil_path() == 2)
      return fail(GB_E_UNSUPPORTED, std::string("TMA stencil path required but not applicable: ") + tma_reason());
    switch (dtype) {
      case GB_DTYPE_F64: return dispatch_star<double>(op, in, out, nin, ph, st, ep, nk);
      case GB_DTYPE_F32: return dispatch_star<float>(op, in, out, nin, ph, st, ep, nk);
      case GB_DTYPE_C128: return dispatch_star<double2>(op, in, out, nin, ph, st, ep, nk);
      default: return dispatch_star<float2>(op, in, out, nin, ph, st, ep, nk);
    }
  }
  switch (dtype) {
    case GB_DTYPE_F64: return launch_box<double>(op, in, out, nin, ph, st, ep, nk);
    case GB_DTYPE_F32: return launch_box<float>(op, in, out, nin, ph, st, ep, nk);
    case GB_DTYPE_C128: return launch_box<double2>(op, in, out, nin, ph, st, ep, nk);
    default: return launch_box<float2>(op, in, out, nin, ph, st, ep, nk);
  }
}

}  // namespace gb

using namespace gb;

extern "C" {

int gb_operator_new(const double* coef_p, const int64_t* offset_p, int np,
                    const int64_t size_c[3], int range, const int64_t neighbor_cd[6],
                    int real, int cfd, gb_operator** out) {
  GB_REQUIRE(out && coef_p && offset_p && size_c && neighbor_cd, "gb_operator_new: null pointer");
  GB_REQUIRE(np > 0 && np <= 64, "gb_operator_new: 1 <= np <= 64 stencil points required");
  GB_REQUIRE(range >= 0 && range <= 6, "gb_operator_new: stencil range must be in [0, 6]");
  for (int c = 0; c < 3; ++c) {
    GB_REQUIRE(size_c[c] > 0 && size_c[c] < (1 << 30), "gb_operator_new: bad grid size");
    // the reference asserts the same ("Stencil longer than domain",
    // gpaw/fd_operators.py:53)
    GB_REQUIRE(range <= size_c[c], "gb_operator_new: stencil longer than domain");
  }
  auto* op = new (std::nothrow) gb_operator();
  if (!op) return fail(GB_E_NOMEM, "gb_operator_new: out of host memory");
  op->np = np;
  op->range = range;
  op->real = real;
  for (int c = 0; c < 3; ++c) {
    op->n[c] = size_c[c];
    // single domain: a neighbour >= 0 on an axis means periodic wrap
    op->pbc[c] = (neighbor_cd[2 * c] >= 0 || neighbor_cd[2 * c + 1] >= 0) ? 1 : 0;
  }
  const int64_t M1 = size_c[1] + 2 * range, M2 = size_c[2] + 2 * range;
  op->coef.assign(coef_p, coef_p + np);
  op->off.resize(np * 3);
  bool on_axes = true;
  int H = 0;
  op->diag = 0.0;
  for (int p = 0; p < np; ++p) {
    // decode the linear padded-array offset o0*M1*M2 + o1*M2 + o2, |o_c| <= range
    int64_t o = offset_p[p];
    int64_t o0 = (o >= 0 ? o + (M1 * M2) / 2 : o - (M1 * M2) / 2) / (M1 * M2);
    int64_t r = o - o0 * M1 * M2;
    int64_t o1 = (r >= 0 ? r + M2 / 2 : r - M2 / 2) / M2;
    int64_t o2 = r - o1 * M2;
    if (std::llabs(o0) > range || std::llabs(o1) > range || std::llabs(o2) > range) {
      delete op;
      return fail(GB_E_INVALID, "gb_operator_new: offset outside the padded range");
    }
    op->off[p * 3 + 0] = (int)o0;
    op->off[p * 3 + 1] = (int)o1;
    op->off[p * 3 + 2] = (int)o2;
    const int nz = (o0 != 0) + (o1 != 0) + (o2 != 0);
    if (nz >= 2) on_axes = false;
    H = std::max<int>(H, (int)std::max({std::llabs(o0), std::llabs(o1), std::llabs(o2)}));
    if (o == 0) op->diag = coef_p[p];   // last zero-offset coefficient wins, as in c/operators.c:332-334
  }
  op->cfd = on_axes ? 1 : 0;
  (void)cfd;
  op->H = H;
  op->center = 0.0;
  memset(op->a, 0, sizeof(op->a));
  for (int p = 0; p < np; ++p) {
    const int* o = &op->off[p * 3];
    if (o[0] == 0 && o[1] == 0 && o[2] == 0) { op->center += coef_p[p]; continue; }
    for (int c = 0; c < 3; ++c)
      if (o[c] != 0) op->a[c][o[c] + HMAX] += coef_p[p];
  }
  if (op->H == 0) op->H = 1;
  *out = op;
  return GB_OK;
}

int gb_operator_apply(const gb_operator* op, const void* in, void* out, int64_t nin, int dtype,
                      const double* phase_cd, void* stream) {
  GB_REQUIRE(op, "gb_operator_apply: null operator");
  GB_REQUIRE(dtype_valid(dtype), "gb_operator_apply: unknown dtype");
  GB_REQUIRE(nin >= 0, "gb_operator_apply: negative batch");
  GB_REQUIRE(dtype_complex(dtype) == !op->real,
             "gb_operator_apply: dtype does not match the operator's real/complex flag");
  if (nin == 0) return GB_OK;
  GB_REQUIRE(in && out, "gb_operator_apply: null data pointer");
  GB_REQUIRE(in != out, "gb_operator_apply: in and out must not alias");
  GB_REQUIRE(!dtype_complex(dtype) || phase_cd, "gb_operator_apply: complex data needs phase_cd");
  cudaStream_t st = (cudaStream_t)stream;
  const double* ph = dtype_complex(dtype) ? phase_cd : nullptr;
  return op_apply(op, in, out, nin, dtype, ph, st, Epilogue());
}

int gb_operator_apply_potential(const gb_operator* op, const void* in, void* out, int64_t nin, int dtype,
                                const void* vt, const double* phase_cd, void* stream) {
  GB_REQUIRE(op && vt, "gb_operator_apply_potential: null operator or potential");
  GB_REQUIRE(dtype_valid(dtype) && nin >= 0, "gb_operator_apply_potential: bad dtype or batch");
  GB_REQUIRE(dtype_complex(dtype) == !op->real,
             "gb_operator_apply_potential: dtype does not match the operator's real/complex flag");
  if (nin == 0) return GB_OK;
  GB_REQUIRE(in && out && in != out, "gb_operator_apply_potential: bad data pointers");
  GB_REQUIRE(!dtype_complex(dtype) || phase_cd, "gb_operator_apply_potential: complex data needs phase_cd");
  Epilogue ep;
  ep.vpot = vt;
  return op_apply(op, in, out, nin, dtype, dtype_complex(dtype) ? phase_cd : nullptr, (cudaStream_t)stream, ep);
}

int gb_operator_apply_k(const gb_operator* op, const void* in, void* out, int64_t nin, int dtype, int nk,
                        const double* phase_kcd, const void* vt, void* stream) {
  GB_REQUIRE(op, "gb_operator_apply_k: null operator");
  GB_REQUIRE(dtype_valid(dtype) && nin >= 0, "gb_operator_apply_k: bad dtype or batch");
  GB_REQUIRE(dtype_complex(dtype) == !op->real,
             "gb_operator_apply_k: dtype does not match the operator's real/complex flag");
  GB_REQUIRE(nk >= 1 && nk <= KMAX, "gb_operator_apply_k: nk must be 1 .. 8");
  GB_REQUIRE(nin % nk == 0, "gb_operator_apply_k: the batch must split into nk equal groups");
  if (nin == 0) return GB_OK;
  GB_REQUIRE(in && out && in != out, "gb_operator_apply_k: bad data pointers");
  GB_REQUIRE(!dtype_complex(dtype) || phase_kcd, "gb_operator_apply_k: complex data needs phases");
  Epilogue ep;
  ep.vpot = vt;
  return op_apply(op, in, out, nin, dtype, dtype_complex(dtype) ? phase_kcd : nullptr, (cudaStream_t)stream, ep,
                  nk);
}

int gb_operator_relax(const gb_operator* op, int relax_method, double* f_g, const double* s_g,
                      int nrelax, double w, void* stream) {
  GB_REQUIRE(op && f_g && s_g, "gb_operator_relax: null pointer");
  GB_REQUIRE(op->real, "gb_operator_relax: real operators only");
  if (relax_method != 2)
    return fail(GB_E_UNSUPPORTED, "gb_operator_relax: only weighted Jacobi (method 2) is implemented");
  GB_REQUIRE(op->diag != 0.0, "gb_operator_relax: zero diagonal");
  BoxArgs a;
  fill_box_args(op, a, nullptr);
  const int64_t N = op->n[0] * op->n[1] * op->n[2];
  double* tmp = nullptr;
  if (cudaMallocAsync(&tmp, N * sizeof(double), (cudaStream_t)stream) != cudaSuccess)
    return fail(GB_E_NOMEM, "gb_operator_relax: scratch allocation failed");
  const int blocks = (int)std::min<int64_t>((N + 255) / 256, (int64_t)sm_count() * 8);
  for (int it = 0; it < nrelax; ++it) {
    jacobi_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(a, f_g, tmp, s_g, w, op->diag);
    cudaMemcpyAsync(f_g, tmp, N * sizeof(double), cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
  }
  cudaFreeAsync(tmp, (cudaStream_t)stream);
  return check_launch("jacobi_kernel");
}

int gb_operator_get_diagonal_element(const gb_operator* op, double* d) {
  GB_REQUIRE(op && d, "gb_operator_get_diagonal_element: null pointer");
  *d = op->diag;
  return GB_OK;
}

int gb_operator_free(gb_operator* op) {
  delete op;
  return GB_OK;
}

}  // extern "C"
