// Localized functions: add / integrate (replaces _gpaw.LFC: c/lfc.c:146-257
// NewLFCObject, 432-505 integrate, 818-885 add, c/lfc.h:79-130 GRID_LOOP).
//
// The reference walks the merged, sorted list of sphere boundaries once per
// band on one core.  Here the same sweep runs once, on the host, when the
// object is built (positions change rarely), and produces two device-side
// indexings of the (grid point, volume, row) incidence:
//
//  * point-major (add):  every grid point covered by at least one sphere owns
//    one thread; it sums  sum_W conj(phase_W) sum_m A_W[row][m] c[x][M_W + m]
//    over the volumes covering it and adds to a[x][G] -- every a[x][G] has a
//    single writer, so there are no atomics and results are deterministic.
//  * function-group-major (integrate): a group is one (atom, radial function)
//    M-range with all its periodic images; one CTA per (group, band block)
//    reduces dv * phase_W * sum_G a[x][G] A_W[row][m] over every image and
//    adds the block's result to c[x][M..M+nm) -- again a single writer.
//
// Derivatives (gb_lfc_derivative, c/lfc.c:1449-1601) are computed on the
// fly from the radial splines: one CTA per (function group, band) walks the
// group's rows, evaluates d/dr_v [f(r) r^l Y_lm] at each point (spline value
// and slope, solid harmonics and their gradients) and reduces
// dv sum_G a[x][G] phase_W d/dr_v Phi to c[x][M][v] -- a single writer.
#include <algorithm>
#include <cstring>
#include <map>
#include <type_traits>
#include <vector>
#include "internal.cuh"
#include "spline.cuh"

struct gb_lfc {
  int nW = 0, nM = 0, maxnm = 0;
  int64_t nG = 0;
  double dv = 1.0;
  int nq = 0;
  // device data
  double* A64 = nullptr;      // concatenated rows of every volume
  float* A32 = nullptr;
  int64_t nA = 0;             // doubles in A
  double2* phase = nullptr;   // [nq][nW]
  // add (point-major)
  int64_t P = 0;              // covered points
  int* pt_G = nullptr;        // [P]
  int* pt_off = nullptr;      // [P+1] into contributions
  int64_t C = 0;              // contributions
  int64_t* ct_aoff = nullptr; // [C] offset into A (doubles)
  int* ct_M = nullptr;        // [C]
  int* ct_nm = nullptr;       // [C]
  int* ct_W = nullptr;        // [C]
  // integrate (group-major)
  int ngroups = 0;
  int* gr_M = nullptr;        // [ngroups]
  int* gr_nm = nullptr;       // [ngroups]
  int* gr_voff = nullptr;     // [ngroups+1] into the volume list
  int* gv_W = nullptr;        // [nW] volumes ordered by group
  int64_t* vol_row0 = nullptr;  // [nW] first global row of W
  int64_t* vol_row1 = nullptr;  // [nW] one past last
  int* row_G = nullptr;       // [rows] grid point of every global row
  int64_t* vol_aoff = nullptr;  // [nW] offset (doubles) of row0 in A
  std::vector<int> h_gr_nm;
  // all-band add for real data (every volume has <= 16 functions): A rows
  // zero-padded to fast_nmax, in contribution order
  int fast_nmax = 0;          // 8 or 16; 0 = not built
  bool full32 = false;        // every contribution: nm == fast_nmax, M and nM multiples of 4
  bool full64 = false;        // the same with multiples of 2 (16-byte FP64 loads)
  float* Ac32 = nullptr;      // [C][fast_nmax]
  double* Ac64 = nullptr;
  // brick-tiled FP32 add / integrate for real data (every volume has <= 8
  // functions, nG a multiple of 4): 32-point chunks of four 8-point
  // sub-tiles; one entry per (volume, sub-tile it touches) with the volume's
  // values there as a dense [m][p] 8 x 8 block (zero where the volume does
  // not cover the point or m >= nm); bricks of consecutive chunks
  bool tiled = false;
  int* tch_c = nullptr;       // [nch] chunk index of every chunk with entries
  int* tch_eoff = nullptr;    // [4 nch + 1] entries of (chunk, sub-tile)
  int* te_info = nullptr;     // [ne] slot in its brick | nm << 8
  float* te_A = nullptr;      // [ne][8][8]
  int tbr_n = 0;              // bricks
  int tbr_smax = 1;           // most slots in a brick
  int tbr_emax = 0;           // most entries in a brick
  int* tbr_ch0 = nullptr;     // [tbr_n + 1] chunk range of each brick
  int* tbr_pbase = nullptr;   // [tbr_n + 1] first (brick, slot) pair
  int64_t tpart_n = 0;        // (brick, slot) pairs
  int* tps_M = nullptr;       // [tpart_n] their group's first function
  int* tps_nm = nullptr;      // [tpart_n] and function count
  int* tps_eoff = nullptr;    // [tpart_n + 1] their entries:
  int* tps_info = nullptr;    //   (entry - brick's first) | sub-tile << 16 | nm << 24
  int* tgr_poff = nullptr;    // [ngroups + 1] the (brick, slot) pairs of each
  int* tgr_pidx = nullptr;    //   group, in brick order
  // work space of the tiled path (transposed coefficients, partial sums);
  // grown outside stream capture only
  mutable void* work = nullptr;
  mutable size_t work_bytes = 0;
  std::vector<void*> allocations;
};

namespace gb {

// trivially-copyable device view passed to the kernels
struct LfcView {
  int nW, nM;
  int64_t nG;
  double dv;
  const double2* phase;
  int64_t P;
  const int* pt_G;
  const int* pt_off;
  const int64_t* ct_aoff;
  const int* ct_M;
  const int* ct_nm;
  const int* ct_W;
  const int* gr_M;
  const int* gr_nm;
  const int* gr_voff;
  const int* gv_W;
  const int64_t* vol_row0;
  const int64_t* vol_row1;
  const int* row_G;
  const int64_t* vol_aoff;
};

// grid geometry for on-the-fly positions (h_cv row-major, local sizes, and
// the global index of the local grid's first point)
struct DerivGeom {
  double h[9];
  int64_t n[3], beg[3];
};

static LfcView view(const gb_lfc* l) {
  LfcView v;
  v.nW = l->nW; v.nM = l->nM; v.nG = l->nG; v.dv = l->dv; v.phase = l->phase;
  v.P = l->P; v.pt_G = l->pt_G; v.pt_off = l->pt_off; v.ct_aoff = l->ct_aoff;
  v.ct_M = l->ct_M; v.ct_nm = l->ct_nm; v.ct_W = l->ct_W; v.gr_M = l->gr_M; v.gr_nm = l->gr_nm;
  v.gr_voff = l->gr_voff; v.gv_W = l->gv_W; v.vol_row0 = l->vol_row0;
  v.vol_row1 = l->vol_row1; v.row_G = l->row_G; v.vol_aoff = l->vol_aoff;
  return v;
}

template <typename T>
static T* dalloc(gb_lfc* l, size_t n) {
  void* p = nullptr;
  if (n == 0) n = 1;
  if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) return nullptr;
  l->allocations.push_back(p);
  return reinterpret_cast<T*>(p);
}

template <typename T>
static bool upload(gb_lfc* l, T** dst, const std::vector<T>& src) {
  *dst = dalloc<T>(l, src.size());
  if (!*dst) return false;
  if (!src.empty() && cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
    return false;
  return true;
}

// --------------------------------------------------------------------- add
template <typename T> struct AType { using A = double; };
template <> struct AType<float> { using A = float; };
template <> struct AType<float2> { using A = float; };

// a row of NMAX values of A (or of the coefficients): 16-byte loads when the
// row is full (nm == NMAX == 8) and 16-byte aligned -- a warp then reads its
// 32 rows in two (FP32) or four (FP64) wide requests instead of 8 strided
// ones -- element loads otherwise
template <typename V, int NMAX>
__device__ __forceinline__ void load_row(const V* __restrict__ src, int nm, V (&dst)[NMAX]) {
  if constexpr (NMAX == 8 && (sizeof(V) == 4 || sizeof(V) == 8)) {
    if (nm == 8 && (reinterpret_cast<uintptr_t>(src) & 15) == 0) {
      if constexpr (sizeof(V) == 4) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(src));
        const float4 b = __ldg(reinterpret_cast<const float4*>(src) + 1);
        dst[0] = a.x; dst[1] = a.y; dst[2] = a.z; dst[3] = a.w;
        dst[4] = b.x; dst[5] = b.y; dst[6] = b.z; dst[7] = b.w;
      } else {
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          const double2 a = __ldg(reinterpret_cast<const double2*>(src) + h);
          dst[2 * h] = a.x;
          dst[2 * h + 1] = a.y;
        }
      }
      return;
    }
  }
#pragma unroll
  for (int m = 0; m < NMAX; ++m) dst[m] = m < nm ? src[m] : (V)0;
}

// one thread per covered point and XB bands; a contribution's NMAX-padded A
// row is loaded once and reused for every band (runtime nm <= NMAX)
template <typename T, int XB, int NMAX>
__global__ void __launch_bounds__(256) lfc_add_kernel(const LfcView l, const typename AType<T>::A* __restrict__ A,
                                                      const T* __restrict__ c_xM, T* __restrict__ a_xG, int64_t nx,
                                                      int q, int64_t per_q) {
  using R = typename Elem<T>::R;
  constexpr bool CPLX = Elem<T>::cplx;
  const int64_t x0 = (int64_t)blockIdx.y * XB;
  const int nb = (int)(nx - x0 < XB ? nx - x0 : XB);
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < l.P; p += (int64_t)gridDim.x * blockDim.x) {
    const int G = l.pt_G[p];
    T acc[XB];
#pragma unroll
    for (int i = 0; i < XB; ++i) acc[i] = zero<T>();
    const int c1 = l.pt_off[p + 1];
    for (int c = l.pt_off[p]; c < c1; ++c) {
      const typename AType<T>::A* Ar = A + l.ct_aoff[c];
      const int M = l.ct_M[c], nm = l.ct_nm[c];
      typename AType<T>::A Aw[NMAX];
      load_row<typename AType<T>::A, NMAX>(Ar, nm, Aw);
      R Av[NMAX];
#pragma unroll
      for (int m = 0; m < NMAX; ++m) Av[m] = (R)Aw[m];
      double pr = 1.0, pi = 0.0;
      if (CPLX && q >= 0 && per_q == 0) {
        const double2 ph = l.phase[(int64_t)q * l.nW + l.ct_W[c]];
        pr = ph.x; pi = -ph.y;   // conj(phase) (c/lfc.c:864)
      }
#pragma unroll
      for (int i = 0; i < XB; ++i) {
        if (i < nb) {
          if (CPLX && q >= 0 && per_q > 0) {
            // k-point of this band: q + band / per_q
            const double2 ph = l.phase[(q + (x0 + i) / per_q) * l.nW + l.ct_W[c]];
            pr = ph.x; pi = -ph.y;
          }
          const T* cx = c_xM + (x0 + i) * l.nM + M;
          T s = zero<T>();
          if constexpr (!CPLX) {
            T cv[NMAX];
            load_row<T, NMAX>(cx, nm, cv);
#pragma unroll
            for (int m = 0; m < NMAX; ++m) s = fmadd(s, Av[m], cv[m]);
          } else {
#pragma unroll
            for (int m = 0; m < NMAX; ++m)
              if (m < nm) s = fmadd(s, Av[m], cx[m]);
          }
          acc[i] = add(acc[i], CPLX ? phase_mul(s, pr, pi) : s);
        }
      }
    }
#pragma unroll
    for (int i = 0; i < XB; ++i) {
      if (i < nb) {
        T* ap = a_xG + (x0 + i) * l.nG + G;
        *ap = add(*ap, acc[i]);
      }
    }
  }
}

// --------------------------------------------------------------- integrate
// one CTA per (function group, XB bands); a group is one atom (all its
// radial functions merged, nm <= NM of them) with all its periodic images
template <typename T, int NM, int XB, int NT>
__global__ void __launch_bounds__(NT) lfc_integrate_kernel(const LfcView l, const typename AType<T>::A* __restrict__ A,
                                                          const T* __restrict__ a_xG, T* __restrict__ c_xM,
                                                          int64_t nx, int q, int group_base, int64_t per_q) {
  using R = typename Elem<T>::R;
  constexpr bool CPLX = Elem<T>::cplx;
  __shared__ T red[NT / 32][XB * NM];
  const int g = group_base + blockIdx.x;
  const int64_t x0 = (int64_t)blockIdx.y * XB;
  const int M = l.gr_M[g];
  const int nm = l.gr_nm[g];
  T acc[XB][NM];
#pragma unroll
  for (int i = 0; i < XB; ++i)
#pragma unroll
    for (int m = 0; m < NM; ++m) acc[i][m] = zero<T>();
  for (int vi = l.gr_voff[g]; vi < l.gr_voff[g + 1]; ++vi) {
    const int W = l.gv_W[vi];
    const int64_t r0 = l.vol_row0[W], r1 = l.vol_row1[W];
    const typename AType<T>::A* AW = A + l.vol_aoff[W];
    double pr = 1.0, pi = 0.0;
    if (CPLX && q >= 0) {
      const double2 ph = l.phase[(int64_t)q * l.nW + W];
      pr = ph.x; pi = ph.y;
    }
    if constexpr (!CPLX) {
      // real data: every image has phase 1, accumulate straight into acc
      // FP32: four rows per pass put 16 gathered loads in flight (1.1x on
      // the Si64 shape); FP64 measured no faster unrolled
      constexpr int RUN = sizeof(R) == 4 ? 4 : 1;
#pragma unroll RUN
      for (int64_t r = r0 + threadIdx.x; r < r1; r += NT) {
        const int G = l.row_G[r];
        typename AType<T>::A Aw[NM];
        load_row<typename AType<T>::A, NM>(AW + (r - r0) * nm, nm, Aw);
        R Ar[NM];
#pragma unroll
        for (int m = 0; m < NM; ++m) Ar[m] = (R)Aw[m];
#pragma unroll
        for (int i = 0; i < XB; ++i) {
          if (x0 + i < nx) {
            const T v = a_xG[(x0 + i) * l.nG + G];
#pragma unroll
            for (int m = 0; m < NM; ++m) acc[i][m] = fmadd(acc[i][m], Ar[m], v);
          }
        }
      }
    } else {
      T part[XB][NM];
#pragma unroll
      for (int i = 0; i < XB; ++i)
#pragma unroll
        for (int m = 0; m < NM; ++m) part[i][m] = zero<T>();
      for (int64_t r = r0 + threadIdx.x; r < r1; r += NT) {
        const int G = l.row_G[r];
        R Ar[NM];
#pragma unroll
        for (int m = 0; m < NM; ++m) Ar[m] = m < nm ? (R)AW[(r - r0) * nm + m] : (R)0;
#pragma unroll
        for (int i = 0; i < XB; ++i) {
          if (x0 + i < nx) {
            const T v = a_xG[(x0 + i) * l.nG + G];
#pragma unroll
            for (int m = 0; m < NM; ++m) part[i][m] = fmadd(part[i][m], Ar[m], v);
          }
        }
      }
#pragma unroll
      for (int i = 0; i < XB; ++i) {
        double qr = pr, qi = pi;
        if (q >= 0 && per_q > 0 && x0 + i < nx) {
          const double2 ph = l.phase[(q + (x0 + i) / per_q) * l.nW + W];
          qr = ph.x; qi = ph.y;
        }
#pragma unroll
        for (int m = 0; m < NM; ++m) acc[i][m] = add(acc[i][m], phase_mul(part[i][m], qr, qi));
      }
    }
  }
  // block reduction: warp shuffles, then across warps
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < XB; ++i)
#pragma unroll
    for (int m = 0; m < NM; ++m) {
      T v = acc[i][m];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        if constexpr (CPLX) {
          v.x += __shfl_down_sync(0xffffffffu, v.x, o);
          v.y += __shfl_down_sync(0xffffffffu, v.y, o);
        } else {
          v += __shfl_down_sync(0xffffffffu, v, o);
        }
      }
      if (lane == 0) red[warp][i * NM + m] = v;
    }
  __syncthreads();
  for (int e = threadIdx.x; e < XB * NM; e += NT) {
    const int i = e / NM, m = e % NM;
    if (x0 + i >= nx || m >= nm) continue;
    T v = zero<T>();
    for (int w = 0; w < NT / 32; ++w) v = add(v, red[w][e]);
    T* cp = c_xM + (x0 + i) * l.nM + M + m;
    *cp = fmadd(*cp, (R)l.dv, v);
  }
}

// ------------------------------------------------ real data, all bands
// For real data (Gamma point: every periodic image has phase 1) and at most
// 16 functions per volume, the add runs every band in one pass: one thread
// per covered point holds the zero-padded A rows of its first KREG
// contributions in registers (a copy of A in contribution order, so a warp's
// row loads are contiguous) and loops over the bands XU at a time, issuing
// the XU read-modify-write loads of a[x][G] before the coefficient loads and
// FMAs of those bands.  Per band it sums the contributions in point order,
// m within each, as lfc_add_kernel does, so the two give identical results.
// (The same all-band treatment of the integrate, with row tiles of A staged in
// shared memory per (group, 16-band) CTA, measured no faster than
// lfc_integrate_kernel on the Si64 shape and slower in FP64, so the integrate
// keeps the kernel above.)
template <typename T, int NMAX, bool FULL>
__device__ __forceinline__ void load_coef(const T* __restrict__ cx, int nm, T (&v)[NMAX]) {
  if constexpr (FULL) {
    // every contribution has NMAX functions at a 16-byte aligned offset
    if constexpr (sizeof(T) == 4) {
#pragma unroll
      for (int h = 0; h < NMAX / 4; ++h) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(cx) + h);
        v[4 * h] = a.x; v[4 * h + 1] = a.y; v[4 * h + 2] = a.z; v[4 * h + 3] = a.w;
      }
    } else {
#pragma unroll
      for (int h = 0; h < NMAX / 2; ++h) {
        const double2 a = __ldg(reinterpret_cast<const double2*>(cx) + h);
        v[2 * h] = a.x; v[2 * h + 1] = a.y;
      }
    }
  } else {
#pragma unroll
    for (int m = 0; m < NMAX; ++m) v[m] = m < nm ? __ldg(cx + m) : (T)0;
  }
}

template <typename T, int NMAX>
__device__ __forceinline__ void load_padded_row(const T* __restrict__ src, T (&v)[NMAX]) {
  if constexpr (sizeof(T) == 4) {
#pragma unroll
    for (int h = 0; h < NMAX / 4; ++h) {
      const float4 a = __ldg(reinterpret_cast<const float4*>(src) + h);
      v[4 * h] = a.x; v[4 * h + 1] = a.y; v[4 * h + 2] = a.z; v[4 * h + 3] = a.w;
    }
  } else {
#pragma unroll
    for (int h = 0; h < NMAX / 2; ++h) {
      const double2 a = __ldg(reinterpret_cast<const double2*>(src) + h);
      v[2 * h] = a.x; v[2 * h + 1] = a.y;
    }
  }
}

// acc[u] += sum_m A[m] c[x0 + u][M + m], u < NU, cx = &c[x0][M] (the
// contribution's sum is formed first, then added, as in lfc_add_kernel)
template <typename T, int NMAX, bool FULL, int NU>
__device__ __forceinline__ void add_contribution(const T (&A)[NMAX], const T* __restrict__ cx, int nM, int nm,
                                                 T (&acc)[NU]) {
#pragma unroll
  for (int u = 0; u < NU; ++u) {
    T cv[NMAX];
    load_coef<T, NMAX, FULL>(cx, nm, cv);
    T t = (T)0;
#pragma unroll
    for (int m = 0; m < NMAX; ++m) t = fmadd(t, A[m], cv[m]);
    acc[u] += t;
    cx += nM;
  }
}

// bands x0 .. x0+NU-1 of one point: a[x][G] += sum_k sum_m A_k[m] c[x][M_k + m]
template <typename T, int NMAX, int KREG, bool FULL, int NU>
__device__ __forceinline__ void add_point_bands(const T (&A)[KREG][NMAX], const T* const (&cb)[KREG],
                                                const int (&nmk)[KREG], int K, int k0,
                                                const int* __restrict__ ct_M, const int* __restrict__ ct_nm,
                                                const T* __restrict__ Ac, const T* __restrict__ c_xM, int nM,
                                                int64_t x0, T* __restrict__ ax, int64_t nG) {
  // the read-modify-write loads first: their latency overlaps the FMAs
  T av[NU], acc[NU];
  {
    const T* q = ax;
#pragma unroll
    for (int u = 0; u < NU; ++u) {
      av[u] = *q;
      acc[u] = (T)0;
      q += nG;
    }
  }
  const int64_t xo = x0 * nM;
#pragma unroll
  for (int k = 0; k < KREG; ++k)
    if (k < K) add_contribution<T, NMAX, FULL, NU>(A[k], cb[k] + xo, nM, nmk[k], acc);
  for (int k = KREG; k < K; ++k) {
    T Ak[NMAX];
    load_padded_row<T, NMAX>(Ac + (int64_t)(k0 + k) * NMAX, Ak);
    add_contribution<T, NMAX, FULL, NU>(Ak, c_xM + ct_M[k0 + k] + xo, nM, ct_nm[k0 + k], acc);
  }
  T* q = ax;
#pragma unroll
  for (int u = 0; u < NU; ++u) {
    *q = av[u] + acc[u];
    q += nG;
  }
}

template <typename T, int NMAX, int KREG, bool FULL, int XU>
__global__ void __launch_bounds__(256) lfc_add_bands_kernel(const int* __restrict__ pt_G,
                                                            const int* __restrict__ pt_off,
                                                            const int* __restrict__ ct_M,
                                                            const int* __restrict__ ct_nm,
                                                            const T* __restrict__ Ac, int64_t P,
                                                            const T* __restrict__ c_xM, int nM,
                                                            T* __restrict__ a_xG, int64_t nG, int64_t nx) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= P) return;
  const int G = pt_G[p];
  const int k0 = pt_off[p], K = pt_off[p + 1] - k0;
  T A[KREG][NMAX];
  const T* cb[KREG];
  int nmk[KREG];
#pragma unroll
  for (int k = 0; k < KREG; ++k) {
    if (k < K) {
      load_padded_row<T, NMAX>(Ac + (int64_t)(k0 + k) * NMAX, A[k]);
      cb[k] = c_xM + ct_M[k0 + k];
      nmk[k] = ct_nm[k0 + k];
    } else {
#pragma unroll
      for (int m = 0; m < NMAX; ++m) A[k][m] = (T)0;
      cb[k] = c_xM;
      nmk[k] = 0;
    }
  }
  const int64_t nfull = nx / XU * XU;
  T* ax = a_xG + G;
  for (int64_t x0 = 0; x0 < nfull; x0 += XU, ax += XU * nG)
    add_point_bands<T, NMAX, KREG, FULL, XU>(A, cb, nmk, K, k0, ct_M, ct_nm, Ac, c_xM, nM, x0, ax, nG);
  for (int64_t x0 = nfull; x0 < nx; ++x0, ax += nG)
    add_point_bands<T, NMAX, KREG, FULL, 1>(A, cb, nmk, K, k0, ct_M, ct_nm, Ac, c_xM, nM, x0, ax, nG);
}

template <typename T, int NM>
static int integrate_nm(const gb_lfc* l, int gbeg, int gcount, const void* a, void* c, int64_t nx, int q,
                        int64_t per_q,
                        cudaStream_t st) {
  // accumulators per thread: XB x NM (twice that for complex images)
  constexpr int XB0 = NM <= 2 ? 16 : (NM <= 4 ? 8 : (NM <= 8 ? 4 : (NM <= 16 ? 2 : 1)));
  constexpr int XB = Elem<T>::cplx ? (XB0 >= 4 ? XB0 / 4 : 1) : XB0;
  constexpr int NT = 128;
  const typename AType<T>::A* A;
  if constexpr (std::is_same<typename AType<T>::A, float>::value) A = l->A32; else A = l->A64;
  dim3 grid((unsigned)gcount, (unsigned)((nx + XB - 1) / XB));
  lfc_integrate_kernel<T, NM, XB, NT><<<grid, NT, 0, st>>>(view(l), A, (const T*)a, (T*)c, nx, q, gbeg, per_q);
  return check_launch("lfc_integrate_kernel");
}

// smallest supported padded function count >= nm
static int nm_class(int nm) {
  for (int c : {1, 2, 4, 8, 16, 32, 64})
    if (nm <= c) return c;
  return 0;
}

template <typename T>
static int add_fast(const gb_lfc* l, const void* c, void* a, int64_t nx, cudaStream_t st) {
  const T* Ac;
  if constexpr (sizeof(T) == 4) Ac = l->Ac32; else Ac = l->Ac64;
  const bool full = (sizeof(T) == 4 ? l->full32 : l->full64) && (reinterpret_cast<uintptr_t>(c) & 15) == 0;
  constexpr int NT = 256, XU = 8;
  const unsigned grid = (unsigned)((l->P + NT - 1) / NT);
  const T* cc = (const T*)c;
  T* aa = (T*)a;
#define GB_ADD_BANDS(NMAX, KREG, FULL)                                                                        \
  lfc_add_bands_kernel<T, NMAX, KREG, FULL, XU><<<grid, NT, 0, st>>>(l->pt_G, l->pt_off, l->ct_M, l->ct_nm, Ac, \
                                                                      l->P, cc, l->nM, aa, l->nG, nx)
  constexpr int K8 = sizeof(T) == 4 ? 4 : 2, K16 = sizeof(T) == 4 ? 2 : 1;
  if (l->fast_nmax == 8) {
    if (full) GB_ADD_BANDS(8, K8, true); else GB_ADD_BANDS(8, K8, false);
  } else {
    if (full) GB_ADD_BANDS(16, K16, true); else GB_ADD_BANDS(16, K16, false);
  }
#undef GB_ADD_BANDS
  return check_launch("lfc_add_bands_kernel");
}

static bool tiles_usable(const gb_lfc* l, const void* a);
static int integrate_tiles(const gb_lfc* l, const float* a, float* c, int64_t nx, cudaStream_t st);

template <typename T>
static int integrate_t(const gb_lfc* l, const void* a, void* c, int64_t nx, int q, cudaStream_t st,
                       int64_t per_q = 0) {
  if constexpr (std::is_same<T, float>::value) {
    if (tiles_usable(l, a))
      return integrate_tiles(l, static_cast<const float*>(a), static_cast<float*>(c), nx, st);
  }
  // groups are sorted by nm on the host; one launch per padded class
  int g = 0;
  while (g < l->ngroups) {
    const int cls = nm_class(l->h_gr_nm[g]);
    int e = g;
    while (e < l->ngroups && nm_class(l->h_gr_nm[e]) == cls) ++e;
    int rc;
    switch (cls) {
      case 1: rc = integrate_nm<T, 1>(l, g, e - g, a, c, nx, q, per_q, st); break;
      case 2: rc = integrate_nm<T, 2>(l, g, e - g, a, c, nx, q, per_q, st); break;
      case 4: rc = integrate_nm<T, 4>(l, g, e - g, a, c, nx, q, per_q, st); break;
      case 8: rc = integrate_nm<T, 8>(l, g, e - g, a, c, nx, q, per_q, st); break;
      case 16: rc = integrate_nm<T, 16>(l, g, e - g, a, c, nx, q, per_q, st); break;
      case 32: rc = integrate_nm<T, 32>(l, g, e - g, a, c, nx, q, per_q, st); break;
      case 64: rc = integrate_nm<T, 64>(l, g, e - g, a, c, nx, q, per_q, st); break;
      default: return fail(GB_E_UNSUPPORTED, "lfc: more than 64 functions in one volume");
    }
    if (rc) return rc;
    g = e;
  }
  return GB_OK;
}

template <typename T, int XB, int NMAX>
static int add_nm(const gb_lfc* l, const void* c, void* a, int64_t nx, int q, cudaStream_t st, int64_t per_q) {
  const typename AType<T>::A* A;
  if constexpr (std::is_same<typename AType<T>::A, float>::value) A = l->A32; else A = l->A64;
  const int NT = 256;
  const int64_t bx = std::min<int64_t>((l->P + NT - 1) / NT, (int64_t)sm_count() * 8);
  dim3 grid((unsigned)bx, (unsigned)((nx + XB - 1) / XB));
  lfc_add_kernel<T, XB, NMAX><<<grid, NT, 0, st>>>(view(l), A, (const T*)c, (T*)a, nx, q, per_q);
  return check_launch("lfc_add_kernel");
}


// ------------------------------------------------ brick-tiled FP32 (real)
// The flattened grid is cut into 32-point chunks of four 8-point sub-tiles;
// an entry is one (volume, sub-tile it touches) with the volume's values
// there as a dense [m][p] 8 x 8 block.  A brick is a run of at most TBRICK
// consecutive chunks with entries that meets at most TSLOTS function groups
// (its slots) and holds at most TBENT entries.  One CTA takes one (brick,
// group of 32 bands) and first copies into shared memory, with coalesced
// 16-byte cp.async copies, the brick's rows of a (a band row pitch of
// 32 TBRICK + 4 floats, so that lanes reading one band each do not collide
// on banks), its entries' blocks and, for the add, the coefficients of its
// slots as [slot][m][band] (rows of cT, c transposed by a first kernel).
// Every operand of the FMAs then comes from shared memory.
//  add:        warp w updates sub-tiles w, w + 8, ... in place (one owner per
//              sub-tile): a[x][p] += sum_e sum_m A_e[m][p] c[x][M_e + m];
//              the brick's rows are then written back.
//  integrate:  warp s sums slot s over its entries (lists made on the host)
//              and writes one partial sum per (brick, slot, band); a second
//              kernel adds dv times each group's partials, in brick order,
//              to c.
// No atomics: the results do not depend on scheduling.
constexpr int TCH = 32;                    // points per chunk
constexpr int TSLOTS = 16;                 // function groups per brick
constexpr int TBRICK = 8;                  // chunks per brick
constexpr int TBENT = 192;                 // entries per brick
constexpr int TBAND = 32;                  // bands per CTA
constexpr int TPITCH = TBRICK * TCH + 4;   // floats per band row in shared memory
constexpr int TADD_WARPS = 16;

struct TileView {
  const int* ch_c;      // [nch] chunk index (first point 32 c) of every used chunk
  const int* ch_eoff;   // [4 nch + 1] entries of (chunk, sub-tile)
  const int* e_info;    // [ne] slot | nm << 8
  const float* e_A;     // [ne][8][8]
  const int* br_ch0;    // [nbr + 1] chunk range of each brick
  const int* br_pbase;  // [nbr + 1] first (brick, slot) pair of each brick
  const int* ps_M;      // [npart] group of each (brick, slot): its first function
  const int* ps_nm;     // [npart] and function count
  const int* ps_eoff;   // [npart + 1] entries of each (brick, slot):
  const int* ps_info;   //   (entry - first entry of the brick) | sub-tile << 16 | nm << 24
};

static TileView tile_view(const gb_lfc* l) {
  return TileView{l->tch_c, l->tch_eoff, l->te_info, l->te_A, l->tbr_ch0, l->tbr_pbase,
                  l->tps_M, l->tps_nm, l->tps_eoff, l->tps_info};
}

// shared-memory copy of brick b for bands x0 .. x0 + nb - 1 (of the rows at a)
__device__ __forceinline__ void brick_stage(const TileView& t, int b, const float* __restrict__ a, int64_t nG,
                                            int x0, int nb, float* sa, float* sA, float* sc,
                                            const float* __restrict__ cT, int ldT) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int k0 = t.br_ch0[b], nk = t.br_ch0[b + 1] - k0;
  for (int x = warp; x < nb; x += nw) {
    const float* src = a + (int64_t)(x0 + x) * nG;
    for (int i = lane; i < nk * 8; i += 32) {
      const int kk = i >> 3, q = i & 7;
      const int64_t G = (int64_t)t.ch_c[k0 + kk] * TCH + 4 * q;
      float* d = sa + x * TPITCH + kk * TCH + 4 * q;
      if (G < nG) cp_async16(d, src + G);
      else *reinterpret_cast<float4*>(d) = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
  const int E0 = t.ch_eoff[4 * k0], E1 = t.ch_eoff[4 * (k0 + nk)];
  for (int i = threadIdx.x; i < (E1 - E0) * 16; i += blockDim.x) cp_async16(sA + 4 * i, t.e_A + (int64_t)E0 * 64 + 4 * i);
  if (sc) {
    const int pbase = t.br_pbase[b], S = t.br_pbase[b + 1] - pbase;
    for (int r = warp; r < S * 8; r += nw) {
      const int s = r >> 3, m = r & 7;
      if (lane < 8) {
        float* d = sc + r * TBAND + 4 * lane;
        if (m < t.ps_nm[pbase + s]) cp_async16(d, cT + (int64_t)(t.ps_M[pbase + s] + m) * ldT + x0 + 4 * lane);
        else *reinterpret_cast<float4*>(d) = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
}

__global__ void lfc_coef_transpose_kernel(const float* __restrict__ c, int nM, int R, int ldT, float* __restrict__ cT) {
  __shared__ float tile[32][33];
  const int M0 = blockIdx.x * 32, x0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int x = x0 + i, M = M0 + threadIdx.x;
    tile[i][threadIdx.x] = (x < R && M < nM) ? c[(int64_t)x * nM + M] : 0.f;
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int M = M0 + i;
    if (M < nM) cT[(int64_t)M * ldT + x0 + threadIdx.x] = tile[threadIdx.x][i];
  }
}

// acc (points 2k, 2k+1 in acc[k]) += A row m (4 float2) * cv
__device__ __forceinline__ void add_row(float2 (&acc)[4], const float4* __restrict__ Ab, int m, float cv) {
  const float4 A0 = Ab[2 * m], A1 = Ab[2 * m + 1];
  const float2 c2 = make_float2(cv, cv);
  acc[0] = __ffma2_rn(make_float2(A0.x, A0.y), c2, acc[0]);
  acc[1] = __ffma2_rn(make_float2(A0.z, A0.w), c2, acc[1]);
  acc[2] = __ffma2_rn(make_float2(A1.x, A1.y), c2, acc[2]);
  acc[3] = __ffma2_rn(make_float2(A1.z, A1.w), c2, acc[3]);
}

__global__ void __launch_bounds__(32 * TADD_WARPS) lfc_add_tiles_kernel(const TileView t, const float* __restrict__ cT,
                                                                       int ldT, float* __restrict__ a, int64_t nG,
                                                                       int R, int sA_floats) {
  extern __shared__ __align__(16) float tsm[];
  float* sa = tsm;
  float* sA = sa + TBAND * TPITCH;
  float* sc = sA + sA_floats;
  const int b = blockIdx.x, x0 = blockIdx.y * TBAND;
  const int nb = min(TBAND, R - x0);
  brick_stage(t, b, a, nG, x0, nb, sa, sA, sc, cT, ldT);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int k0 = t.br_ch0[b], nk = t.br_ch0[b + 1] - k0;
  const int E0 = t.ch_eoff[4 * k0];
  for (int st = warp; st < 4 * nk; st += TADD_WARPS) {
    const int e0 = t.ch_eoff[4 * k0 + st], e1 = t.ch_eoff[4 * k0 + st + 1];
    if (e0 == e1) continue;
    float* row = sa + lane * TPITCH + 8 * st;
    const float4 u = *reinterpret_cast<const float4*>(row), v = *reinterpret_cast<const float4*>(row + 4);
    float2 acc[4] = {make_float2(u.x, u.y), make_float2(u.z, u.w), make_float2(v.x, v.y), make_float2(v.z, v.w)};
    int info = t.e_info[e0];
    for (int e = e0; e < e1; ++e) {
      const int nm = info >> 8;
      const float4* Ab = reinterpret_cast<const float4*>(sA + (e - E0) * 64);
      const float* cs = sc + (info & 255) * 8 * TBAND + lane;
      if (e + 1 < e1) info = t.e_info[e + 1];
      if (nm == 8) {
#pragma unroll
        for (int m = 0; m < 8; ++m) add_row(acc, Ab, m, cs[m * TBAND]);
      } else {
        for (int m = 0; m < nm; ++m) add_row(acc, Ab, m, cs[m * TBAND]);
      }
    }
    *reinterpret_cast<float4*>(row) = make_float4(acc[0].x, acc[0].y, acc[1].x, acc[1].y);
    *reinterpret_cast<float4*>(row + 4) = make_float4(acc[2].x, acc[2].y, acc[3].x, acc[3].y);
  }
  __syncthreads();
  const int nw = blockDim.x >> 5;
  for (int x = warp; x < nb; x += nw) {
    float* dst = a + (int64_t)(x0 + x) * nG;
    for (int i = lane; i < nk * 8; i += 32) {
      const int kk = i >> 3, q = i & 7;
      const int64_t G = (int64_t)t.ch_c[k0 + kk] * TCH + 4 * q;
      if (G < nG)
        *reinterpret_cast<float4*>(dst + G) = *reinterpret_cast<const float4*>(sa + x * TPITCH + kk * TCH + 4 * q);
    }
  }
}

// acc[m] (even / odd point sums) += A row m . av
__device__ __forceinline__ void int_row(float2 (&acc)[8], const float4* __restrict__ Ab, int m, const float2 (&av)[4]) {
  const float4 A0 = Ab[2 * m], A1 = Ab[2 * m + 1];
  float2 s = acc[m];
  s = __ffma2_rn(make_float2(A0.x, A0.y), av[0], s);
  s = __ffma2_rn(make_float2(A0.z, A0.w), av[1], s);
  s = __ffma2_rn(make_float2(A1.x, A1.y), av[2], s);
  s = __ffma2_rn(make_float2(A1.z, A1.w), av[3], s);
  acc[m] = s;
}

__global__ void __launch_bounds__(32 * TSLOTS) lfc_integrate_tiles_kernel(const TileView t,
                                                                         const float* __restrict__ a, int64_t nG,
                                                                         int R, float* __restrict__ part) {
  extern __shared__ __align__(16) float tsm[];
  float* sa = tsm;
  float* sA = sa + TBAND * TPITCH;
  const int b = blockIdx.x, x0 = blockIdx.y * TBAND;
  const int nb = min(TBAND, R - x0);
  brick_stage(t, b, a, nG, x0, nb, sa, sA, nullptr, nullptr, 0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int pbase = t.br_pbase[b], S = t.br_pbase[b + 1] - pbase;
  if (warp >= S) return;
  float2 acc[8];
#pragma unroll
  for (int m = 0; m < 8; ++m) acc[m] = make_float2(0.f, 0.f);
  const int q0 = t.ps_eoff[pbase + warp], q1 = t.ps_eoff[pbase + warp + 1];
  int info = q0 < q1 ? t.ps_info[q0] : 0;
  for (int q = q0; q < q1; ++q) {
    const int el = info & 0xffff, lst = (info >> 16) & 255, nm = info >> 24;
    if (q + 1 < q1) info = t.ps_info[q + 1];
    const float* row = sa + lane * TPITCH + 8 * lst;
    const float4 u = *reinterpret_cast<const float4*>(row), v = *reinterpret_cast<const float4*>(row + 4);
    const float2 av[4] = {make_float2(u.x, u.y), make_float2(u.z, u.w), make_float2(v.x, v.y), make_float2(v.z, v.w)};
    const float4* Ab = reinterpret_cast<const float4*>(sA + el * 64);
    if (nm == 8) {
#pragma unroll
      for (int m = 0; m < 8; ++m) int_row(acc, Ab, m, av);
    } else {
#pragma unroll
      for (int m = 0; m < 8; ++m)
        if (m < nm) int_row(acc, Ab, m, av);
    }
  }
  if (lane < nb) {
    float4* d = reinterpret_cast<float4*>(part + ((int64_t)(pbase + warp) * R + x0 + lane) * 8);
    d[0] = make_float4(acc[0].x + acc[0].y, acc[1].x + acc[1].y, acc[2].x + acc[2].y, acc[3].x + acc[3].y);
    d[1] = make_float4(acc[4].x + acc[4].y, acc[5].x + acc[5].y, acc[6].x + acc[6].y, acc[7].x + acc[7].y);
  }
}

// c[x][M_g + m] += dv sum of group g's partials.  A CTA takes 32 outputs
// (x, m) of one group -- four bands -- and eight slices of its partial list:
// thread (slice s, output o) sums partials s, s + 8, ... (32 consecutive
// floats per partial: coalesced), then the eight sums are added in slice
// order.  Fixed order throughout: results do not depend on scheduling.
__global__ void __launch_bounds__(256) lfc_tiles_reduce_kernel(const int* __restrict__ gr_M,
                                                              const int* __restrict__ gr_nm,
                                                              const int* __restrict__ poff,
                                                              const int* __restrict__ pidx,
                                                              const float* __restrict__ part, int R,
                                                              float* __restrict__ c, int nM, float dv) {
  __shared__ float red[8][33];
  const int g = blockIdx.y;
  const int o = threadIdx.x & 31, sl = threadIdx.x >> 5;
  const int i = blockIdx.x * 32 + o;              // output (x, m) = (i / 8, i % 8)
  float s = 0.f;
  if (i < R * 8) {
    const float* pp = part + i;
    const int64_t ps = (int64_t)R * 8;
    const int q1 = poff[g + 1];
    for (int q = poff[g] + sl; q < q1; q += 8) s += pp[pidx[q] * ps];
  }
  red[sl][o] = s;
  __syncthreads();
  if (sl == 0 && i < R * 8) {
    const int x = i >> 3, m = i & 7;
    if (m < gr_nm[g]) {
      float t = red[0][o];
#pragma unroll
      for (int k = 1; k < 8; ++k) t += red[k][o];
      float* cp = c + (int64_t)x * nM + gr_M[g] + m;
      *cp = fmaf(dv, t, *cp);
    }
  }
}

// grow the work space (never inside stream capture)
static int tile_work(const gb_lfc* l, size_t bytes, cudaStream_t st) {
  if (bytes <= l->work_bytes) return GB_OK;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
    return fail(GB_E_INVALID, "lfc: the tiled FP32 path needs a larger work space; make one call of this size "
                              "before capturing it in a graph");
  if (l->work) {
    if (cudaStreamSynchronize(st) != cudaSuccess) return check_launch("lfc work space");
    cudaFree(l->work);
    l->work = nullptr;
    l->work_bytes = 0;
  }
  if (cudaMalloc(&l->work, bytes) != cudaSuccess) {
    l->work = nullptr;
    return fail(GB_E_NOMEM, "lfc: work space allocation failed");
  }
  l->work_bytes = bytes;
  return GB_OK;
}

static int tile_smem_attr() {
  static int done = 0;
  if (!done) {
    const int mx = (TBAND * TPITCH + TBENT * 64 + TSLOTS * 8 * TBAND) * (int)sizeof(float);
    if (cudaFuncSetAttribute(lfc_add_tiles_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) != cudaSuccess ||
        cudaFuncSetAttribute(lfc_integrate_tiles_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) !=
            cudaSuccess)
      return check_launch("lfc tiled shared memory");
    done = 1;
  }
  return GB_OK;
}

// usable for this call: FP32 real data, rows 16-byte aligned
static bool tiles_usable(const gb_lfc* l, const void* a) {
  return l->tiled && (reinterpret_cast<uintptr_t>(a) & 15) == 0;
}

// passes of at most 256 bands bound the work space
static int add_tiles(const gb_lfc* l, const float* c, float* a, int64_t nx, cudaStream_t st) {
  if (l->tbr_n == 0) return GB_OK;
  int rc = tile_smem_attr();
  if (rc) return rc;
  const int Rmax = (int)std::min<int64_t>(nx, 256);
  rc = tile_work(l, (size_t)l->nM * ((Rmax + 31) / 32 * 32) * sizeof(float), st);
  if (rc) return rc;
  float* cT = static_cast<float*>(l->work);
  const int sA_floats = l->tbr_emax * 64;
  const int smem = (TBAND * TPITCH + sA_floats + TSLOTS * 8 * TBAND) * (int)sizeof(float);
  for (int64_t x0 = 0; x0 < nx; x0 += 256) {
    const int R = (int)std::min<int64_t>(nx - x0, 256);
    const int ldT = (R + 31) / 32 * 32;
    dim3 tg((unsigned)((l->nM + 31) / 32), (unsigned)(ldT / 32));
    lfc_coef_transpose_kernel<<<tg, dim3(32, 8), 0, st>>>(c + x0 * l->nM, l->nM, R, ldT, cT);
    dim3 grid((unsigned)l->tbr_n, (unsigned)(ldT / TBAND));
    lfc_add_tiles_kernel<<<grid, 32 * TADD_WARPS, smem, st>>>(tile_view(l), cT, ldT, a + x0 * l->nG, l->nG, R,
                                                              sA_floats);
    rc = check_launch("lfc_add_tiles_kernel");
    if (rc) return rc;
  }
  return GB_OK;
}

static int integrate_tiles(const gb_lfc* l, const float* a, float* c, int64_t nx, cudaStream_t st) {
  if (l->tbr_n == 0) return GB_OK;
  int rc = tile_smem_attr();
  if (rc) return rc;
  const int Rmax = (int)std::min<int64_t>(nx, 256);
  rc = tile_work(l, (size_t)l->tpart_n * Rmax * 8 * sizeof(float), st);
  if (rc) return rc;
  float* part = static_cast<float*>(l->work);
  const int smem = (TBAND * TPITCH + l->tbr_emax * 64) * (int)sizeof(float);
  for (int64_t x0 = 0; x0 < nx; x0 += 256) {
    const int R = (int)std::min<int64_t>(nx - x0, 256);
    dim3 grid((unsigned)l->tbr_n, (unsigned)((R + TBAND - 1) / TBAND));
    lfc_integrate_tiles_kernel<<<grid, 32 * l->tbr_smax, smem, st>>>(tile_view(l), a + x0 * l->nG, l->nG, R, part);
    rc = check_launch("lfc_integrate_tiles_kernel");
    if (rc) return rc;
    dim3 rg((unsigned)((R * 8 + 31) / 32), (unsigned)l->ngroups);
    lfc_tiles_reduce_kernel<<<rg, 256, 0, st>>>(l->gr_M, l->gr_nm, l->tgr_poff, l->tgr_pidx, part, R,
                                                c + x0 * l->nM, l->nM, (float)l->dv);
    rc = check_launch("lfc_tiles_reduce_kernel");
    if (rc) return rc;
  }
  return GB_OK;
}


template <typename T>
static int add_t(const gb_lfc* l, const void* c, void* a, int64_t nx, int q, cudaStream_t st,
                 int64_t per_q = 0) {
  if (l->P == 0) return GB_OK;
  if constexpr (std::is_same<T, float>::value) {
    if (tiles_usable(l, a)) return add_tiles(l, static_cast<const float*>(c), static_cast<float*>(a), nx, st);
  }
  if constexpr (!Elem<T>::cplx) {
    if (l->fast_nmax) return add_fast<T>(l, c, a, nx, st);
  }
  switch (nm_class(l->maxnm)) {
    case 1: return add_nm<T, 8, 1>(l, c, a, nx, q, st, per_q);
    case 2: return add_nm<T, 8, 2>(l, c, a, nx, q, st, per_q);
    case 4: return add_nm<T, 8, 4>(l, c, a, nx, q, st, per_q);
    case 8: return add_nm<T, 8, 8>(l, c, a, nx, q, st, per_q);
    case 16: return add_nm<T, 4, 16>(l, c, a, nx, q, st, per_q);
    case 32: return add_nm<T, 2, 32>(l, c, a, nx, q, st, per_q);
    case 64: return add_nm<T, 1, 64>(l, c, a, nx, q, st, per_q);
    default: return fail(GB_E_UNSUPPORTED, "lfc: more than 64 functions in one volume");
  }
}

static __global__ void to_float(const double* a, float* b, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

}  // namespace gb

namespace gb {
SplineDev spline_view(const gb_spline* s);

struct SplineM {          // the radial function of one M and its m index
  SplineDev s;
  int m;
};

// one CTA per (function group, band); up to 16 functions per volume
template <typename T>
__global__ void __launch_bounds__(128) lfc_derivative_kernel(const LfcView l, const SplineM* __restrict__ spl,
                                                             const double* __restrict__ pos_W, DerivGeom geo,
                                                             const T* __restrict__ a_xG, T* __restrict__ c_xMv,
                                                             int q) {
  constexpr bool CPLX = Elem<T>::cplx;
  using Acc = typename std::conditional<CPLX, double2, double>::type;
  constexpr int NT = 128, NMV = 48;
  __shared__ Acc red[NT / 32][NMV];
  const int g = blockIdx.x;
  const int64_t x = blockIdx.y;
  const int M0 = l.gr_M[g];
  const int nm = l.gr_nm[g];
  Acc acc[NMV];
#pragma unroll
  for (int i = 0; i < NMV; ++i) acc[i] = zero<Acc>();
  for (int vi = l.gr_voff[g]; vi < l.gr_voff[g + 1]; ++vi) {
    const int W = l.gv_W[vi];
    double pr = 1.0, pi = 0.0;
    if (CPLX && q >= 0) {
      const double2 ph = l.phase[(int64_t)q * l.nW + W];
      pr = ph.x;
      pi = ph.y;
    }
    const double px = pos_W[3 * W], py = pos_W[3 * W + 1], pz = pos_W[3 * W + 2];
    for (int64_t r = l.vol_row0[W] + threadIdx.x; r < l.vol_row1[W]; r += NT) {
      const int64_t G = l.row_G[r];
      const int64_t i2 = G % geo.n[2] + geo.beg[2];
      const int64_t i1 = (G / geo.n[2]) % geo.n[1] + geo.beg[1];
      const int64_t i0 = G / (geo.n[2] * geo.n[1]) + geo.beg[0];
      const double X = geo.h[0] * i0 + geo.h[3] * i1 + geo.h[6] * i2 - px;
      const double Y = geo.h[1] * i0 + geo.h[4] * i1 + geo.h[7] * i2 - py;
      const double Z = geo.h[2] * i0 + geo.h[5] * i1 + geo.h[8] * i2 - pz;
      const double r2 = X * X + Y * Y + Z * Z;
      const double rr = sqrt(r2);
      Acc av;
      if constexpr (CPLX) {
        const T v = a_xG[x * l.nG + G];
        av = make_double2((double)v.x * pr - (double)v.y * pi, (double)v.x * pi + (double)v.y * pr);
      } else {
        av = (double)a_xG[x * l.nG + G];
      }
      // per function: f, df/dr once, then every m
      const double* coef_prev = nullptr;
      double f = 0.0, df = 0.0;
      double Yl[5], dY[15];
      for (int k = 0; k < nm && k < 16; ++k) {
        const SplineM sm = spl[M0 + k];
        if (sm.s.coef != coef_prev || sm.m == 0) {
          spline_eval(sm.s, rr, f, df);
          const double fr = rr > 1e-15 ? df / rr : 0.0;
          solid_harmonics(sm.s.l, fr, X, Y, Z, r2, Yl);        // (df/dr / r) r^l Y_lm
          solid_harmonics_gradient(sm.s.l, f, X, Y, Z, dY);    // f d(r^l Y_lm)/dr_v
          coef_prev = sm.s.coef;
        }
        const double d0 = dY[3 * sm.m] + Yl[sm.m] * X;
        const double d1 = dY[3 * sm.m + 1] + Yl[sm.m] * Y;
        const double d2 = dY[3 * sm.m + 2] + Yl[sm.m] * Z;
#pragma unroll
        for (int kk = 0; kk < 16; ++kk)
          if (kk == k) {
            if constexpr (CPLX) {
              acc[3 * kk] = make_double2(acc[3 * kk].x + av.x * d0, acc[3 * kk].y + av.y * d0);
              acc[3 * kk + 1] = make_double2(acc[3 * kk + 1].x + av.x * d1, acc[3 * kk + 1].y + av.y * d1);
              acc[3 * kk + 2] = make_double2(acc[3 * kk + 2].x + av.x * d2, acc[3 * kk + 2].y + av.y * d2);
            } else {
              acc[3 * kk] += av * d0;
              acc[3 * kk + 1] += av * d1;
              acc[3 * kk + 2] += av * d2;
            }
          }
      }
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < NMV; ++i) {
    Acc v = acc[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      if constexpr (CPLX) {
        v.x += __shfl_down_sync(0xffffffffu, v.x, o);
        v.y += __shfl_down_sync(0xffffffffu, v.y, o);
      } else {
        v += __shfl_down_sync(0xffffffffu, v, o);
      }
    }
    if (lane == 0) red[warp][i] = v;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 3 * nm && e < NMV; e += NT) {
    Acc v = zero<Acc>();
    for (int w = 0; w < NT / 32; ++w) v = add(v, red[w][e]);
    T* cp = c_xMv + (x * l.nM + M0) * 3 + e;
    if constexpr (CPLX) {
      cp->x += (typename Elem<T>::R)(v.x * l.dv);
      cp->y += (typename Elem<T>::R)(v.y * l.dv);
    } else {
      *cp += (T)(v * l.dv);
    }
  }
}

template <typename T>
static int derivative_t(const gb_lfc* l, const SplineM* spl, const double* pos, const DerivGeom& geo,
                        const void* a, void* c, int64_t nx, int q, cudaStream_t st) {
  if (l->ngroups == 0) return GB_OK;
  const dim3 grid((unsigned)l->ngroups, (unsigned)nx);
  lfc_derivative_kernel<T><<<grid, 128, 0, st>>>(view(l), spl, pos, geo, static_cast<const T*>(a),
                                                 static_cast<T*>(c), q);
  return check_launch("lfc_derivative_kernel");
}

}  // namespace gb

using namespace gb;

extern "C" {

int gb_lfc_free(gb_lfc* l) {
  if (!l) return GB_OK;
  if (l->work) cudaFree(l->work);
  for (void* p : l->allocations) cudaFree(p);
  delete l;
  return GB_OK;
}

int gb_lfc_new(int nW, const double* A_all, const int64_t* ngm_W, const int* nm_W, const int* M_W, int nB,
               const int* G_B, const int* W_B, double dv, int nq, const double* phase_qW, int64_t nG, int nM,
               gb_lfc** out) {
  GB_REQUIRE(out && nW >= 0 && nB >= 0 && nG > 0 && nM >= 0, "gb_lfc_new: bad arguments");
  GB_REQUIRE(nW == 0 || (A_all && ngm_W && nm_W && M_W && G_B && W_B), "gb_lfc_new: null pointer");
  GB_REQUIRE(nq == 0 || phase_qW, "gb_lfc_new: phases missing");
  GB_REQUIRE(nG < (int64_t)1 << 31, "gb_lfc_new: grid too large for 32-bit point indices");
  auto* l = new (std::nothrow) gb_lfc();
  if (!l) return fail(GB_E_NOMEM, "gb_lfc_new: out of host memory");
  l->nW = nW; l->nG = nG; l->nM = nM; l->dv = dv; l->nq = nq;
  // global row / A offsets per volume
  std::vector<int64_t> row0(nW + 1, 0), aoff(nW + 1, 0);
  for (int W = 0; W < nW; ++W) {
    if (nm_W[W] < 1 || ngm_W[W] < 0 || M_W[W] < 0 || M_W[W] + nm_W[W] > nM) {
      gb_lfc_free(l);
      return fail(GB_E_INVALID, "gb_lfc_new: bad volume description");
    }
    row0[W + 1] = row0[W] + ngm_W[W];
    aoff[W + 1] = aoff[W] + ngm_W[W] * nm_W[W];
    l->maxnm = std::max(l->maxnm, nm_W[W]);
  }
  // GRID_LOOP sweep (c/lfc.h:79-130): the rows of a volume are consumed in
  // increasing G over the runs in which it is current.
  std::vector<int> row_G(row0[nW]);
  std::vector<int64_t> next_row(row0.begin(), row0.end() - 1);
  std::vector<int> cur;                 // current volumes
  std::vector<int> pos_in_cur(nW, -1);
  std::vector<int> pt_G, pt_off(1, 0);
  std::vector<int64_t> ct_aoff;
  std::vector<int> ct_M, ct_nm, ct_W;
  int Ga = 0;
  for (int B = 0; B < nB; ++B) {
    const int Gb = G_B[B];
    if (Gb < Ga || Gb > nG) {
      gb_lfc_free(l);
      return fail(GB_E_INVALID, "gb_lfc_new: boundary list not sorted or out of range");
    }
    if (Gb > Ga && !cur.empty()) {
      for (int G = Ga; G < Gb; ++G) {
        pt_G.push_back(G);
        for (int W : cur) {
          const int64_t r = next_row[W]++;
          if (r >= row0[W + 1]) {
            gb_lfc_free(l);
            return fail(GB_E_INVALID, "gb_lfc_new: boundaries cover more points than a volume has rows");
          }
          row_G[r] = G;
          ct_aoff.push_back(aoff[W] + (r - row0[W]) * nm_W[W]);
          ct_M.push_back(M_W[W]);
          ct_nm.push_back(nm_W[W]);
          ct_W.push_back(W);
        }
        pt_off.push_back((int)ct_W.size());
      }
    }
    const int Wn = W_B[B];
    if (Wn >= 0) {
      if (Wn >= nW || pos_in_cur[Wn] >= 0) {
        gb_lfc_free(l);
        return fail(GB_E_INVALID, "gb_lfc_new: bad volume entry");
      }
      pos_in_cur[Wn] = (int)cur.size();
      cur.push_back(Wn);
    } else {
      const int Wo = -1 - Wn;
      if (Wo >= nW || pos_in_cur[Wo] < 0) {
        gb_lfc_free(l);
        return fail(GB_E_INVALID, "gb_lfc_new: volume leaves before entering");
      }
      const int i = pos_in_cur[Wo];
      cur[i] = cur.back();
      pos_in_cur[cur[i]] = i;
      cur.pop_back();
      pos_in_cur[Wo] = -1;
    }
    Ga = Gb;
  }
  for (int W = 0; W < nW; ++W)
    if (next_row[W] != row0[W + 1]) {
      gb_lfc_free(l);
      return fail(GB_E_INVALID, "gb_lfc_new: volume rows and boundary runs disagree");
    }
  // function groups: volumes sharing (M, nm), ordered by nm for per-class launches
  std::map<std::pair<int, int>, std::vector<int>> groups;   // (nm, M) -> volumes
  for (int W = 0; W < nW; ++W) groups[{nm_W[W], M_W[W]}].push_back(W);
  std::vector<int> gr_M, gr_nm, gr_voff(1, 0), gv_W;
  for (auto& kv : groups) {
    gr_nm.push_back(kv.first.first);
    gr_M.push_back(kv.first.second);
    for (int W : kv.second) gv_W.push_back(W);
    gr_voff.push_back((int)gv_W.size());
  }
  // zero-padded A rows in contribution order for the all-band real add
  std::vector<double> hAc;
  if (l->maxnm <= 16) {
    const int F = l->maxnm <= 8 ? 8 : 16;
    l->fast_nmax = F;
    bool full32 = nM % 4 == 0, full64 = nM % 2 == 0;
    hAc.assign(ct_aoff.size() * F, 0.0);
    for (size_t c = 0; c < ct_aoff.size(); ++c) {
      for (int m = 0; m < ct_nm[c]; ++m) hAc[c * F + m] = A_all[ct_aoff[c] + m];
      full32 = full32 && ct_nm[c] == F && ct_M[c] % 4 == 0;
      full64 = full64 && ct_nm[c] == F && ct_M[c] % 2 == 0;
    }
    l->full32 = full32;
    l->full64 = full64;
  }
  // brick tiling for the FP32 real path
  std::vector<int> tch_c, tch_eoff, te_nm, te_slot, te_lst, te_info, tbr_ch0, tbr_pbase, tps_M, tps_nm, tps_eoff,
      tps_info, tgr_poff, tgr_pidx;
  std::vector<float> te_A;
  int tbr_smax = 1, tbr_emax = 0;
  bool tiled = l->maxnm <= 8 && nG % 4 == 0 && nW > 0;
  if (tiled) {
    const int ngr = (int)gr_M.size();
    std::vector<int> vol_group(nW);
    for (int gi = 0; gi < ngr; ++gi)
      for (int v = gr_voff[gi]; v < gr_voff[gi + 1]; ++v) vol_group[gv_W[v]] = gi;
    // entries: (sub-tile, volume) with their blocks
    struct Ent { int64_t st; int W; int64_t blk; };
    std::vector<Ent> ents;
    std::vector<float> blocks;
    for (int W = 0; W < nW; ++W) {
      int64_t last = -1;
      for (int64_t r = row0[W]; r < row0[W + 1]; ++r) {
        const int64_t G = row_G[r];
        if (G / 8 != last) {
          last = G / 8;
          ents.push_back({last, W, (int64_t)(blocks.size() / 64)});
          blocks.resize(blocks.size() + 64, 0.f);
        }
        float* b = blocks.data() + ents.back().blk * 64;
        for (int m = 0; m < nm_W[W]; ++m)
          b[m * 8 + (int)(G % 8)] = (float)A_all[aoff[W] + (r - row0[W]) * nm_W[W] + m];
      }
    }
    std::sort(ents.begin(), ents.end(),
              [](const Ent& x, const Ent& y) { return x.st != y.st ? x.st < y.st : x.W < y.W; });
    std::vector<int> te_g;   // group of every entry
    tch_eoff.push_back(0);
    for (size_t i = 0; i < ents.size();) {
      const int64_t ch = ents[i].st / 4;
      tch_c.push_back((int)ch);
      for (int j = 0; j < 4; ++j) {
        for (; i < ents.size() && ents[i].st == ch * 4 + j; ++i) {
          te_nm.push_back(nm_W[ents[i].W]);
          te_g.push_back(vol_group[ents[i].W]);
          te_A.insert(te_A.end(), blocks.begin() + ents[i].blk * 64, blocks.begin() + ents[i].blk * 64 + 64);
        }
        tch_eoff.push_back((int)te_nm.size());
      }
    }
    const size_t ne = te_nm.size();
    te_slot.assign(ne, 0);
    te_lst.assign(ne, 0);
    // bricks: <= TBRICK consecutive chunks, <= TSLOTS groups, <= TBENT entries
    std::vector<int> slot_of(ngr, -1), brick_groups, newg;
    std::vector<std::vector<int>> group_parts(ngr);
    tbr_ch0.push_back(0);
    tbr_pbase.push_back(0);
    tps_eoff.push_back(0);
    auto close_brick = [&](int end_chunk) {
      const int b0 = tbr_ch0.back();
      const int E0 = tch_eoff[4 * b0], E1 = tch_eoff[4 * end_chunk];
      for (size_t k = 0; k < brick_groups.size(); ++k) {
        const int g = brick_groups[k];
        group_parts[g].push_back(tbr_pbase.back() + (int)k);
        tps_M.push_back(gr_M[g]);
        tps_nm.push_back(gr_nm[g]);
        for (int e = E0; e < E1; ++e)
          if (te_slot[e] == (int)k) tps_info.push_back((e - E0) | te_lst[e] << 16 | te_nm[e] << 24);
        tps_eoff.push_back((int)tps_info.size());
        slot_of[g] = -1;
      }
      tbr_smax = std::max(tbr_smax, (int)brick_groups.size());
      tbr_emax = std::max(tbr_emax, E1 - E0);
      tbr_pbase.push_back(tbr_pbase.back() + (int)brick_groups.size());
      tbr_ch0.push_back(end_chunk);
      brick_groups.clear();
    };
    auto chunk_groups = [&](size_t ci, bool only_new) {
      newg.clear();
      for (int e = tch_eoff[4 * ci]; e < tch_eoff[4 * ci + 4]; ++e) {
        const int g = te_g[e];
        if ((!only_new || slot_of[g] < 0) && std::find(newg.begin(), newg.end(), g) == newg.end()) newg.push_back(g);
      }
    };
    for (size_t ci = 0; ci < tch_c.size(); ++ci) {
      const int nent = tch_eoff[4 * ci + 4] - tch_eoff[4 * ci];
      chunk_groups(ci, true);
      const int in_brick = (int)ci - tbr_ch0.back();
      if (in_brick > 0 && (in_brick == TBRICK || brick_groups.size() + newg.size() > (size_t)TSLOTS ||
                           tch_eoff[4 * ci + 4] - tch_eoff[4 * tbr_ch0.back()] > TBENT)) {
        close_brick((int)ci);
        chunk_groups(ci, false);
      }
      if (newg.size() > (size_t)TSLOTS || nent > TBENT) {
        tiled = false;   // one chunk is too crowded: keep the point-major kernels
        break;
      }
      for (int g : newg) {
        slot_of[g] = (int)brick_groups.size();
        brick_groups.push_back(g);
      }
      const int kk = (int)ci - tbr_ch0.back();
      for (int j = 0; j < 4; ++j)
        for (int e = tch_eoff[4 * ci + j]; e < tch_eoff[4 * ci + j + 1]; ++e) {
          te_slot[e] = slot_of[te_g[e]];
          te_lst[e] = 4 * kk + j;
        }
    }
    if (tiled) {
      close_brick((int)tch_c.size());
      te_info.resize(ne);
      for (size_t e = 0; e < ne; ++e) te_info[e] = te_slot[e] | te_nm[e] << 8;
      tgr_poff.push_back(0);
      for (int gi = 0; gi < ngr; ++gi) {
        tgr_pidx.insert(tgr_pidx.end(), group_parts[gi].begin(), group_parts[gi].end());
        tgr_poff.push_back((int)tgr_pidx.size());
      }
    }
  }
  l->ngroups = (int)gr_M.size();
  l->h_gr_nm = gr_nm;
  l->P = (int64_t)pt_G.size();
  l->C = (int64_t)ct_W.size();
  l->nA = aoff[nW];
  std::vector<int64_t> vr0(row0.begin(), row0.end() - 1), vr1(row0.begin() + 1, row0.end());
  std::vector<int64_t> va(aoff.begin(), aoff.end() - 1);
  std::vector<double> hA(A_all, A_all + l->nA);
  std::vector<double2> ph;
  for (int64_t i = 0; i < (int64_t)nq * nW; ++i) ph.push_back(make_double2(phase_qW[2 * i], phase_qW[2 * i + 1]));
  bool ok = upload(l, &l->A64, hA) && upload(l, &l->pt_G, pt_G) && upload(l, &l->pt_off, pt_off) &&
            upload(l, &l->ct_aoff, ct_aoff) && upload(l, &l->ct_M, ct_M) && upload(l, &l->ct_nm, ct_nm) &&
            upload(l, &l->ct_W, ct_W) && upload(l, &l->gr_M, gr_M) && upload(l, &l->gr_nm, gr_nm) &&
            upload(l, &l->gr_voff, gr_voff) && upload(l, &l->gv_W, gv_W) && upload(l, &l->vol_row0, vr0) &&
            upload(l, &l->vol_row1, vr1) && upload(l, &l->row_G, row_G) && upload(l, &l->vol_aoff, va) &&
            upload(l, &l->phase, ph);
  if (ok) {
    l->A32 = dalloc<float>(l, l->nA);
    ok = l->A32 != nullptr;
    if (ok && l->nA) {
      to_float<<<std::min<int64_t>((l->nA + 255) / 256, 4096), 256>>>(l->A64, l->A32, l->nA);
      ok = cudaDeviceSynchronize() == cudaSuccess;
    }
  }
  if (ok && l->fast_nmax) {
    ok = upload(l, &l->Ac64, hAc);
    if (ok) {
      l->Ac32 = dalloc<float>(l, hAc.size());
      ok = l->Ac32 != nullptr;
    }
    if (ok && !hAc.empty()) {
      to_float<<<std::min<int64_t>(((int64_t)hAc.size() + 255) / 256, 4096), 256>>>(l->Ac64, l->Ac32,
                                                                                      (int64_t)hAc.size());
      ok = cudaDeviceSynchronize() == cudaSuccess;
    }
  }
  if (ok && tiled) {
    ok = upload(l, &l->tch_c, tch_c) && upload(l, &l->tch_eoff, tch_eoff) && upload(l, &l->te_info, te_info) &&
         upload(l, &l->te_A, te_A) && upload(l, &l->tbr_ch0, tbr_ch0) && upload(l, &l->tbr_pbase, tbr_pbase) &&
         upload(l, &l->tps_M, tps_M) && upload(l, &l->tps_nm, tps_nm) && upload(l, &l->tps_eoff, tps_eoff) &&
         upload(l, &l->tps_info, tps_info) &&
         upload(l, &l->tgr_poff, tgr_poff) && upload(l, &l->tgr_pidx, tgr_pidx);
    l->tiled = ok;
    l->tbr_n = (int)tbr_ch0.size() - 1;
    l->tbr_smax = tbr_smax;
    l->tbr_emax = tbr_emax;
    l->tpart_n = tbr_pbase.back();
  }
  if (!ok) {
    gb_lfc_free(l);
    return fail(GB_E_NOMEM, "gb_lfc_new: device allocation / upload failed");
  }
  *out = l;
  return GB_OK;
}

int gb_lfc_tiled(const gb_lfc* l) { return l && l->tiled ? 1 : 0; }

int gb_lfc_add(const gb_lfc* l, const void* c_xM, void* a_xG, int64_t nx, int dtype, int q, void* stream) {
  GB_REQUIRE(l && dtype_valid(dtype) && nx >= 0, "gb_lfc_add: bad arguments");
  if (nx == 0) return GB_OK;
  GB_REQUIRE(c_xM && a_xG, "gb_lfc_add: null array");
  GB_REQUIRE(q < l->nq, "gb_lfc_add: k-point index out of range");
  cudaStream_t st = (cudaStream_t)stream;
  switch (dtype) {
    case GB_DTYPE_F64: return add_t<double>(l, c_xM, a_xG, nx, -1, st);
    case GB_DTYPE_F32: return add_t<float>(l, c_xM, a_xG, nx, -1, st);
    case GB_DTYPE_C128: return add_t<double2>(l, c_xM, a_xG, nx, q, st);
    default: return add_t<float2>(l, c_xM, a_xG, nx, q, st);
  }
}

int gb_lfc_integrate(const gb_lfc* l, const void* a_xG, void* c_xM, int64_t nx, int dtype, int q, void* stream) {
  GB_REQUIRE(l && dtype_valid(dtype) && nx >= 0, "gb_lfc_integrate: bad arguments");
  if (nx == 0) return GB_OK;
  GB_REQUIRE(c_xM && a_xG, "gb_lfc_integrate: null array");
  GB_REQUIRE(q < l->nq, "gb_lfc_integrate: k-point index out of range");
  cudaStream_t st = (cudaStream_t)stream;
  switch (dtype) {
    case GB_DTYPE_F64: return integrate_t<double>(l, a_xG, c_xM, nx, -1, st);
    case GB_DTYPE_F32: return integrate_t<float>(l, a_xG, c_xM, nx, -1, st);
    case GB_DTYPE_C128: return integrate_t<double2>(l, a_xG, c_xM, nx, q, st);
    default: return integrate_t<float2>(l, a_xG, c_xM, nx, q, st);
  }
}

int gb_lfc_add_k(const gb_lfc* l, const void* c_xM, void* a_xG, int64_t nx, int dtype, int nk, void* stream) {
  GB_REQUIRE(l && dtype_valid(dtype) && nx >= 0, "gb_lfc_add_k: bad arguments");
  GB_REQUIRE(dtype_complex(dtype), "gb_lfc_add_k: k-point batches are complex");
  GB_REQUIRE(nk >= 1 && nk <= l->nq && nx % nk == 0, "gb_lfc_add_k: nk must divide the batch and be <= nq");
  if (nx == 0) return GB_OK;
  GB_REQUIRE(c_xM && a_xG, "gb_lfc_add_k: null array");
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t per = nx / nk;
  if (dtype == GB_DTYPE_C128) return add_t<double2>(l, c_xM, a_xG, nx, 0, st, per);
  return add_t<float2>(l, c_xM, a_xG, nx, 0, st, per);
}

int gb_lfc_integrate_k(const gb_lfc* l, const void* a_xG, void* c_xM, int64_t nx, int dtype, int nk,
                       void* stream) {
  GB_REQUIRE(l && dtype_valid(dtype) && nx >= 0, "gb_lfc_integrate_k: bad arguments");
  GB_REQUIRE(dtype_complex(dtype), "gb_lfc_integrate_k: k-point batches are complex");
  GB_REQUIRE(nk >= 1 && nk <= l->nq && nx % nk == 0,
             "gb_lfc_integrate_k: nk must divide the batch and be <= nq");
  if (nx == 0) return GB_OK;
  GB_REQUIRE(c_xM && a_xG, "gb_lfc_integrate_k: null array");
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t per = nx / nk;
  if (dtype == GB_DTYPE_C128) return integrate_t<double2>(l, a_xG, c_xM, nx, 0, st, per);
  return integrate_t<float2>(l, a_xG, c_xM, nx, 0, st, per);
}

int gb_lfc_derivative(const gb_lfc* l, const void* a_xG, void* c_xMv, int64_t nx, const double h_cv[9],
                      const int64_t n_c[3], const gb_spline* const* spline_M, const int64_t beg_c[3],
                      const double* pos_Wv, int q, int dtype, void* stream) {
  GB_REQUIRE(l && dtype_valid(dtype) && nx >= 0, "gb_lfc_derivative: bad arguments");
  if (nx == 0 || l->nM == 0) return GB_OK;
  GB_REQUIRE(a_xG && c_xMv && h_cv && n_c && beg_c && pos_Wv && spline_M, "gb_lfc_derivative: null argument");
  GB_REQUIRE(q < l->nq, "gb_lfc_derivative: k-point index out of range");
  GB_REQUIRE(nx < 65536, "gb_lfc_derivative: at most 65535 grids per call");
  GB_REQUIRE(n_c[0] * n_c[1] * n_c[2] == l->nG, "gb_lfc_derivative: grid size does not match the object");
  for (int g = 0; g < l->ngroups; ++g)
    if (l->h_gr_nm[g] > 16) return fail(GB_E_UNSUPPORTED, "gb_lfc_derivative: more than 16 functions in a volume");
  // per M: the spline and its m index (m runs 0 .. 2l across consecutive
  // entries of one function, as the reference's spline_M list repeats each
  // function's spline 2l + 1 times)
  std::vector<SplineM> hs(l->nM);
  for (int M = 0; M < l->nM; ++M) {
    const gb_spline* sp = spline_M[M];
    if (!sp) return fail(GB_E_INVALID, "gb_lfc_derivative: null spline in spline_M");
    const int nmf = 2 * sp->l + 1;
    int m = 0;
    if (M > 0 && spline_M[M - 1] == sp && hs[M - 1].m + 1 < nmf) m = hs[M - 1].m + 1;
    hs[M] = SplineM{spline_view(sp), m};
  }
  DerivGeom geo;
  for (int c = 0; c < 3; ++c) {
    geo.n[c] = n_c[c];
    geo.beg[c] = beg_c[c];
  }
  for (int i = 0; i < 9; ++i) geo.h[i] = h_cv[i];
  cudaStream_t st = (cudaStream_t)stream;
  void* work = nullptr;
  const size_t sbytes = hs.size() * sizeof(SplineM), pbytes = (size_t)l->nW * 3 * sizeof(double);
  if (cudaMallocAsync(&work, sbytes + pbytes + 16, st) != cudaSuccess)
    return fail(GB_E_NOMEM, "gb_lfc_derivative: work space allocation failed");
  SplineM* d_spl = static_cast<SplineM*>(work);
  double* d_pos = reinterpret_cast<double*>(static_cast<char*>(work) + (sbytes + 15) / 16 * 16);
  int rc = GB_OK;
  if (cudaMemcpyAsync(d_spl, hs.data(), sbytes, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(d_pos, pos_Wv, pbytes, cudaMemcpyHostToDevice, st) != cudaSuccess)
    rc = fail(GB_E_CUDA, "gb_lfc_derivative: upload failed");
  if (!rc) {
    switch (dtype) {
      case GB_DTYPE_F64: rc = derivative_t<double>(l, d_spl, d_pos, geo, a_xG, c_xMv, nx, -1, st); break;
      case GB_DTYPE_F32: rc = derivative_t<float>(l, d_spl, d_pos, geo, a_xG, c_xMv, nx, -1, st); break;
      case GB_DTYPE_C128: rc = derivative_t<double2>(l, d_spl, d_pos, geo, a_xG, c_xMv, nx, q, st); break;
      default: rc = derivative_t<float2>(l, d_spl, d_pos, geo, a_xG, c_xMv, nx, q, st); break;
    }
  }
  cudaFreeAsync(work, st);
  // the host vectors above were read by the copies: finish them before return
  if (cudaStreamSynchronize(st) != cudaSuccess && !rc) rc = fail(GB_E_CUDA, "gb_lfc_derivative: sync failed");
  return rc;
}

}  // extern "C"
