// Per-band inner products of RMM-DIIS (gpaw/eigensolvers/rmmdiis.py:
// 133-145, 175-190: <R|R>, <dR|R>, <dR|dR> and the DIIS matrix
// <R_i|R_j> over the stored residuals), all bands per launch.
//
//   gb_band_dots:  out[n]       = Re sum_G conj(a[n,G]) b[n,G]
//   gb_band_gram:  out[n][i][j] = Re sum_G conj(X[n,i,G]) X[n,j,G], i,j < k
//
// One CTA of 1024 threads per band streams the band's grid points once with
// 16-byte loads and accumulates in FP64 whatever the storage precision (the
// sums feed FP64 line searches and DIIS solves); a fixed-order block
// reduction keeps results deterministic.  HBM-bound: bytes = inputs read
// once.
#include <algorithm>
#include "internal.cuh"

namespace gb {

template <typename T>
__device__ __forceinline__ double redot(const T& a, const T& b);
template <> __device__ __forceinline__ double redot(const double& a, const double& b) { return a * b; }
template <> __device__ __forceinline__ double redot(const float& a, const float& b) { return (double)a * (double)b; }
template <> __device__ __forceinline__ double redot(const double2& a, const double2& b) { return a.x * b.x + a.y * b.y; }
template <> __device__ __forceinline__ double redot(const float2& a, const float2& b) {
  return (double)a.x * b.x + (double)a.y * b.y;
}

constexpr int BT = 1024;

// sum over the CTA of NV values per thread, result in out[0..NV) of thread 0
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* out) {
  __shared__ double red[BT / 32][NV];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double x = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[warp][k] = x;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0.0;
    for (int w = 0; w < BT / 32; ++w) s += red[w][threadIdx.x];
    out[threadIdx.x] = s;
  }
}

template <typename T>
__global__ void __launch_bounds__(BT) band_dots_kernel(const T* __restrict__ a, const T* __restrict__ b,
                                                       int64_t lda, int64_t ldb, int64_t N,
                                                       double* __restrict__ out) {
  constexpr int VEC = 16 / (int)sizeof(T);
  const int64_t n = blockIdx.x;
  const T* pa = a + n * lda;
  const T* pb = b + n * ldb;
  double acc[1] = {0.0};
  const bool vec = ((reinterpret_cast<uintptr_t>(pa) | reinterpret_cast<uintptr_t>(pb)) & 15) == 0;
  int64_t done = 0;
  if (vec) {
    const int64_t nv = N / VEC;
    const float4* va = reinterpret_cast<const float4*>(pa);
    const float4* vb = reinterpret_cast<const float4*>(pb);
    for (int64_t i = threadIdx.x; i < nv; i += BT) {
      const float4 x = __ldcs(va + i), y = __ldcs(vb + i);
      const T* ex = reinterpret_cast<const T*>(&x);
      const T* ey = reinterpret_cast<const T*>(&y);
#pragma unroll
      for (int k = 0; k < VEC; ++k) acc[0] += redot(ex[k], ey[k]);
    }
    done = nv * VEC;
  }
  for (int64_t i = done + threadIdx.x; i < N; i += BT) acc[0] += redot(pa[i], pb[i]);
  block_sum<1>(acc, out + n);
}

template <typename T, int K>
__global__ void __launch_bounds__(BT) band_gram_kernel(const T* __restrict__ X, int64_t ldn, int64_t ldi,
                                                       int64_t N, double* __restrict__ out) {
  constexpr int NP = K * (K + 1) / 2;
  const int64_t n = blockIdx.x;
  double acc[NP];
#pragma unroll
  for (int p = 0; p < NP; ++p) acc[p] = 0.0;
  const T* base = X + n * ldn;
  for (int64_t g = threadIdx.x; g < N; g += BT) {
    T x[K];
#pragma unroll
    for (int i = 0; i < K; ++i) x[i] = base[i * ldi + g];
    int p = 0;
#pragma unroll
    for (int i = 0; i < K; ++i)
#pragma unroll
      for (int j = i; j < K; ++j) acc[p++] += redot(x[i], x[j]);
  }
  __shared__ double tri[NP];
  block_sum<NP>(acc, tri);
  __syncthreads();
  if (threadIdx.x < K * K) {
    const int i = threadIdx.x / K, j = threadIdx.x % K;
    const int lo = i < j ? i : j, hi = i < j ? j : i;
    const int p = lo * K - lo * (lo - 1) / 2 + (hi - lo);
    out[n * K * K + threadIdx.x] = tri[p];
  }
}

template <typename T>
static int gram_t(const void* X, int64_t nb, int k, int64_t ldn, int64_t ldi, int64_t N, double* out,
                  cudaStream_t st) {
  const T* x = static_cast<const T*>(X);
  switch (k) {
    case 1: band_gram_kernel<T, 1><<<(unsigned)nb, BT, 0, st>>>(x, ldn, ldi, N, out); break;
    case 2: band_gram_kernel<T, 2><<<(unsigned)nb, BT, 0, st>>>(x, ldn, ldi, N, out); break;
    case 3: band_gram_kernel<T, 3><<<(unsigned)nb, BT, 0, st>>>(x, ldn, ldi, N, out); break;
    case 4: band_gram_kernel<T, 4><<<(unsigned)nb, BT, 0, st>>>(x, ldn, ldi, N, out); break;
    case 5: band_gram_kernel<T, 5><<<(unsigned)nb, BT, 0, st>>>(x, ldn, ldi, N, out); break;
    default: return fail(GB_E_UNSUPPORTED, "gb_band_gram: k must be 1..5");
  }
  return check_launch("band_gram_kernel");
}

}  // namespace gb

using namespace gb;

extern "C" {

int gb_band_dots(int64_t nb, int64_t N, const void* a, int64_t lda, const void* b, int64_t ldb, int dtype,
                 double* out, void* stream) {
  GB_REQUIRE(nb >= 0 && N >= 0 && dtype_valid(dtype), "gb_band_dots: bad arguments");
  if (nb == 0) return GB_OK;
  GB_REQUIRE(a && b && out && lda >= N && ldb >= N, "gb_band_dots: null array or bad stride");
  GB_REQUIRE(nb < (int64_t)1 << 31, "gb_band_dots: too many bands");
  cudaStream_t st = (cudaStream_t)stream;
  switch (dtype) {
    case GB_DTYPE_F64:
      band_dots_kernel<double><<<(unsigned)nb, BT, 0, st>>>((const double*)a, (const double*)b, lda, ldb, N, out);
      break;
    case GB_DTYPE_F32:
      band_dots_kernel<float><<<(unsigned)nb, BT, 0, st>>>((const float*)a, (const float*)b, lda, ldb, N, out);
      break;
    case GB_DTYPE_C128:
      band_dots_kernel<double2><<<(unsigned)nb, BT, 0, st>>>((const double2*)a, (const double2*)b, lda, ldb, N, out);
      break;
    default:
      band_dots_kernel<float2><<<(unsigned)nb, BT, 0, st>>>((const float2*)a, (const float2*)b, lda, ldb, N, out);
  }
  return check_launch("band_dots_kernel");
}

int gb_band_gram(int64_t nb, int k, int64_t N, const void* X, int64_t ldn, int64_t ldi, int dtype, double* out,
                 void* stream) {
  GB_REQUIRE(nb >= 0 && N >= 0 && k >= 1 && dtype_valid(dtype), "gb_band_gram: bad arguments");
  if (nb == 0) return GB_OK;
  // the k vectors of every band must not overlap: band-major (each band's
  // vectors side by side) or vector-major (each vector's bands side by side)
  const bool band_major = ldi >= N && ldn >= (int64_t)k * ldi - (ldi - N);
  const bool vec_major = ldn >= N && ldi >= nb * ldn - (ldn - N);
  GB_REQUIRE(X && out && (band_major || vec_major), "gb_band_gram: null array or bad stride");
  GB_REQUIRE(nb < (int64_t)1 << 31, "gb_band_gram: too many bands");
  cudaStream_t st = (cudaStream_t)stream;
  switch (dtype) {
    case GB_DTYPE_F64: return gram_t<double>(X, nb, k, ldn, ldi, N, out, st);
    case GB_DTYPE_F32: return gram_t<float>(X, nb, k, ldn, ldi, N, out, st);
    case GB_DTYPE_C128: return gram_t<double2>(X, nb, k, ldn, ldi, N, out, st);
    default: return gram_t<float2>(X, nb, k, ldn, ldi, N, out, st);
  }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Small dense solves of the DIIS steps (the bordered <R_i|R_j> system of
// gpaw/eigensolvers/rmmdiis.py:175-190, one per band, and the Pulay mixer's
// system): nb independent n x n FP64 systems, n <= 8, Gaussian elimination
// with partial pivoting, one thread per system, no host synchronisation (a
// singular system sets info[s] = 1 and leaves x[s] = 0).
namespace gb {

constexpr int SMALL_N = 8;

__global__ void small_solve_kernel(int64_t nb, int n, const double* __restrict__ A, const double* __restrict__ b,
                                   double* __restrict__ x, int* __restrict__ info) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= nb) return;
  double M[SMALL_N][SMALL_N + 1];
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j) M[i][j] = A[(s * n + i) * n + j];
    M[i][n] = b[s * n + i];
  }
  double amax = 0.0;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) amax = fmax(amax, fabs(M[i][j]));
  int bad = !(amax > 0.0) || !isfinite(amax);
  for (int k = 0; k < n && !bad; ++k) {
    int p = k;
    for (int i = k + 1; i < n; ++i)
      if (fabs(M[i][k]) > fabs(M[p][k])) p = i;
    if (!(fabs(M[p][k]) > 0.0)) {   // exactly singular, as LAPACK's getrf reports it
      bad = 1;
      break;
    }
    if (p != k)
      for (int j = k; j <= n; ++j) {
        const double t = M[k][j];
        M[k][j] = M[p][j];
        M[p][j] = t;
      }
    for (int i = k + 1; i < n; ++i) {
      const double f = M[i][k] / M[k][k];
      for (int j = k; j <= n; ++j) M[i][j] -= f * M[k][j];
    }
  }
  if (!bad) {
    for (int i = n - 1; i >= 0; --i) {
      double t = M[i][n];
      for (int j = i + 1; j < n; ++j) t -= M[i][j] * M[j][n];
      M[i][n] = t / M[i][i];
      if (!isfinite(M[i][n])) bad = 1;
    }
  }
  for (int i = 0; i < n; ++i) x[s * n + i] = bad ? 0.0 : M[i][n];
  if (info) info[s] = bad;
}

}  // namespace gb

extern "C" int gb_small_solve(int64_t nb, int n, const double* A, const double* b, double* x, int* info,
                              void* stream) {
  GB_REQUIRE(nb >= 0 && n >= 1 && n <= gb::SMALL_N, "gb_small_solve: need 1 <= n <= 8");
  if (nb == 0) return GB_OK;
  GB_REQUIRE(A && b && x, "gb_small_solve: null array");
  const int T = 128;
  gb::small_solve_kernel<<<(unsigned)((nb + T - 1) / T), T, 0, (cudaStream_t)stream>>>(nb, n, A, b, x, info);
  return check_launch("small_solve_kernel");
}

// ---------------------------------------------------------------------------
// Per-band linear combinations of RMM-DIIS (gpaw/eigensolvers/rmmdiis.py:
// 150-200: R -= eps psi, psi += lambda dpsi, R += lambda dR, and the DIIS
// recombinations psi = sum_i alpha_i psi_i, R = sum_i alpha_i R_i):
//   out[n*ldo + G] = sum_{i<k} coef[n*k + i] * x_i[n*ldx_i + G],   k <= 4,
// coefficients FP64 on the device (rounded to the working precision), one
// launch for all bands; out may be one of the inputs (element-wise update).
namespace gb {

constexpr int COMB_MAX = 4;
struct CombArgs {
  const void* x[COMB_MAX];
  int64_t ldx[COMB_MAX];
  void* out;
  int64_t ldo;
  int64_t N;
  int k;
  const double* coef;
};

template <typename T, int K>
__global__ void __launch_bounds__(256) band_combine_kernel(const CombArgs a) {
  using R = typename Elem<T>::R;
  constexpr int VEC = 16 / (int)sizeof(T);
  const int64_t n = blockIdx.y;
  R c[K];
#pragma unroll
  for (int i = 0; i < K; ++i) c[i] = (R)a.coef[n * K + i];
  const T* x[K];
#pragma unroll
  for (int i = 0; i < K; ++i) x[i] = static_cast<const T*>(a.x[i]) + n * a.ldx[i];
  T* o = static_cast<T*>(a.out) + n * a.ldo;
  bool vec = (reinterpret_cast<uintptr_t>(o) & 15) == 0;
#pragma unroll
  for (int i = 0; i < K; ++i) vec = vec && (reinterpret_cast<uintptr_t>(x[i]) & 15) == 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int64_t done = 0;
  if (vec) {
    const int64_t nv = a.N / VEC;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += stride) {
      T acc[VEC];
      {
        const float4 w = reinterpret_cast<const float4*>(x[0])[v];
        const T* e = reinterpret_cast<const T*>(&w);
#pragma unroll
        for (int j = 0; j < VEC; ++j) acc[j] = scale(c[0], e[j]);
      }
#pragma unroll
      for (int i = 1; i < K; ++i) {
        const float4 w = reinterpret_cast<const float4*>(x[i])[v];
        const T* e = reinterpret_cast<const T*>(&w);
#pragma unroll
        for (int j = 0; j < VEC; ++j) acc[j] = fmadd(acc[j], c[i], e[j]);
      }
      reinterpret_cast<float4*>(o)[v] = *reinterpret_cast<const float4*>(acc);
    }
    done = nv * VEC;
  }
  for (int64_t g = done + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < a.N; g += stride) {
    T acc = scale(c[0], x[0][g]);
#pragma unroll
    for (int i = 1; i < K; ++i) acc = fmadd(acc, c[i], x[i][g]);
    o[g] = acc;
  }
}

template <typename T>
static int combine_t(const CombArgs& a, int64_t nb, cudaStream_t st) {
  constexpr int VEC = 16 / (int)sizeof(T);
  const int64_t per_band = (a.N / VEC + 255) / 256;
  const int64_t want = std::max<int64_t>(1, (int64_t)sm_count() * 8 / std::max<int64_t>(nb, 1));
  dim3 grid((unsigned)std::max<int64_t>(1, std::min<int64_t>(per_band, want)), (unsigned)nb);
  switch (a.k) {
    case 1: band_combine_kernel<T, 1><<<grid, 256, 0, st>>>(a); break;
    case 2: band_combine_kernel<T, 2><<<grid, 256, 0, st>>>(a); break;
    case 3: band_combine_kernel<T, 3><<<grid, 256, 0, st>>>(a); break;
    default: band_combine_kernel<T, 4><<<grid, 256, 0, st>>>(a); break;
  }
  return check_launch("band_combine_kernel");
}

}  // namespace gb

extern "C" int gb_band_combine(int64_t nb, int64_t N, int k, const double* coef, const void* const* x,
                               const int64_t* ldx, void* out, int64_t ldo, int dtype, void* stream) {
  GB_REQUIRE(nb >= 0 && N >= 0 && k >= 1 && k <= gb::COMB_MAX && dtype_valid(dtype),
             "gb_band_combine: bad arguments (1 <= k <= 4)");
  if (nb == 0 || N == 0) return GB_OK;
  GB_REQUIRE(nb < 65536, "gb_band_combine: at most 65535 bands per call");
  GB_REQUIRE(coef && x && ldx && out && ldo >= N, "gb_band_combine: null array or bad stride");
  gb::CombArgs a{};
  for (int i = 0; i < k; ++i) {
    GB_REQUIRE(x[i] && ldx[i] >= N, "gb_band_combine: null input or bad stride");
    a.x[i] = x[i];
    a.ldx[i] = ldx[i];
  }
  a.out = out; a.ldo = ldo; a.N = N; a.k = k; a.coef = coef;
  cudaStream_t st = (cudaStream_t)stream;
  switch (dtype) {
    case GB_DTYPE_F64: return gb::combine_t<double>(a, nb, st);
    case GB_DTYPE_F32: return gb::combine_t<float>(a, nb, st);
    case GB_DTYPE_C128: return gb::combine_t<double2>(a, nb, st);
    default: return gb::combine_t<float2>(a, nb, st);
  }
}
