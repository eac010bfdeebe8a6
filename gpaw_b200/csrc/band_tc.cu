// Band-space GEMMs of the eigensolver on the 5th-generation tensor cores
// (tcgen05, sm_100a) for FP32 wave functions:
//
//   gram    C[i][j] = alpha sum_G A[i][G] B[j][G]          FP64 result
//           the overlap S_nn = dv psi psi^T (gpaw/wavefunctions/fdpw.py:
//           394-424) and H_nn = dv psi^T (T + v) psi (gpaw/eigensolvers/
//           eigensolver.py:174-236)
//   rotate  Y[n][G] = sum_k U[n][k] X[k][G] (+ beta Z[n][G])  FP32 in and out
//           psi <- U psi of the subspace rotation and of the Cholesky
//           orthonormalisation (the same files)
//
// FP32 accuracy from TF32 tensor cores by the three-product split: every
// operand value x is written as hi + lo with hi = RN_tf32(x) and
// lo = RN_tf32(x - hi), both exact TF32 numbers (so the tensor core's own
// input conversion loses nothing), and a b ~ hi_a hi_b + hi_a lo_b + lo_a hi_b;
// the dropped lo_a lo_b term and the rounding of lo stay below 2^-22 relative
// per product.  Products accumulate in FP32 in tensor memory (TMEM) over one
// CTA's share of the sum; the gram partial sums are combined in FP64 in a
// fixed order (deterministic).  The tensor core's FP32 additions truncate,
// so a long sum shrinks by about half an ulp per MMA (~1e-6 relative for a
// 160-band rotation); the Z term lets a caller rotate by U - I and add X back
// exactly (psi + (U - I) psi), which confines that bias to the correction.
//
// Both kernels are warp-specialised, one CTA per SM:
//   warp 0      TMA producer: 32-column tiles (128-byte rows, 128-byte
//               swizzle) of A/B (gram) or of X and the pre-split U (rotate)
//               into a ring of NS stages, completion on mbarriers
//   warp 1      TMEM allocation and the MMA issuer (one thread):
//               tcgen05.mma.cta_group::1.kind::tf32, M = 128, N = NT <= 256,
//               K = 8 per instruction, three per k-step; tcgen05.commit hands
//               a stage back to the producer once its MMAs are done
//   splitters   gram: warps 4-11, rotate: warps 4-7; read a landed
//               stage, write hi in place and lo beside it, fence the
//               generic-proxy writes for the tensor core
//   epilogue    tcgen05.ld of the accumulator (32 lanes x 16 columns per
//               load; warp w reads TMEM lanes 32 (w % 4) ..): gram -> FP64
//               partials (warps 4-7 after their last stage), rotate -> Y with
//               a warp's stores along 32 consecutive grid points (warps 8-11,
//               TMEM double-buffered so the next tile's MMAs overlap; the
//               optional Z term is loaded a chunk ahead)
// Operand layouts (shared-memory matrix descriptors, 128-byte swizzle):
//   gram A, B and rotate U are K-major (rows of 32 FP32 along the sum
//   index; 8-row groups 1024 bytes apart; a k-step of 8 advances 32 bytes);
//   rotate X is MN-major (rows of 32 grid points per band, 128-byte swizzle
//   of 32-byte units -- the MN-major layout of the TF32 MMA; 4-band groups
//   512 bytes apart, 4 boxes of 32 points 4096 bytes apart; a k-step of 8
//   bands advances 1024 bytes).
// Every wait is bounded (tma.cuh); a timed-out wait records an error code,
// raises a CTA-wide abort flag and the CTA drains its own TMA copies and
// MMAs (bounded) and frees its TMEM before it returns.
#include <algorithm>
#include <cstring>
#include <cudaTypedefs.h>
#include "internal.cuh"
#include "tma.cuh"
#include "tcgen05.cuh"

namespace gb {

__device__ int g_tc_error = 0;

int band_tc_error_flag(int clear) {
  int v = 0;
  cudaMemcpyFromSymbol(&v, g_tc_error, sizeof(int));
  if (clear && v) {
    int z = 0;
    cudaMemcpyToSymbol(g_tc_error, &z, sizeof(int));
  }
  return v;
}

namespace {

using namespace tc;

__device__ __forceinline__ void split4(float4& v, float4& lo) {
  float4 h;
  h.x = rn_tf32(v.x); h.y = rn_tf32(v.y); h.z = rn_tf32(v.z); h.w = rn_tf32(v.w);
  lo.x = rn_tf32(v.x - h.x); lo.y = rn_tf32(v.y - h.y); lo.z = rn_tf32(v.z - h.z); lo.w = rn_tf32(v.w - h.w);
  v = h;
}

// split n4 float4 of a landed tile in place (hi) and into `lo`, NT threads,
// four independent 16-byte loads in flight per thread
template <int NT>
__device__ __forceinline__ void split_tile(uint8_t* hi_p, uint8_t* lo_p, int n4, int ct) {
  float4* h = reinterpret_cast<float4*>(hi_p);
  float4* l = reinterpret_cast<float4*>(lo_p);
  int i = ct;
  for (; i + 3 * NT < n4; i += 4 * NT) {
    float4 v[4], lo[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = h[i + k * NT];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      split4(v[k], lo[k]);
      h[i + k * NT] = v[k];
      l[i + k * NT] = lo[k];
    }
  }
  for (; i < n4; i += NT) {
    float4 v = h[i], lo;
    split4(v, lo);
    h[i] = v;
    l[i] = lo;
  }
}

// bounded wait that also gives up when another role of the CTA aborted
__device__ __forceinline__ bool tc_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag, int where) {
  for (long long i = 0; i < WAIT_LIMIT; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 255) == 255 && *abort_flag) return false;
  }
  *abort_flag = 1;
  atomicCAS(&g_tc_error, 0, where);
  return false;
}

constexpr int TM = 128;            // M tile (rows of A / grid points)
constexpr int KB = 32;             // FP32 elements per 128-byte row
constexpr uint32_t ATILE = TM * 128;   // bytes of a 128-row, 32-column tile

struct GramArgs {
  int na, nb, nkb;                 // rows of A, B; 32-point blocks of the sum
  int mtiles, ntiles, nsplit, NT, NS;
  uint32_t ncols;                  // TMEM columns allocated
  double* W;                       // partials [nsplit][na][nb]
};

struct RotArgs {
  int nn, nk;                      // rows of Y (= rows of U), rows of X
  int64_t K;                       // grid points
  int ptiles, ntiles, nkc, NT, NS;
  float* Y;
  int64_t ldy;
  const float* Z;                  // optional: Y += beta Z (Z shaped like Y)
  int64_t ldz;
  float beta;
};

// shared-memory carve-up shared by both kernels: NS stages of
// [X/A hi | X/A lo | B/U hi | B/U lo], then the barriers
struct Carve {
  uint8_t* base;
  uint32_t stage_bytes, b_bytes;
  __device__ uint8_t* ahi(int s) const { return base + (size_t)s * stage_bytes; }
  __device__ uint8_t* alo(int s) const { return ahi(s) + ATILE; }
  __device__ uint8_t* bhi(int s) const { return ahi(s) + 2 * ATILE; }
  __device__ uint8_t* blo(int s) const { return bhi(s) + b_bytes; }
};

__device__ __forceinline__ uint8_t* aligned_smem(uint8_t* p) {
  const uint32_t a = su32(p);
  return p + ((1024u - (a & 1023u)) & 1023u);
}

// ----------------------------------------------------------------- gram
__global__ void __launch_bounds__(384, 1)
    gram_tc_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                   const GramArgs g) {
  extern __shared__ uint8_t tc_smem_raw[];
  uint8_t* sm = aligned_smem(tc_smem_raw);
  const int NS = g.NS;
  Carve cv{sm, 2 * ATILE + 2u * (uint32_t)g.NT * 128u, (uint32_t)g.NT * 128u};
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + (size_t)NS * cv.stage_bytes);
  uint64_t* conv = full + NS;
  uint64_t* empty = conv + NS;
  uint64_t* done = empty + NS;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int bid = blockIdx.x;
  const int nt = bid % g.ntiles, mt = (bid / g.ntiles) % g.mtiles, split = bid / (g.ntiles * g.mtiles);
  const int kb0 = (int)((int64_t)split * g.nkb / g.nsplit), kb1 = (int)((int64_t)(split + 1) * g.nkb / g.nsplit);
  const int nk = kb1 - kb0;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NS; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&conv[s], 8);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    *abort_flag = 0;
    mbar_fence_init();
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, g.ncols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      tma_prefetch_desc(&tmA);
      tma_prefetch_desc(&tmB);
      const uint32_t bytes = ATILE + cv.b_bytes;
      int it = 0;
      for (; it < nk; ++it) {
        const int s = it % NS, u = it / NS;
        if (u > 0 && !tc_wait(&empty[s], (u - 1) & 1, abort_flag, 101)) break;
        mbar_arrive_expect_tx(&full[s], bytes);
        const int k = (kb0 + it) * KB;
        tma_load_2d(cv.ahi(s), &tmA, &full[s], k, mt * TM);
        tma_load_2d(cv.bhi(s), &tmB, &full[s], k, nt * g.NT);
      }
      // drain: the last copy issued into every stage has landed
      for (int s = 0; s < NS && s < it; ++s) {
        const int last = s + ((it - 1 - s) / NS) * NS;
        mbar_wait(&full[s], (last / NS) & 1);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = idesc_tf32(g.NT, 0, 0);
      for (int it = 0; it < nk; ++it) {
        const int s = it % NS, u = it / NS;
        if (!tc_wait(&conv[s], u & 1, abort_flag, 102)) break;
        tc_fence_after();
        const uint32_t ah = su32(cv.ahi(s)), al = su32(cv.alo(s)), bh = su32(cv.bhi(s)), bl = su32(cv.blo(s));
#pragma unroll
        for (int j = 0; j < KB / 8; ++j) {
          const uint64_t dah = sdesc_sw128(ah + 32 * j, 16, 1024), dal = sdesc_sw128(al + 32 * j, 16, 1024);
          const uint64_t dbh = sdesc_sw128(bh + 32 * j, 16, 1024), dbl = sdesc_sw128(bl + 32 * j, 16, 1024);
          mma_tf32(tmem, dah, dbh, idesc, (it > 0 || j > 0) ? 1u : 0u);
          mma_tf32(tmem, dah, dbl, idesc, 1u);
          mma_tf32(tmem, dal, dbh, idesc, 1u);
        }
        mma_commit(&empty[s]);
      }
      mma_commit(done);
    }
  } else if (warp >= 4) {
    const int ct = threadIdx.x - 128;   // 0 .. 255 over warps 4-11
    const int n4a = ATILE / 16, n4b = (int)(cv.b_bytes / 16);
    bool ok = true;
    for (int it = 0; it < nk; ++it) {
      const int s = it % NS, u = it / NS;
      if (!tc_wait(&full[s], u & 1, abort_flag, 103)) { ok = false; break; }
      split_tile<256>(cv.ahi(s), cv.alo(s), n4a, ct);
      split_tile<256>(cv.bhi(s), cv.blo(s), n4b, ct);
      fence_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&conv[s]);
    }
    if (warp >= 8) ok = false;   // warps 4-7 (TMEM lanes 0-127) drain the accumulator
    // epilogue: FP32 partial sums -> FP64 workspace
    if (warp < 8 && ok && nk > 0) ok = tc_wait(done, 0, abort_flag, 104);
    tc_fence_after();
    const int q = warp & 3;
    const int row = mt * TM + 32 * q + lane;
    double* wrow = g.W + ((int64_t)split * g.na + row) * g.nb;
    for (int c = 0; c < (warp < 8 ? g.NT / 16 : 0); ++c) {
      uint32_t r[16];
      if (ok && nk > 0) {
        tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + 16 * c, r);
        tmem_wait_ld();
      } else {
#pragma unroll
        for (int i = 0; i < 16; ++i) r[i] = 0u;
      }
      if (row < g.na) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int col = nt * g.NT + 16 * c + i;
          if (col < g.nb) wrow[col] = (double)__uint_as_float(r[i]);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    // every MMA this CTA issued is complete before its TMEM goes back
    if (nk > 0) mbar_wait(done, 0);
    tc_fence_after();
    tmem_dealloc(tmem, g.ncols);
  }
}

// C[i*ldc + j] = alpha sum_s W[s][i][j], fixed order over s
__global__ void gram_reduce_kernel(const double* __restrict__ W, int nsplit, int na, int nb, double alpha,
                                   double* __restrict__ C, int64_t ldc) {
  const int64_t n = (int64_t)na * nb;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < nsplit; ++k) s += W[(int64_t)k * n + e];
    C[(e / nb) * ldc + e % nb] = alpha * s;
  }
}

// --------------------------------------------------------------- rotate
__global__ void __launch_bounds__(384, 1)
    rotate_tc_kernel(const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmUh,
                     const __grid_constant__ CUtensorMap tmUl, const RotArgs g) {
  extern __shared__ uint8_t tc_smem_raw[];
  uint8_t* sm = aligned_smem(tc_smem_raw);
  const int NS = g.NS;
  Carve cv{sm, 2 * ATILE + 2u * (uint32_t)g.NT * 128u, (uint32_t)g.NT * 128u};
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + (size_t)NS * cv.stage_bytes);
  uint64_t* conv = full + NS;
  uint64_t* empty = conv + NS;
  uint64_t* tfull = empty + NS;     // [2] accumulator ready
  uint64_t* tempty = tfull + 2;     // [2] accumulator drained
  uint64_t* drain = tempty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ntile_all = g.ptiles * g.ntiles;
  const int my_tiles = blockIdx.x < ntile_all ? (ntile_all - 1 - blockIdx.x) / gridDim.x + 1 : 0;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NS; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&conv[s], 4);
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&tfull[a], 1);
      mbar_init(&tempty[a], 4);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    mbar_fence_init();
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int total = my_tiles * g.nkc;

  if (warp == 0) {
    if (lane == 0) {
      tma_prefetch_desc(&tmX);
      tma_prefetch_desc(&tmUh);
      tma_prefetch_desc(&tmUl);
      const uint32_t bytes = ATILE + 2 * cv.b_bytes;
      int it = 0;
      for (; it < total; ++it) {
        const int s = it % NS, u = it / NS;
        const int t = blockIdx.x + (it / g.nkc) * gridDim.x, kc = it % g.nkc;
        const int nt = t % g.ntiles, pt = t / g.ntiles;
        if (u > 0 && !tc_wait(&empty[s], (u - 1) & 1, abort_flag, 201)) break;
        mbar_arrive_expect_tx(&full[s], bytes);
#pragma unroll
        for (int i = 0; i < TM / 32; ++i)
          tma_load_2d(cv.ahi(s) + i * 4096, &tmX, &full[s], pt * TM + 32 * i, kc * KB);
        tma_load_2d(cv.bhi(s), &tmUh, &full[s], kc * KB, nt * g.NT);
        tma_load_2d(cv.blo(s), &tmUl, &full[s], kc * KB, nt * g.NT);
      }
      for (int s = 0; s < NS && s < it; ++s) {
        const int last = s + ((it - 1 - s) / NS) * NS;
        mbar_wait(&full[s], (last / NS) & 1);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = idesc_tf32(g.NT, 1, 0);
      int it = 0;
      bool ok = true;
      for (int lt = 0; lt < my_tiles && ok; ++lt) {
        const int a = lt & 1;
        if (lt >= 2 && !tc_wait(&tempty[a], ((lt >> 1) - 1) & 1, abort_flag, 202)) break;
        tc_fence_after();
        const uint32_t d = tmem + 256u * a;
        for (int kc = 0; kc < g.nkc; ++kc, ++it) {
          const int s = it % NS, u = it / NS;
          if (!tc_wait(&conv[s], u & 1, abort_flag, 203)) { ok = false; break; }
          tc_fence_after();
          const uint32_t xh = su32(cv.ahi(s)), xl = su32(cv.alo(s)), uh = su32(cv.bhi(s)), ul = su32(cv.blo(s));
#pragma unroll
          for (int j = 0; j < KB / 8; ++j) {
            // MN-major X: 4-band groups 512 bytes apart, 32-point atoms 4096
            const uint64_t dxh = sdesc(xh + 1024 * j, 4096, 512, SW128_B32);
            const uint64_t dxl = sdesc(xl + 1024 * j, 4096, 512, SW128_B32);
            const uint64_t duh = sdesc_sw128(uh + 32 * j, 16, 1024), dul = sdesc_sw128(ul + 32 * j, 16, 1024);
            mma_tf32(d, dxh, duh, idesc, (kc > 0 || j > 0) ? 1u : 0u);
            mma_tf32(d, dxh, dul, idesc, 1u);
            mma_tf32(d, dxl, duh, idesc, 1u);
          }
          mma_commit(&empty[s]);
        }
        if (ok) mma_commit(&tfull[a]);
      }
      mma_commit(drain);
    }
  } else if (warp >= 4 && warp < 8) {
    const int ct = threadIdx.x - 128;   // 0 .. 127
    for (int it = 0; it < total; ++it) {
      const int s = it % NS, u = it / NS;
      if (!tc_wait(&full[s], u & 1, abort_flag, 204)) break;
      split_tile<128>(cv.ahi(s), cv.alo(s), (int)(ATILE / 16), ct);
      fence_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&conv[s]);
    }
  } else if (warp >= 8) {
    const int q = warp & 3;
    for (int lt = 0; lt < my_tiles; ++lt) {
      const int a = lt & 1;
      if (!tc_wait(&tfull[a], (lt >> 1) & 1, abort_flag, 205)) break;
      tc_fence_after();
      const int t = blockIdx.x + lt * gridDim.x;
      const int nt = t % g.ntiles, pt = t / g.ntiles;
      const int64_t p = (int64_t)pt * TM + 32 * q + lane;
      const bool pin = p < g.K;
      // Z (read-only) for chunk c is loaded one chunk ahead, so its latency
      // hides behind the TMEM load and the stores of the previous chunk
      float z[16], zn[16];
      auto load_z = [&](int c, float (&dst)[16]) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int n = nt * g.NT + 16 * c + i;
          dst[i] = (g.Z && pin && n < g.nn) ? __ldg(g.Z + (int64_t)n * g.ldz + p) : 0.f;
        }
      };
      load_z(0, z);
      const int nch = g.NT / 16;
      for (int c = 0; c < nch; ++c) {
        if (c + 1 < nch) load_z(c + 1, zn);
        uint32_t r[16];
        tmem_ld16(tmem + 256u * a + ((uint32_t)(32 * q) << 16) + 16 * c, r);
        tmem_wait_ld();
        if (pin) {
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const int n = nt * g.NT + 16 * c + i;
            if (n < g.nn) g.Y[(int64_t)n * g.ldy + p] = fmaf(g.beta, z[i], __uint_as_float(r[i]));
          }
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) z[i] = zn[i];
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[a]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    mbar_wait(drain, 0);
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// hi / lo TF32 parts of an FP64 matrix (rows x cols, leading dims lds / ldd)
__global__ void tf32_split_kernel(const double* __restrict__ x, int64_t rows, int64_t cols, int64_t lds,
                                  float* __restrict__ hi, float* __restrict__ lo, int64_t ldd) {
  const int64_t n = rows * ldd;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e / ldd, c = e % ldd;
    float h = 0.f, l = 0.f;
    if (c < cols) {
      const double v = x[r * lds + c];
      h = rn_tf32((float)v);
      l = rn_tf32((float)(v - (double)h));
    }
    hi[e] = h;
    lo[e] = l;
  }
}

// ----------------------------------------------------------------- host
bool encode_2d(CUtensorMap* map, const void* base, uint64_t inner, uint64_t outer, uint64_t row_bytes,
               uint32_t box_inner, uint32_t box_outer,
               CUtensorMapSwizzle swz = CU_TENSOR_MAP_SWIZZLE_128B) {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess || !p)
      return false;
    fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  cuuint64_t d[2] = {inner, outer};
  cuuint64_t s[1] = {row_bytes};
  cuuint32_t b[2] = {box_inner, box_outer};
  cuuint32_t e[2] = {1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(base), d, s, b, e,
            CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

constexpr int SMEM_LIMIT = 227 * 1024;

// N tile: a multiple of 16 of at most 256 columns, balanced over the tiles
void n_tiling(int64_t n, int& NT, int& ntiles) {
  ntiles = (int)((n + 255) / 256);
  const int64_t per = (n + ntiles - 1) / ntiles;
  NT = (int)std::max<int64_t>(16, (per + 15) / 16 * 16);
}

int stages_for(int NT) {
  const int stage = 2 * (int)ATILE + 2 * NT * 128;
  return std::min(4, (SMEM_LIMIT - 2048) / stage);
}

struct GramPlan {
  int mtiles, ntiles, NT, nsplit, nkb, NS;
};

GramPlan gram_plan(int64_t na, int64_t nb, int64_t K) {
  GramPlan p;
  p.mtiles = (int)((na + TM - 1) / TM);
  n_tiling(nb, p.NT, p.ntiles);
  p.nkb = (int)((K + KB - 1) / KB);
  const int tiles = p.mtiles * p.ntiles;
  const int sms = sm_count();
  p.nsplit = std::max(1, std::min(sms / std::max(1, tiles), (p.nkb + 7) / 8));
  p.NS = stages_for(p.NT);
  return p;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

}  // namespace
}  // namespace gb

using namespace gb;

extern "C" {

int gb_band_gram_tc_workspace(int64_t na, int64_t nb, int64_t K, int64_t* bytes) {
  GB_REQUIRE(bytes && na >= 0 && nb >= 0 && K >= 0, "gb_band_gram_tc_workspace: bad arguments");
  if (na == 0 || nb == 0) {
    *bytes = 0;
    return GB_OK;
  }
  const GramPlan p = gram_plan(na, nb, K);
  *bytes = (int64_t)p.nsplit * na * nb * (int64_t)sizeof(double);
  return GB_OK;
}

int gb_band_gram_tc(int64_t na, int64_t nb, int64_t K, const float* A, int64_t lda, const float* B, int64_t ldb,
                    double alpha, double* C, int64_t ldc, void* work, int64_t work_bytes, void* stream) {
  GB_REQUIRE(na >= 0 && nb >= 0 && K >= 0, "gb_band_gram_tc: bad sizes");
  if (na == 0 || nb == 0) return GB_OK;
  GB_REQUIRE(A && B && C && work && lda >= K && ldb >= K && ldc >= nb, "gb_band_gram_tc: null array or bad stride");
  GB_REQUIRE(na < (1 << 30) && nb < (1 << 30) && K < ((int64_t)1 << 36), "gb_band_gram_tc: too large");
  if (K == 0 || lda % 4 || ldb % 4 || !aligned16(A) || !aligned16(B))
    return fail(GB_E_UNSUPPORTED, "gb_band_gram_tc: needs K > 0, 16-byte aligned rows (ld % 4 == 0)");
  const GramPlan p = gram_plan(na, nb, K);
  GB_REQUIRE(work_bytes >= (int64_t)p.nsplit * na * nb * (int64_t)sizeof(double),
             "gb_band_gram_tc: workspace too small");
  CUtensorMap tmA, tmB;
  if (!encode_2d(&tmA, A, (uint64_t)K, (uint64_t)na, (uint64_t)lda * 4, KB, TM) ||
      !encode_2d(&tmB, B, (uint64_t)K, (uint64_t)nb, (uint64_t)ldb * 4, KB, (uint32_t)p.NT))
    return fail(GB_E_UNSUPPORTED, "gb_band_gram_tc: cuTensorMapEncodeTiled rejected the layout");
  cudaStream_t st = (cudaStream_t)stream;
  GramArgs g;
  g.na = (int)na;
  g.nb = (int)nb;
  g.nkb = p.nkb;
  g.mtiles = p.mtiles;
  g.ntiles = p.ntiles;
  g.nsplit = p.nsplit;
  g.NT = p.NT;
  g.NS = p.NS;
  g.ncols = p.NT <= 32 ? 32 : p.NT <= 64 ? 64 : p.NT <= 128 ? 128 : 256;
  g.W = static_cast<double*>(work);
  const int smem = p.NS * (2 * (int)ATILE + 2 * p.NT * 128) + 1024 + 256;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(gram_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_LIMIT);
    attr = true;
  }
  const unsigned grid = (unsigned)(p.mtiles * p.ntiles * p.nsplit);
  gram_tc_kernel<<<grid, 384, smem, st>>>(tmA, tmB, g);
  int rc = check_launch("gram_tc_kernel");
  if (rc != GB_OK) return rc;
  const int64_t n = na * nb;
  const unsigned rb = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 4096));
  gram_reduce_kernel<<<rb, 256, 0, st>>>(g.W, p.nsplit, (int)na, (int)nb, alpha, C, ldc);
  return check_launch("gram_reduce_kernel");
}

int gb_tf32_split(int64_t rows, int64_t cols, const double* x, int64_t lds, float* hi, float* lo, int64_t ldd,
                  void* stream) {
  GB_REQUIRE(rows >= 0 && cols >= 0 && lds >= cols && ldd >= cols, "gb_tf32_split: bad sizes");
  if (rows == 0 || ldd == 0) return GB_OK;
  GB_REQUIRE(x && hi && lo, "gb_tf32_split: null array");
  const int64_t n = rows * ldd;
  const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 4096));
  tf32_split_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(x, rows, cols, lds, hi, lo, ldd);
  return check_launch("tf32_split_kernel");
}

int gb_band_rotate_tc(int64_t nn, int64_t nk, int64_t K, const float* Uhi, const float* Ulo, int64_t ldu,
                      const float* X, int64_t ldx, float beta, const float* Z, int64_t ldz, float* Y, int64_t ldy,
                      void* stream) {
  GB_REQUIRE(nn >= 0 && nk >= 0 && K >= 0, "gb_band_rotate_tc: bad sizes");
  if (nn == 0 || K == 0) return GB_OK;
  GB_REQUIRE(nk > 0 && Uhi && Ulo && X && Y && ldu >= nk && ldx >= K && ldy >= K,
             "gb_band_rotate_tc: null array or bad stride");
  GB_REQUIRE(nn < (1 << 30) && nk < (1 << 30) && K < ((int64_t)1 << 36), "gb_band_rotate_tc: too large");
  GB_REQUIRE(X != Y, "gb_band_rotate_tc: Y must not alias X");
  GB_REQUIRE(!Z || ldz >= K, "gb_band_rotate_tc: bad stride of Z");
  if (ldu % 4 || ldx % 4 || !aligned16(Uhi) || !aligned16(Ulo) || !aligned16(X))
    return fail(GB_E_UNSUPPORTED, "gb_band_rotate_tc: needs 16-byte aligned rows (ld % 4 == 0)");
  RotArgs g;
  n_tiling(nn, g.NT, g.ntiles);
  g.nn = (int)nn;
  g.nk = (int)nk;
  g.K = K;
  g.ptiles = (int)((K + TM - 1) / TM);
  g.nkc = (int)((nk + KB - 1) / KB);
  g.NS = stages_for(g.NT);
  g.Y = Y;
  g.ldy = ldy;
  g.Z = Z;
  g.ldz = ldz;
  g.beta = beta;
  CUtensorMap tmX, tmUh, tmUl;
  if (!encode_2d(&tmX, X, (uint64_t)K, (uint64_t)nk, (uint64_t)ldx * 4, 32, KB,
                 CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B) ||
      !encode_2d(&tmUh, Uhi, (uint64_t)nk, (uint64_t)nn, (uint64_t)ldu * 4, KB, (uint32_t)g.NT) ||
      !encode_2d(&tmUl, Ulo, (uint64_t)nk, (uint64_t)nn, (uint64_t)ldu * 4, KB, (uint32_t)g.NT))
    return fail(GB_E_UNSUPPORTED, "gb_band_rotate_tc: cuTensorMapEncodeTiled rejected the layout");
  const int smem = g.NS * (2 * (int)ATILE + 2 * g.NT * 128) + 1024 + 256;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(rotate_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_LIMIT);
    attr = true;
  }
  const int tiles = g.ptiles * g.ntiles;
  const unsigned grid = (unsigned)std::max(1, std::min(tiles, sm_count()));
  rotate_tc_kernel<<<grid, 384, smem, (cudaStream_t)stream>>>(tmX, tmUh, tmUl, g);
  return check_launch("rotate_tc_kernel");
}

}  // extern "C"
