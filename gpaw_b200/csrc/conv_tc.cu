// 16-channel 3x3x3 convolution on a periodic grid on the tcgen05 tensor
// cores: the level-2 layer of the learned preconditioner (no reference
// counterpart; the network stands in for the V-cycle of
// c/fd_preconditioner.c).
//
//   y[b][co][p] = sum_{ci < 16} sum_{k < 27} w[co][ci][k] x[b][ci][p + o_k]
//
// as an implicit GEMM without im2col: a CTA keeps the input planes
// z - 1 .. z + 1 of one band (a ring of four slots, the next plane staged
// while the current one's MMAs run), padded by the periodic halo, in the canonical
// K-major no-swizzle layout of the MMA -- [channel quad][padded point][4
// channels], 16 bytes per point, so a core matrix is 8 consecutive points
// (SBO = 128 bytes) and the two channel quads of a K = 8 step are one quad
// stride apart (LBO).  A tap (dz, dy, dx) is then the same operand with its
// start address moved by the tap's linear offset in the padded block, and
// the output plane is ceil(P1 P2 / 128) tiles of 128 consecutive padded
// points (halo points are computed and dropped):
//   D[128 points][16 co] += A_tap[128 points][8 ci] . W_tap[16 co][8 ci]^T
// with tcgen05.mma.cta_group::1.kind::tf32 (M = 128, N = 16, K = 8) issued
// by one thread per (tile, channel half) -- up to four threads, each with its
// own accumulator, since a single thread cannot issue these small MMAs fast
// enough -- 27 taps x 2 products per pair.  The
// weights are BF16 and therefore exact TF32 numbers; the activations are
// split x = hi + lo (RN TF32 parts) so the products keep FP32 accuracy.
// The accumulators (TMEM, 2 x 16 columns per tile) are read back with
// tcgen05.ld.32x32b by warps 4-7 (one padded point per lane) and the
// interior points are written, 16 channels each.  Waits are bounded.
#include <algorithm>
#include <cuda_bf16.h>
#include "internal.cuh"
#include "tma.cuh"
#include "tcgen05.cuh"

namespace gb {

__device__ int g_conv_tc_error = 0;

int conv_tc_error_flag(int clear) {
  int v = 0;
  cudaMemcpyFromSymbol(&v, g_conv_tc_error, sizeof(int));
  if (clear && v) {
    int z = 0;
    cudaMemcpyToSymbol(g_conv_tc_error, &z, sizeof(int));
  }
  return v;
}

namespace {
using namespace tc;

struct ConvTcArgs {
  const float* x;                 // (nb, 16, n0, n1, n2)
  float* y;                       // (nb, cout, n0, n1, n2)
  const __nv_bfloat16* w;         // [cout][16][27]
  int64_t nb;
  int cout, n0, n1, n2;
  int P1, P2, PP, tiles, margin, npts, zchunk, accumulate, nissue;
  uint32_t ncols;
};

__device__ __forceinline__ float rn_tf32_(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

// shared-memory descriptor without swizzle (layout type 0)
__device__ __forceinline__ uint64_t sdesc_none(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return sdesc(saddr, lbo, sbo, 0u);
}

// ring of 4 staged planes (each with its own margins): the MMAs of plane z
// read the slots of z - 1, z, z + 1 while the CTA stages plane z + 2 into
// the fourth
__global__ void __launch_bounds__(256, 1) conv16_tc_kernel(const ConvTcArgs a) {
  extern __shared__ __align__(128) unsigned char ctc_smem[];
  float* sW = reinterpret_cast<float*>(ctc_smem);              // [27][4][16][4]
  float* Xhi = sW + 27 * 4 * 16 * 4;                            // [4 slots][4 quads][npts][4]
  float* Xlo = Xhi + 4 * 4 * a.npts * 4;
  uint64_t* done = reinterpret_cast<uint64_t*>(Xlo + 4 * 4 * a.npts * 4);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int n0 = a.n0, n1 = a.n1, n2 = a.n2, P2 = a.P2, PP = a.PP;

  for (int e = tid; e < 27 * 256; e += blockDim.x) {
    const int tap = e >> 8, r = e & 255, q = r >> 6, co = (r >> 2) & 15, i = r & 3;
    sW[e] = co < a.cout ? __bfloat162float(a.w[(co * 16 + 4 * q + i) * 27 + tap]) : 0.f;
  }
  // margins of every slot and quad: zero (only dropped halo outputs read them)
  for (int e = tid; e < 16 * 2 * a.margin; e += blockDim.x) {
    const int sq = e / (2 * a.margin), m = e % (2 * a.margin);
    const int pt = m < a.margin ? m : a.margin + PP + (m - a.margin);
    reinterpret_cast<float4*>(Xhi)[sq * a.npts + pt] = make_float4(0.f, 0.f, 0.f, 0.f);
    reinterpret_cast<float4*>(Xlo)[sq * a.npts + pt] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  if (tid == 0) {
    mbar_init(done, a.nissue);
    mbar_fence_init();
  }
  if (warp == 1) {
    tmem_alloc(tslot, a.ncols);
    tmem_relinquish();
  }
  const int64_t b = blockIdx.y;
  const int64_t nplane = (int64_t)n1 * n2, nvol = nplane * n0;
  const float* xb = a.x + b * 16 * nvol;
  const int z_beg = blockIdx.x * a.zchunk, z_end = min(z_beg + a.zchunk, n0);
  auto slot_of = [&](int p) { return (p - z_beg + 1) & 3; };
  // stage input plane p (periodic) into its slot, split hi / lo
  // (all of a thread's loads for a plane are issued before any is used:
  // up to 8 x 4 values in flight instead of one L2 round trip per 4)
  auto stage = [&](int p) {
    constexpr int MAXIT = 8;
    const int sl = slot_of(p);
    const int zs = p < 0 ? p + n0 : (p >= n0 ? p - n0 : p);
    for (int e0 = tid; e0 < 4 * PP; e0 += MAXIT * 256) {
      float v[MAXIT][4];
#pragma unroll
      for (int it = 0; it < MAXIT; ++it) {
        const int e = e0 + it * 256;
        if (e < 4 * PP) {
          const int q = e / PP, r = e % PP, yy = r / P2, xx = r % P2;
          int ys = yy - 1, xs = xx - 1;
          ys = ys < 0 ? ys + n1 : (ys >= n1 ? ys - n1 : ys);
          xs = xs < 0 ? xs + n2 : (xs >= n2 ? xs - n2 : xs);
          const float* src = xb + (int64_t)(4 * q) * nvol + zs * nplane + (int64_t)ys * n2 + xs;
#pragma unroll
          for (int i = 0; i < 4; ++i) v[it][i] = __ldg(src + i * nvol);
        }
      }
#pragma unroll
      for (int it = 0; it < MAXIT; ++it) {
        const int e = e0 + it * 256;
        if (e < 4 * PP) {
          const int q = e / PP, r = e % PP;
          float h[4], l[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            h[i] = rn_tf32_(v[it][i]);
            l[i] = rn_tf32_(v[it][i] - h[i]);
          }
          const int pt = (sl * 4 + q) * a.npts + a.margin + r;
          reinterpret_cast<float4*>(Xhi)[pt] = make_float4(h[0], h[1], h[2], h[3]);
          reinterpret_cast<float4*>(Xlo)[pt] = make_float4(l[0], l[1], l[2], l[3]);
        }
      }
    }
  };
  stage(z_beg - 1);
  stage(z_beg);
  if (z_beg + 1 < z_end + 1) stage(z_beg + 1);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(16 >> 3) << 17) |
                         ((uint32_t)(128 >> 4) << 24);
  const uint32_t qstride = (uint32_t)a.npts * 16u;
  uint32_t phase = 0;
  bool ok = true;
  for (int z = z_beg; z < z_end; ++z) {
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp < a.nissue && lane == 0) {
      // issuer w (warps 0 .. nissue - 1) feeds the (tile, channel half)
      // pairs w, w + nissue, ...; every pair has its own accumulator
      // (columns 16 (2 t + c)), so the issuers are independent and each
      // commits to `done` (nissue arrivals).  Descriptors differ only in the
      // start address (bits 0-13, 16-byte units, addresses < 256 KB): three
      // base descriptors plus offsets.
      const uint64_t ah0 = sdesc_none(su32(Xhi), qstride, 128);
      const uint64_t al0 = sdesc_none(su32(Xlo), qstride, 128);
      const uint64_t bw0 = sdesc_none(su32(sW), 256, 128);
      const uint32_t npts = (uint32_t)a.npts;
      uint32_t sbase[3];
#pragma unroll
      for (int dz = 0; dz < 3; ++dz) sbase[dz] = (uint32_t)(slot_of(z + dz - 1) * 4) * npts;
      const int rowoff[3] = {-P2, 0, P2};
      for (int pr = warp; pr < 2 * a.tiles; pr += a.nissue) {
        const int t = pr >> 1, c = pr & 1;
        const uint32_t d = tmem + 16u * pr;
        const int tb = a.margin + t * 128;
#pragma unroll
        for (int tap = 0; tap < 27; ++tap) {
          const uint32_t off = sbase[tap / 9] + (uint32_t)(tb + rowoff[(tap / 3) % 3] + (tap % 3 - 1));
          const uint64_t delta = off + 2u * c * npts;
          const uint64_t bw = bw0 + (uint64_t)(tap * 64 + c * 32);
          mma_tf32(d, ah0 + delta, bw, idesc, tap > 0 ? 1u : 0u);
          mma_tf32(d, al0 + delta, bw, idesc, 1u);
        }
      }
      mma_commit(done);
    }
    // the next plane's input goes to the slot plane z - 2 used
    if (z + 2 < z_end + 1) stage(z + 2);
    if (warp >= 4) {
      if (ok && !mbar_wait(done, phase)) {
        ok = false;
        atomicCAS(&g_conv_tc_error, 0, 301);
      }
      tc_fence_after();
      const int q4 = warp & 3;
      for (int t = 0; t < a.tiles; ++t) {
        uint32_t r[16], r1[16];
        tmem_ld16(tmem + 32u * t + ((uint32_t)(32 * q4) << 16), r);
        tmem_ld16(tmem + 32u * t + 16u + ((uint32_t)(32 * q4) << 16), r1);
        tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 16; ++i) r[i] = __float_as_uint(__uint_as_float(r[i]) + __uint_as_float(r1[i]));
        const int lin = t * 128 + 32 * q4 + lane;          // padded point of the plane
        const int yy = lin / P2, xx = lin % P2;
        if (ok && lin < PP && yy >= 1 && yy <= n1 && xx >= 1 && xx <= n2) {
          float* yp = a.y + (b * a.cout) * nvol + z * nplane + (int64_t)(yy - 1) * n2 + (xx - 1);
          for (int co = 0; co < a.cout; ++co) {
            const float v = __uint_as_float(r[co]);
            if (a.accumulate) yp[co * nvol] += v;
            else yp[co * nvol] = v;
          }
        }
      }
      tc_fence_before();
    } else if (warp < a.nissue) {
      // the MMAs must be complete before the ring advances past their slots
      if (ok && !mbar_wait(done, phase)) ok = false;
    }
    phase ^= 1u;
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, a.ncols);
  }
}

}  // namespace

// plan and launch; 0 (not launched) when the layout does not apply
int conv16_tc_try(const float* x, const void* w_bf16, float* y, int64_t nb, int cout, int n0, int n1, int n2,
                  int accumulate, cudaStream_t st, int* launched) {
  *launched = 0;
  if (cout < 1 || cout > 16 || nb < 1 || nb > 65535 || n0 < 2 || n1 < 2 || n2 < 2) return GB_OK;
  ConvTcArgs a;
  a.x = x;
  a.y = y;
  a.w = reinterpret_cast<const __nv_bfloat16*>(w_bf16);
  a.nb = nb;
  a.cout = cout;
  a.n0 = n0; a.n1 = n1; a.n2 = n2;
  a.P1 = n1 + 2;
  a.P2 = n2 + 2;
  a.PP = a.P1 * a.P2;
  a.tiles = (a.PP + 127) / 128;
  if (a.tiles * 32 > 512) return GB_OK;
  const int m = std::max(a.P2 + 1, a.tiles * 128 - a.PP + a.P2 + 1);
  a.margin = (m + 7) / 8 * 8;
  a.npts = a.PP + 2 * a.margin;                   // one slot of one quad
  if (a.npts > 16383) return GB_OK;
  // three plane chunks per band (measured best of 1..7 chunks on 14^3 x 160)
  a.zchunk = std::max(1, std::min(n0, (n0 + 2) / 3));
  a.accumulate = accumulate;
  a.nissue = std::min(4, 2 * a.tiles);            // MMA-issuing threads (warps 0-3)
  uint32_t nc = 32;
  while (nc < (uint32_t)(32 * a.tiles)) nc *= 2;
  if (nc > 512) return GB_OK;
  a.ncols = nc;
  const size_t smem = (size_t)(27 * 256 + 2 * 4 * 4 * a.npts * 4) * sizeof(float) + 64;
  if (smem > 220 * 1024) return GB_OK;
  static size_t attr = 0;
  if (smem > attr) {
    cudaFuncSetAttribute(conv16_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr = smem;
  }
  const dim3 grid((unsigned)((n0 + a.zchunk - 1) / a.zchunk), (unsigned)nb);
  conv16_tc_kernel<<<grid, 256, smem, st>>>(a);
  *launched = 1;
  return check_launch("conv16_tc_kernel");
}

}  // namespace gb
