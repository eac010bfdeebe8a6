// 3x3x3 convolutions for the learned preconditioner (no reference
// counterpart: this is the network that stands in for the multigrid
// V-cycle of c/fd_preconditioner.c).
//
//   forward        y[b][co][p] = sum_ci sum_k w[co][ci][k] x[b][ci][p + o_k]
//   backward-data  the same kernel with w'[ci][co][k] = w[co][ci][26 - k]
//                  (the adjoint of a zero-padded or periodic convolution is
//                  the convolution with the flipped kernel and the same
//                  boundary), built on the host
//   backward-wt    dw[co][ci][k] = sum_b sum_p dy[b][co][p] x[b][ci][p + o_k]
//
// Activations are FP32, weights BF16 (converted to FP32 in shared memory),
// accumulation FP32.  Boundaries per axis: zero padding or periodic wrap
// (the grid's own boundary conditions).  Forward: a CTA covers 1 x 16 x 32
// points (1 x 32 x 32 for one output channel); input channels are staged
// with their halo in shared memory four at a time (a warp per row, lanes
// over columns), the weights once, laid out [ci][k][co] so that four output
// channels' weights come in one 16-byte broadcast load; every thread keeps
// 4 (8 for one output channel) consecutive points x all output channels in
// registers.  Backward-weight: CTAs
// over (co, ci) pairs x chunks of the points; each reduces its chunk's 27
// sums and adds them to dw with FP32 atomics (dw accumulates, as before).
#include <cuda_bf16.h>
#include <algorithm>
#include "internal.cuh"

namespace gb {

struct ConvArgs {
  const float* x;
  float* y;
  const __nv_bfloat16* w;   // [cout][cin][27]
  int64_t nb;
  int cin, cout;
  int n0, n1, n2;
  int pbc0, pbc1, pbc2;
  int accumulate;           // y += conv(x) instead of y = conv(x)
};

// forward tile: one plane (axis 0) x CY rows x CZ points; a thread owns PX
// consecutive points of one row and all COUT outputs of them.  Single-output
// convolutions use PX = 8 (one weight load per 8 FMAs), the others PX = 4.
constexpr int CZ = 32, CTHREADS = 128, CCH = 4;
template <int COUT> struct ConvTile {
  static constexpr int PX = COUT == 1 ? 8 : 4;
  static constexpr int CY = CTHREADS / (CZ / PX);      // 32 or 16 rows
  static constexpr int SY = CY + 2;                    // staged rows
  static constexpr int SZP = CZ + PX;                  // padded row pitch (floats), >= CZ + 2, multiple of 4
};

__device__ __forceinline__ int cwrap(int i, int n) {
  int r = i % n;
  return r < 0 ? r + n : r;
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(CTHREADS) conv3d_fwd_kernel(const ConvArgs a) {
  using TL = ConvTile<COUT>;
  constexpr int PX = TL::PX, CY = TL::CY, SY = TL::SY, SZP = TL::SZP;
  constexpr int CC = CIN < CCH ? CIN : CCH;
  extern __shared__ __align__(16) float conv_smem[];
  float* sw = conv_smem;                                     // [ci][k][co]
  float* sx = conv_smem + ((CIN * 27 * COUT + 3) / 4) * 4;   // [cc][3][SY][SZP]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int e = tid; e < COUT * CIN * 27; e += CTHREADS) {
    const int co = e / (CIN * 27), ci = (e / 27) % CIN, k = e % 27;
    sw[(ci * 27 + k) * COUT + co] = __bfloat162float(a.w[e]);
  }
  const int tyn = (a.n1 + CY - 1) / CY, tzn = (a.n2 + CZ - 1) / CZ;
  const int64_t ntile = (int64_t)a.n0 * tyn * tzn;
  const int64_t n012 = (int64_t)a.n0 * a.n1 * a.n2;
  const int ty = tid / (CZ / PX), tz = (tid % (CZ / PX)) * PX;
  for (int64_t t = blockIdx.x; t < ntile * a.nb; t += gridDim.x) {
    const int64_t b = t / ntile;
    int64_t r = t % ntile;
    const int i0 = (int)(r / (tyn * tzn));
    r %= tyn * tzn;
    const int j0 = (int)(r / tzn) * CY, k0 = (int)(r % tzn) * CZ;
    // the staged columns of this lane (fixed for the tile)
    int gz0 = k0 - 1 + lane, gz1 = k0 - 1 + 32 + lane;
    bool oz0 = true, oz1 = lane < 2;
    if (gz0 < 0 || gz0 >= a.n2) { if (a.pbc2) gz0 = cwrap(gz0, a.n2); else oz0 = false; }
    if (gz1 < 0 || gz1 >= a.n2) { if (a.pbc2) gz1 = cwrap(gz1, a.n2); else oz1 = false; }
    float acc[PX][COUT];
#pragma unroll
    for (int p = 0; p < PX; ++p)
#pragma unroll
      for (int co = 0; co < COUT; ++co) acc[p][co] = 0.f;
    for (int c0 = 0; c0 < CIN; c0 += CC) {
      __syncthreads();   // previous pass (and the weight staging) done
      // one warp per staged row (channel, plane, row): lanes over columns
      for (int row = warp; row < CC * 3 * SY; row += CTHREADS / 32) {
        const int jj = row % SY, ii = (row / SY) % 3, cc = row / (3 * SY);
        int g0 = i0 - 1 + ii, g1 = j0 - 1 + jj;
        bool ok = true;
        if (g0 < 0 || g0 >= a.n0) { if (a.pbc0) g0 = cwrap(g0, a.n0); else ok = false; }
        if (g1 < 0 || g1 >= a.n1) { if (a.pbc1) g1 = cwrap(g1, a.n1); else ok = false; }
        const float* src = a.x + (b * CIN + c0 + cc) * n012 + ((int64_t)g0 * a.n1 + g1) * a.n2;
        float* dst = sx + row * SZP;
        // asynchronous 4-byte copies: every row's loads are in flight at once
        if (ok && oz0) cp_async4(dst + lane, src + gz0); else dst[lane] = 0.f;
        if (lane < 2) {
          if (ok && oz1) cp_async4(dst + 32 + lane, src + gz1); else dst[32 + lane] = 0.f;
        }
      }
      cp_async_commit();
      cp_async_wait<0>();
      __syncthreads();
#pragma unroll 1
      for (int cc = 0; cc < CC; ++cc) {
        const float* wc = sw + (c0 + cc) * 27 * COUT;
#pragma unroll
        for (int dx = 0; dx < 3; ++dx)
#pragma unroll
          for (int dy = 0; dy < 3; ++dy) {
            const float* rowp = sx + ((cc * 3 + dx) * SY + ty + dy) * SZP + tz;
            float in[PX + 2];
#pragma unroll
            for (int q = 0; q < PX; q += 4) {
              const float4 v4 = *reinterpret_cast<const float4*>(rowp + q);
              in[q] = v4.x; in[q + 1] = v4.y; in[q + 2] = v4.z; in[q + 3] = v4.w;
            }
            in[PX] = rowp[PX];
            in[PX + 1] = rowp[PX + 1];
#pragma unroll
            for (int dz = 0; dz < 3; ++dz) {
              const float* wk = wc + (dx * 9 + dy * 3 + dz) * COUT;
              if constexpr (COUT % 4 == 0) {
#pragma unroll
                for (int co = 0; co < COUT; co += 4) {
                  const float4 w4 = *reinterpret_cast<const float4*>(wk + co);
#pragma unroll
                  for (int p = 0; p < PX; ++p) {
                    acc[p][co] = fmaf(w4.x, in[p + dz], acc[p][co]);
                    acc[p][co + 1] = fmaf(w4.y, in[p + dz], acc[p][co + 1]);
                    acc[p][co + 2] = fmaf(w4.z, in[p + dz], acc[p][co + 2]);
                    acc[p][co + 3] = fmaf(w4.w, in[p + dz], acc[p][co + 3]);
                  }
                }
              } else {
#pragma unroll
                for (int co = 0; co < COUT; ++co) {
                  const float w = wk[co];
#pragma unroll
                  for (int p = 0; p < PX; ++p) acc[p][co] = fmaf(w, in[p + dz], acc[p][co]);
                }
              }
            }
          }
      }
    }
    const int gj = j0 + ty;
    if (gj < a.n1) {
#pragma unroll
      for (int co = 0; co < COUT; ++co) {
        float* yp = a.y + (b * COUT + co) * n012 + ((int64_t)i0 * a.n1 + gj) * a.n2;
#pragma unroll
        for (int p = 0; p < PX; ++p) {
          const int gk = k0 + tz + p;
          if (gk < a.n2) yp[gk] = a.accumulate ? yp[gk] + acc[p][co] : acc[p][co];
        }
      }
    }
  }
}

// dw[co][ci][k] += sum_b sum_p dy[b][co][p] x[b][ci][p + o_k]   (FP32)
// grid: (cin * cout channel pairs) x (chunks of the band x point range);
// each CTA reduces its chunk and adds its 27 sums to dw with atomics
__global__ void __launch_bounds__(256) conv3d_bwd_w_kernel(const float* __restrict__ x, const float* __restrict__ dy,
                                                           float* __restrict__ dw, int64_t nb, int cin, int cout, int n0,
                                                           int n1, int n2, int pbc0, int pbc1, int pbc2) {
  const int co = blockIdx.x / cin, ci = blockIdx.x % cin;
  const int64_t n012 = (int64_t)n0 * n1 * n2;
  const int64_t total = nb * n012;
  const int64_t e0 = total * blockIdx.y / gridDim.y, e1 = total * (blockIdx.y + 1) / gridDim.y;
  float acc[27];
#pragma unroll
  for (int k = 0; k < 27; ++k) acc[k] = 0.f;
  for (int64_t e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
    const int64_t b = e / n012, p = e % n012;
    const int g2 = (int)(p % n2), g1 = (int)((p / n2) % n1), g0 = (int)(p / ((int64_t)n1 * n2));
    const float d = dy[(b * cout + co) * n012 + p];
    if (d == 0.f) continue;
    const float* xb = x + (b * cin + ci) * n012;
#pragma unroll
    for (int k = 0; k < 27; ++k) {
      int h0 = g0 + k / 9 - 1, h1 = g1 + (k / 3) % 3 - 1, h2 = g2 + k % 3 - 1;
      bool ok = true;
      if (h0 < 0 || h0 >= n0) { if (pbc0) h0 = cwrap(h0, n0); else ok = false; }
      if (h1 < 0 || h1 >= n1) { if (pbc1) h1 = cwrap(h1, n1); else ok = false; }
      if (h2 < 0 || h2 >= n2) { if (pbc2) h2 = cwrap(h2, n2); else ok = false; }
      if (ok) acc[k] = fmaf(d, xb[((int64_t)h0 * n1 + h1) * n2 + h2], acc[k]);
    }
  }
  __shared__ float red[8][27];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 27; ++k) {
    float v = acc[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < 27) {
    float v = 0.f;
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) v += red[w][threadIdx.x];
    atomicAdd(&dw[((int64_t)co * cin + ci) * 27 + threadIdx.x], v);
  }
}

template <int CIN, int COUT>
static int fwd_launch(const ConvArgs& a, cudaStream_t st) {
  using TL = ConvTile<COUT>;
  constexpr int CC = CIN < CCH ? CIN : CCH;
  const int64_t tiles = (int64_t)a.n0 * ((a.n1 + TL::CY - 1) / TL::CY) * ((a.n2 + CZ - 1) / CZ) * a.nb;
  const size_t smem = (size_t)(((CIN * 27 * COUT + 3) / 4) * 4 + CC * 3 * TL::SY * TL::SZP) * sizeof(float);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(conv3d_fwd_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr = true;
  }
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, conv3d_fwd_kernel<CIN, COUT>, CTHREADS, smem);
  const int64_t blocks = std::min<int64_t>(tiles, (int64_t)sm_count() * std::max(per_sm, 1) * 2);
  conv3d_fwd_kernel<CIN, COUT><<<(unsigned)std::max<int64_t>(blocks, 1), CTHREADS, smem, st>>>(a);
  return check_launch("conv3d_fwd_kernel");
}

}  // namespace gb

using namespace gb;

extern "C" {

int gb_conv3d_forward(const float* x, const void* w_bf16, float* y, int64_t nb, int cin, int cout,
                      const int64_t n_c[3], const int pbc_c[3], int accumulate, void* stream) {
  GB_REQUIRE(x && w_bf16 && y && n_c && pbc_c && nb >= 0, "gb_conv3d_forward: bad arguments");
  if (nb == 0) return GB_OK;
  ConvArgs a{x, y, reinterpret_cast<const __nv_bfloat16*>(w_bf16), nb, cin, cout,
             (int)n_c[0], (int)n_c[1], (int)n_c[2], pbc_c[0], pbc_c[1], pbc_c[2], accumulate};
  cudaStream_t st = (cudaStream_t)stream;
  if (cin == 1 && cout == 1) return fwd_launch<1, 1>(a, st);
  if (cin == 1 && cout == 16) return fwd_launch<1, 16>(a, st);
  if (cin == 16 && cout == 16) return fwd_launch<16, 16>(a, st);
  if (cin == 16 && cout == 1) return fwd_launch<16, 1>(a, st);
  return fail(GB_E_UNSUPPORTED, "gb_conv3d_forward: channel pair not in {(1,1), (1,16), (16,16), (16,1)}");
}

int gb_conv3d_backward_weight(const float* x, const float* dy, float* dw, int64_t nb, int cin, int cout,
                              const int64_t n_c[3], const int pbc_c[3], void* stream) {
  GB_REQUIRE(x && dy && dw && n_c && pbc_c && nb >= 0 && cin > 0 && cout > 0,
             "gb_conv3d_backward_weight: bad arguments");
  if (nb == 0) return GB_OK;
  // enough chunks to fill the GPU about four times over, each >= 4096 points
  const int64_t total = nb * n_c[0] * n_c[1] * n_c[2];
  const int64_t want = std::max<int64_t>(1, (int64_t)sm_count() * 8 / (cin * cout));
  const int64_t chunks = std::max<int64_t>(1, std::min<int64_t>(want, total / 4096));
  dim3 grid((unsigned)(cin * cout), (unsigned)std::min<int64_t>(chunks, 65535));
  conv3d_bwd_w_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(x, dy, dw, nb, cin, cout, (int)n_c[0],
                                                                    (int)n_c[1], (int)n_c[2], pbc_c[0], pbc_c[1],
                                                                    pbc_c[2]);
  return check_launch("conv3d_bwd_w_kernel");
}

}  // extern "C"
