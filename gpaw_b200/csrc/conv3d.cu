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
// (the grid's own boundary conditions).  Forward: a CTA stages a 1 x 4 x 32
// point tile of all input channels plus halo in shared memory and every
// thread produces all output channels of one point.  Backward-weight: CTAs
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

constexpr int CT0 = 1, CT1 = 4, CT2 = 32;   // tile
constexpr int HT0 = CT0 + 2, HT1 = CT1 + 2, HT2 = CT2 + 2;

__device__ __forceinline__ int cwrap(int i, int n) {
  int r = i % n;
  return r < 0 ? r + n : r;
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(CT1 * CT2) conv3d_fwd_kernel(const ConvArgs a) {
  extern __shared__ float conv_smem[];
  float (*sx)[HT0][HT1][HT2] = reinterpret_cast<float (*)[HT0][HT1][HT2]>(conv_smem);
  float* sw = conv_smem + CIN * HT0 * HT1 * HT2;
  const int tid = threadIdx.x;
  for (int e = tid; e < COUT * CIN * 27; e += blockDim.x) sw[e] = __bfloat162float(a.w[e]);
  const int t1n = (a.n1 + CT1 - 1) / CT1, t2n = (a.n2 + CT2 - 1) / CT2;
  const int64_t ntile = (int64_t)a.n0 * t1n * t2n;
  const int64_t n012 = (int64_t)a.n0 * a.n1 * a.n2;
  for (int64_t t = blockIdx.x; t < ntile * a.nb; t += gridDim.x) {
    const int64_t b = t / ntile;
    int64_t r = t % ntile;
    const int i0 = (int)(r / (t1n * t2n));
    r %= t1n * t2n;
    const int j0 = (int)(r / t2n) * CT1, k0 = (int)(r % t2n) * CT2;
    __syncthreads();
    for (int e = tid; e < CIN * HT0 * HT1 * HT2; e += blockDim.x) {
      const int kk = e % HT2, jj = (e / HT2) % HT1, ii = (e / (HT2 * HT1)) % HT0, ci = e / (HT2 * HT1 * HT0);
      int g0 = i0 - 1 + ii, g1 = j0 - 1 + jj, g2 = k0 - 1 + kk;
      float v = 0.f;
      bool ok = true;
      if (g0 < 0 || g0 >= a.n0) { if (a.pbc0) g0 = cwrap(g0, a.n0); else ok = false; }
      if (g1 < 0 || g1 >= a.n1) { if (a.pbc1) g1 = cwrap(g1, a.n1); else ok = false; }
      if (g2 < 0 || g2 >= a.n2) { if (a.pbc2) g2 = cwrap(g2, a.n2); else ok = false; }
      if (ok) v = a.x[(b * CIN + ci) * n012 + ((int64_t)g0 * a.n1 + g1) * a.n2 + g2];
      sx[ci][ii][jj][kk] = v;
    }
    __syncthreads();
    const int tj = tid / CT2, tk = tid % CT2;
    const int gj = j0 + tj, gk = k0 + tk;
    if (gj >= a.n1 || gk >= a.n2) continue;
    float acc[COUT];
#pragma unroll
    for (int co = 0; co < COUT; ++co) acc[co] = 0.f;
#pragma unroll 1
    for (int ci = 0; ci < CIN; ++ci) {
#pragma unroll
      for (int k = 0; k < 27; ++k) {
        const float v = sx[ci][k / 9][tj + (k / 3) % 3][tk + k % 3];
#pragma unroll
        for (int co = 0; co < COUT; ++co) acc[co] = fmaf(sw[(co * CIN + ci) * 27 + k], v, acc[co]);
      }
    }
    const int64_t p = ((int64_t)i0 * a.n1 + gj) * a.n2 + gk;
#pragma unroll
    for (int co = 0; co < COUT; ++co) {
      float* yp = a.y + (b * COUT + co) * n012 + p;
      *yp = a.accumulate ? *yp + acc[co] : acc[co];
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
  const int64_t tiles = (int64_t)a.n0 * ((a.n1 + CT1 - 1) / CT1) * ((a.n2 + CT2 - 1) / CT2) * a.nb;
  const int64_t blocks = std::min<int64_t>(tiles, (int64_t)sm_count() * 8);
  const size_t smem = (size_t)(CIN * HT0 * HT1 * HT2 + COUT * CIN * 27) * sizeof(float);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(conv3d_fwd_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr = true;
  }
  conv3d_fwd_kernel<CIN, COUT><<<(unsigned)std::max<int64_t>(blocks, 1), CT1 * CT2, smem, st>>>(a);
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
