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
#include <mutex>
#include "internal.cuh"

namespace gb {

// tcgen05 implicit-GEMM convolution of 16 input channels (conv_tc.cu)
int conv16_tc_try(const float* x, const void* w_bf16, float* y, int64_t nb, int cout, int n0, int n1, int n2,
                  int accumulate, cudaStream_t st, int* launched);

struct ConvArgs {
  const float* x;
  const float* x2;          // when set: input channel 1 comes from here (CIN = 2)
  float* y;
  const __nv_bfloat16* w;   // [cout][cin][27]
  int64_t nb;
  int cin, cout;
  int n0, n1, n2;
  int pbc0, pbc1, pbc2;
  int accumulate;           // y += conv(x) instead of y = conv(x)
};

// forward tile: one plane (axis 0) x CY rows x CZT points; a thread owns PX
// consecutive points of one row and all COUT outputs of them (PX = 8 for a
// single output channel: one weight load per 8 FMAs; 4 otherwise).  Rows of
// at most 16 points use 16-wide tiles.  The shared row pitch keeps the
// 16-byte loads of a warp free of bank conflicts on 32-wide tiles (2-way on
// 16-wide ones).
constexpr int CCH = 4;
template <int COUT, int CZT> struct ConvTile {
  static constexpr int PX = COUT == 1 ? 8 : 4;
  static constexpr int CY = 16 * (CZT == 32 && COUT == 1 ? 2 : 1);
  static constexpr int THREADS = CY * (CZT / PX);
  static constexpr int SY = CY + 2;
  // staged window: global columns k0 - 4 .. k0 + CZT + 3 (16-byte chunks when
  // the row length is a multiple of 4); pitch free of bank conflicts for the
  // 16-byte loads on 32-wide tiles
  static constexpr int CH = (CZT + 8) / 4;           // chunks per staged row
  static constexpr int SZP = CZT == 32 ? (PX == 8 ? 44 : 40) : CZT + 12;
};

__device__ __forceinline__ int cwrap(int i, int n) {
  int r = i % n;
  return r < 0 ? r + n : r;
}

template <int CIN, int COUT, int CZT>
__global__ void __launch_bounds__(ConvTile<COUT, CZT>::THREADS) conv3d_fwd_kernel(const ConvArgs a) {
  using TL = ConvTile<COUT, CZT>;
  constexpr int PX = TL::PX, CY = TL::CY, SY = TL::SY, SZP = TL::SZP, NT = TL::THREADS;
  constexpr int CC = CIN < CCH ? CIN : CCH;
  constexpr int NW = (NT + 31) / 32;
  extern __shared__ __align__(16) float conv_smem[];
  float* sw = conv_smem;                                     // [ci][k][co]
  float* sx = conv_smem + ((CIN * 27 * COUT + 3) / 4) * 4;   // [cc][3][SY][SZP]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int e = tid; e < COUT * CIN * 27; e += NT) {
    const int co = e / (CIN * 27), ci = (e / 27) % CIN, k = e % 27;
    sw[(ci * 27 + k) * COUT + co] = __bfloat162float(a.w[e]);
  }
  const int tyn = (a.n1 + CY - 1) / CY, tzn = (a.n2 + CZT - 1) / CZT;
  const int64_t ntile = (int64_t)a.n0 * tyn * tzn;
  const int64_t n012 = (int64_t)a.n0 * a.n1 * a.n2;
  const int ty = tid / (CZT / PX), tz = (tid % (CZT / PX)) * PX;
  const int xin = a.x2 ? 1 : CIN;     // channels per sample in x
  const bool vec_rows = (a.n2 % 4) == 0;   // 16-byte aligned rows: chunk staging
  const bool even_rows = (a.n2 % 2) == 0;  // 8-byte aligned rows
  for (int64_t t = blockIdx.x; t < ntile * a.nb; t += gridDim.x) {
    const int64_t b = t / ntile;
    int64_t r = t % ntile;
    const int i0 = (int)(r / (tyn * tzn));
    r %= tyn * tzn;
    const int j0 = (int)(r / tzn) * CY, k0 = (int)(r % tzn) * CZT;
    float acc[PX][COUT];
#pragma unroll
    for (int p = 0; p < PX; ++p)
#pragma unroll
      for (int co = 0; co < COUT; ++co) acc[p][co] = 0.f;
    for (int c0 = 0; c0 < CIN; c0 += CC) {
      __syncthreads();   // previous pass (and the weight staging) done
      if (vec_rows) {
        // 16-byte chunks: a warp stages 32 / CH rows per iteration
        constexpr int RPW = 32 / TL::CH;
        const int lr = lane / TL::CH, ck = lane % TL::CH;
        int gz = k0 - 4 + 4 * ck;
        bool oz = true;
        if (gz < 0 || gz >= a.n2) { if (a.pbc2) gz = cwrap(gz, a.n2); else oz = false; }
        for (int row0 = warp * RPW; row0 < CC * 3 * SY; row0 += NW * RPW) {
          const int row = row0 + lr;
          if (lr < RPW && row < CC * 3 * SY) {
            const int jj = row % SY, ii = (row / SY) % 3, cc = row / (3 * SY);
            int g0 = i0 - 1 + ii, g1 = j0 - 1 + jj;
            bool ok = oz;
            if (g0 < 0 || g0 >= a.n0) { if (a.pbc0) g0 = cwrap(g0, a.n0); else ok = false; }
            if (g1 < 0 || g1 >= a.n1) { if (a.pbc1) g1 = cwrap(g1, a.n1); else ok = false; }
            const int ch = c0 + cc;
            const float* xs = (a.x2 && ch == 1) ? a.x2 : a.x;
            const int chx = a.x2 ? 0 : ch;
            float* dst = sx + row * SZP + 4 * ck;
            if (ok) cp_async16(dst, xs + (b * xin + chx) * n012 + ((int64_t)g0 * a.n1 + g1) * a.n2 + gz);
            else *reinterpret_cast<float4*>(dst) = make_float4(0.f, 0.f, 0.f, 0.f);
          }
        }
      } else if (even_rows) {
        // 8-byte chunks (even row length): a warp stages 32 / CH8 rows per iteration
        constexpr int CH8 = (CZT + 8) / 2;
        constexpr int RPW = 32 / CH8;
        const int lr = lane / CH8, ck = lane % CH8;
        int gz = k0 - 4 + 2 * ck;
        bool oz = true;
        if (gz < 0 || gz >= a.n2) { if (a.pbc2) gz = cwrap(gz, a.n2); else oz = false; }
        for (int row0 = warp * RPW; row0 < CC * 3 * SY; row0 += NW * RPW) {
          const int row = row0 + lr;
          if (lr < RPW && row < CC * 3 * SY) {
            const int jj = row % SY, ii = (row / SY) % 3, cc = row / (3 * SY);
            int g0 = i0 - 1 + ii, g1 = j0 - 1 + jj;
            bool ok = oz;
            if (g0 < 0 || g0 >= a.n0) { if (a.pbc0) g0 = cwrap(g0, a.n0); else ok = false; }
            if (g1 < 0 || g1 >= a.n1) { if (a.pbc1) g1 = cwrap(g1, a.n1); else ok = false; }
            const int ch = c0 + cc;
            const float* xs = (a.x2 && ch == 1) ? a.x2 : a.x;
            const int chx = a.x2 ? 0 : ch;
            float* dst = sx + row * SZP + 2 * ck;
            if (ok) cp_async8(dst, xs + (b * xin + chx) * n012 + ((int64_t)g0 * a.n1 + g1) * a.n2 + gz);
            else *reinterpret_cast<float2*>(dst) = make_float2(0.f, 0.f);
          }
        }
      } else {
        // element copies (odd row length): one warp per row
        for (int row = warp; row < CC * 3 * SY; row += NW) {
          const int jj = row % SY, ii = (row / SY) % 3, cc = row / (3 * SY);
          int g0 = i0 - 1 + ii, g1 = j0 - 1 + jj;
          bool ok = true;
          if (g0 < 0 || g0 >= a.n0) { if (a.pbc0) g0 = cwrap(g0, a.n0); else ok = false; }
          if (g1 < 0 || g1 >= a.n1) { if (a.pbc1) g1 = cwrap(g1, a.n1); else ok = false; }
          const int ch = c0 + cc;
          const float* xs = (a.x2 && ch == 1) ? a.x2 : a.x;
          const int chx = a.x2 ? 0 : ch;
          const float* src = xs + (b * xin + chx) * n012 + ((int64_t)g0 * a.n1 + g1) * a.n2;
          float* dst = sx + row * SZP;
          for (int c = lane; c < CZT + 8; c += 32) {
            int gz = k0 - 4 + c;
            bool okz = ok;
            if (gz < 0 || gz >= a.n2) { if (a.pbc2) gz = cwrap(gz, a.n2); else okz = false; }
            if (okz) cp_async4(dst + c, src + gz); else dst[c] = 0.f;
          }
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
            // staged column c holds global column k0 - 4 + c: this thread's
            // inputs k0 + tz - 1 .. k0 + tz + PX sit at tz + 3 .. tz + PX + 4
            const float* rowp = sx + ((cc * 3 + dx) * SY + ty + dy) * SZP + tz;
            float win[PX + 8];
#pragma unroll
            for (int q = 0; q < PX + 8; q += 4) {
              const float4 v4 = *reinterpret_cast<const float4*>(rowp + q);
              win[q] = v4.x; win[q + 1] = v4.y; win[q + 2] = v4.z; win[q + 3] = v4.w;
            }
            float in[PX + 2];
#pragma unroll
            for (int i = 0; i < PX + 2; ++i) in[i] = win[3 + i];
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

// 16 -> 16 channels on a periodic grid small enough to stage a few whole
// planes (the level-2 convolution of the learned preconditioner): a CTA
// takes TP output planes of one band, stages input planes z0 - 1 .. z0 + TP
// of all 16 channels with their periodic halo ([plane][ci][n1 + 2][n2 + 2])
// and the weights ([ci][tap][co]) once, then every thread accumulates two
// neighbouring points of a row x 16 output channels: per (input channel,
// tap) two shared loads of the input, four broadcast 16-byte weight loads
// and 32 FMAs.
constexpr int C16_TP = 2;

__global__ void __launch_bounds__(256) conv16_periodic_kernel(const ConvArgs a) {
  extern __shared__ __align__(16) float c16_smem[];
  const int n0 = a.n0, n1 = a.n1, n2 = a.n2;
  const int P1 = n1 + 2, P2 = n2 + 2, PP = P1 * P2;
  float* sw = c16_smem;                       // [16][27][16]
  float* sx = c16_smem + 16 * 27 * 16;        // [TP + 2][16][P1][P2]
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int e = tid; e < 16 * 16 * 27; e += nt) {
    const int co = e / (16 * 27), ci = (e / 27) % 16, k = e % 27;
    sw[(ci * 27 + k) * 16 + co] = __bfloat162float(a.w[e]);
  }
  const int z0 = blockIdx.x * C16_TP;
  const int64_t b = blockIdx.y;
  const int64_t n012 = (int64_t)n0 * n1 * n2;
  const float* xb = a.x + b * 16 * n012;
  // stage (TP + 2) planes x 16 channels with the periodic halo
  const int nst = (C16_TP + 2) * 16 * PP;
  for (int e = tid; e < nst; e += nt) {
    const int px = e % P2;
    int r = e / P2;
    const int py = r % P1;
    r /= P1;
    const int ci = r % 16, pz = r / 16;
    int z = z0 - 1 + pz, y = py - 1, x = px - 1;
    z = z < 0 ? z + n0 : (z >= n0 ? z - n0 : z);
    y = y < 0 ? y + n1 : (y >= n1 ? y - n1 : y);
    x = x < 0 ? x + n2 : (x >= n2 ? x - n2 : x);
    sx[e] = __ldg(xb + ci * n012 + ((int64_t)z * n1 + y) * n2 + x);
  }
  __syncthreads();
  const int hx = n2 >> 1;                      // point pairs per row
  const int per_plane = n1 * hx;
  const int zl = tid / per_plane;
  if (zl >= C16_TP || z0 + zl >= n0) return;
  const int rem = tid % per_plane;
  const int y = rem / hx, x = 2 * (rem % hx);
  float acc0[16], acc1[16];
#pragma unroll
  for (int co = 0; co < 16; ++co) { acc0[co] = 0.f; acc1[co] = 0.f; }
#pragma unroll 1
  for (int ci = 0; ci < 16; ++ci) {
#pragma unroll
    for (int dz = 0; dz < 3; ++dz)
#pragma unroll
      for (int dy = 0; dy < 3; ++dy) {
        const float* row = sx + ((zl + dz) * 16 + ci) * PP + (y + dy) * P2 + x;
        const float v0 = row[0], v1 = row[1], v2 = row[2], v3 = row[3];
#pragma unroll
        for (int dx = 0; dx < 3; ++dx) {
          const float va = dx == 0 ? v0 : (dx == 1 ? v1 : v2);
          const float vb = dx == 0 ? v1 : (dx == 1 ? v2 : v3);
          const float4* w4 = reinterpret_cast<const float4*>(sw + (ci * 27 + dz * 9 + dy * 3 + dx) * 16);
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const float4 w = w4[q];
            acc0[4 * q] = fmaf(w.x, va, acc0[4 * q]);
            acc0[4 * q + 1] = fmaf(w.y, va, acc0[4 * q + 1]);
            acc0[4 * q + 2] = fmaf(w.z, va, acc0[4 * q + 2]);
            acc0[4 * q + 3] = fmaf(w.w, va, acc0[4 * q + 3]);
            acc1[4 * q] = fmaf(w.x, vb, acc1[4 * q]);
            acc1[4 * q + 1] = fmaf(w.y, vb, acc1[4 * q + 1]);
            acc1[4 * q + 2] = fmaf(w.z, vb, acc1[4 * q + 2]);
            acc1[4 * q + 3] = fmaf(w.w, vb, acc1[4 * q + 3]);
          }
        }
      }
  }
  float* yb = a.y + b * 16 * n012 + ((int64_t)(z0 + zl) * n1 + y) * n2 + x;
#pragma unroll
  for (int co = 0; co < 16; ++co) {
    float* yp = yb + co * n012;
    if (a.accumulate) {
      yp[0] += acc0[co];
      yp[1] += acc1[co];
    } else {
      yp[0] = acc0[co];
      yp[1] = acc1[co];
    }
  }
}

// smem bytes of conv16_periodic_kernel for a grid (0 when it does not apply)
static size_t conv16_smem(const ConvArgs& a) {
  if (!(a.pbc0 && a.pbc1 && a.pbc2) || a.n2 % 2 || a.n0 < 2) return 0;
  if ((int64_t)C16_TP * a.n1 * (a.n2 / 2) > 256 || a.nb > 65535) return 0;
  const size_t bytes = (size_t)(16 * 27 * 16 + (C16_TP + 2) * 16 * (a.n1 + 2) * (a.n2 + 2)) * sizeof(float);
  return bytes <= 200 * 1024 ? bytes : 0;
}

static int conv16_launch(const ConvArgs& a, size_t smem, cudaStream_t st) {
  static size_t attr = 0;
  if (smem > attr) {
    cudaFuncSetAttribute(conv16_periodic_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr = smem;
  }
  const int threads = ((C16_TP * a.n1 * (a.n2 / 2) + 31) / 32) * 32;
  const dim3 grid((unsigned)((a.n0 + C16_TP - 1) / C16_TP), (unsigned)a.nb);
  conv16_periodic_kernel<<<grid, threads, smem, st>>>(a);
  return check_launch("conv16_periodic_kernel");
}

// dw[co][ci][k] += sum_b sum_p dy[b][co][p] x[b][ci][p + o_k]   (FP32)
// grid: (cin * cout channel pairs) x (chunks of the band x point range);
// each CTA reduces its chunk in a fixed order and writes its 27 sums to
// part[pair][chunk]; conv3d_bwd_w_reduce_kernel adds them to dw in chunk
// order, so the gradient does not depend on scheduling
__global__ void __launch_bounds__(256) conv3d_bwd_w_kernel(const float* __restrict__ x, const float* __restrict__ dy,
                                                           float* __restrict__ part, int64_t nb, int cin, int cout,
                                                           int n0, int n1, int n2, int pbc0, int pbc1, int pbc2) {
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
    part[((int64_t)blockIdx.x * gridDim.y + blockIdx.y) * 27 + threadIdx.x] = v;
  }
}

// dw[pair][k] += sum over chunks c (in order) of part[pair][c][k]
__global__ void conv3d_bwd_w_reduce_kernel(const float* __restrict__ part, int nchunk, int n,
                                           float* __restrict__ dw) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int pair = i / 27, k = i - pair * 27;
  const float* p = part + (int64_t)pair * nchunk * 27 + k;
  float s = 0.f;
  for (int c = 0; c < nchunk; ++c) s += p[(int64_t)c * 27];
  dw[i] += s;
}

template <int CIN, int COUT, int CZT>
static int fwd_launch_t(const ConvArgs& a, cudaStream_t st) {
  using TL = ConvTile<COUT, CZT>;
  constexpr int CC = CIN < CCH ? CIN : CCH;
  const int64_t tiles = (int64_t)a.n0 * ((a.n1 + TL::CY - 1) / TL::CY) * ((a.n2 + CZT - 1) / CZT) * a.nb;
  const size_t smem = (size_t)(((CIN * 27 * COUT + 3) / 4) * 4 + CC * 3 * TL::SY * TL::SZP) * sizeof(float);
  auto kern = conv3d_fwd_kernel<CIN, COUT, CZT>;
  static int per_sm = -1;
  if (per_sm < 0) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TL::THREADS, smem);
    if (per_sm < 1) per_sm = 1;
  }
  const int64_t blocks = std::min<int64_t>(tiles, (int64_t)sm_count() * per_sm * 2);
  kern<<<(unsigned)std::max<int64_t>(blocks, 1), TL::THREADS, smem, st>>>(a);
  return check_launch("conv3d_fwd_kernel");
}

template <int CIN, int COUT>
static int fwd_launch(const ConvArgs& a, cudaStream_t st) {
  if (a.n2 <= 16) return fwd_launch_t<CIN, COUT, 16>(a, st);
  return fwd_launch_t<CIN, COUT, 32>(a, st);
}

}  // namespace gb

using namespace gb;

// the memory pool of the weight-gradient partial sums on the current
// device (created once, release threshold unlimited); null on failure
static cudaMemPool_t part_pool() {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (!pools[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    if (cudaMemPoolCreate(&p, &props) != cudaSuccess) return nullptr;
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[dev] = p;
  }
  return pools[dev];
}

extern "C" {

int gb_conv3d_forward(const float* x, const void* w_bf16, float* y, int64_t nb, int cin, int cout,
                      const int64_t n_c[3], const int pbc_c[3], int accumulate, void* stream) {
  GB_REQUIRE(x && w_bf16 && y && n_c && pbc_c && nb >= 0, "gb_conv3d_forward: bad arguments");
  if (nb == 0) return GB_OK;
  ConvArgs a{x, nullptr, y, reinterpret_cast<const __nv_bfloat16*>(w_bf16), nb, cin, cout,
             (int)n_c[0], (int)n_c[1], (int)n_c[2], pbc_c[0], pbc_c[1], pbc_c[2], accumulate};
  cudaStream_t st = (cudaStream_t)stream;
  if (cin == 1 && cout == 1) return fwd_launch<1, 1>(a, st);
  if (cin == 1 && cout == 16) return fwd_launch<1, 16>(a, st);
  if (cin == 16 && cout == 16) {
    // tensor cores first (periodic grids), then the staged-plane kernel
    if (a.pbc0 && a.pbc1 && a.pbc2) {
      int launched = 0;
      const int rc = conv16_tc_try(x, w_bf16, y, nb, 16, a.n0, a.n1, a.n2, accumulate, st, &launched);
      if (rc != GB_OK || launched) return rc;
    }
    const size_t sm16 = conv16_smem(a);
    if (sm16) return conv16_launch(a, sm16, st);
    return fwd_launch<16, 16>(a, st);
  }
  if (cin == 16 && cout == 1) return fwd_launch<16, 1>(a, st);
  return fail(GB_E_UNSUPPORTED, "gb_conv3d_forward: channel pair not in {(1,1), (1,16), (16,16), (16,1)}");
}

int gb_conv3d_forward_pair(const float* x0, const float* x1, const void* w_bf16, float* y, int64_t nb,
                           const int64_t n_c[3], const int pbc_c[3], void* stream) {
  GB_REQUIRE(x0 && x1 && w_bf16 && y && n_c && pbc_c && nb >= 0, "gb_conv3d_forward_pair: bad arguments");
  if (nb == 0) return GB_OK;
  ConvArgs a{x0, x1, y, reinterpret_cast<const __nv_bfloat16*>(w_bf16), nb, 2, 1,
             (int)n_c[0], (int)n_c[1], (int)n_c[2], pbc_c[0], pbc_c[1], pbc_c[2], 0};
  return fwd_launch<2, 1>(a, (cudaStream_t)stream);
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
  const int nchunk = (int)std::min<int64_t>(chunks, 65535);
  dim3 grid((unsigned)(cin * cout), (unsigned)nchunk);
  // per-CTA partial sums in stream-ordered memory (freed on the stream
  // after the reduction), so concurrent calls on different streams do not
  // share them; from a pool of this library that keeps freed memory, so
  // the thousands of calls of a training run do not map and unmap it
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemPool_t pool = part_pool();
  float* part = nullptr;
  if (!pool || cudaMallocFromPoolAsync(reinterpret_cast<void**>(&part),
                                       (size_t)cin * cout * nchunk * 27 * sizeof(float), pool, st) != cudaSuccess)
    return fail(GB_E_NOMEM, "gb_conv3d_backward_weight: partial-sum allocation failed");
  conv3d_bwd_w_kernel<<<grid, 256, 0, st>>>(x, dy, part, nb, cin, cout, (int)n_c[0], (int)n_c[1], (int)n_c[2],
                                            pbc_c[0], pbc_c[1], pbc_c[2]);
  int rc = check_launch("conv3d_bwd_w_kernel");
  if (rc == GB_OK) {
    const int n = cin * cout * 27;
    conv3d_bwd_w_reduce_kernel<<<(n + 255) / 256, 256, 0, st>>>(part, nchunk, n, dw);
    rc = check_launch("conv3d_bwd_w_reduce_kernel");
  }
  cudaFreeAsync(part, st);
  return rc;
}

}  // extern "C"
