// 16-channel 3x3x3 convolution on a periodic grid on the tcgen05 tensor
// cores: the level-2 layer of the learned preconditioner (no reference
// counterpart; the network stands in for the V-cycle of
// c/fd_preconditioner.c).
//
//   y[b][co][z][p] = sum_{ci < 16} sum_{dz, dy, dx} w[co][ci][dz][dy][dx]
//                                  x[b][ci][z + dz - 1][p + (dy - 1, dx - 1)]
//
// as an implicit GEMM without im2col.  The flattened output planes (band,
// z) are cut into ranges of at most `per` planes, one range per CTA (two
// CTAs per SM, the whole grid in one wave for the Si64 shape).  A CTA walks
// the INPUT planes of its range in order (z_lo - 1 .. z_hi per band
// segment, periodic in z), each staged once into one of two shared-memory
// slots -- padded by the periodic (y, x) halo, split x = hi + lo into RN TF32
// parts, in the canonical K-major no-swizzle layout of the MMA:
// [channel quad][padded point][4 channels], 16 bytes per point, so a core
// matrix is 8 consecutive points (SBO = 128 bytes) and the two channel quads
// of a K = 8 step are one quad stride apart (LBO).  An in-plane tap (dy, dx)
// is the same operand with its start address moved by the tap's offset in
// the padded plane.
//
// The three z taps are folded into N: the B operand of tap (dy, dx) has 48
// rows n = 16 k + co holding w[co][ci][2 - k][dy][dx], and one input plane
// z_in contributes, through one MMA per (tap, channel half, hi / lo), to the
// accumulators of output planes z_in - 1 + k, k = 0, 1, 2.  Output plane o
// of the range owns TMEM columns 16 o .. 16 o + 15 of each 128-point tile,
// so the three accumulators of an input plane are 48 adjacent columns:
//   D[128 points][16 (o .. o + 2)][16 co] += A_tap[128 points][8 ci] . B_tap[48][8 ci]^T
// (tcgen05.mma.cta_group::1.kind::tf32, M = 128, N = 48; N = 16 or 32 at
// the ends of a segment, where fewer output planes are wanted).  Each A
// tile is read from shared memory 36 times per input plane for 48
// accumulator columns, against 108 times for 16 columns when every z tap
// is its own MMA; TMEM is zeroed once, every MMA accumulates.  The weights
// are BF16 and therefore exact TF32 numbers; hi and lo products keep FP32
// accuracy.
//
// Per input plane: one thread per tile (lane 0 of warps 0-1) issues the
// tile's 36 MMAs and commits them to an mbarrier; warps 4-7 meanwhile read
// back (tcgen05.ld.32x32b, one padded point per lane) the output plane that
// the previous input plane completed and store its interior points, and
// warps 2-7 stage the next input plane into the other slot.  Thread 0 alone
// waits on the mbarrier (bounded; a timeout sets the error flag and ends
// the CTA's loop), the rest of the CTA at the barrier that follows.
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

constexpr int CT_THREADS = 256;
constexpr int CT_STAGERS = 192;          // warps 2-7
constexpr int CT_WROWS = 48;             // B rows per tap: (k, co)
constexpr int CT_WFLOATS = 9 * 4 * CT_WROWS * 4;

struct ConvTcArgs {
  const float* x;                 // (nb, 16, n0, n1, n2)
  float* y;                       // (nb, cout, n0, n1, n2)
  const __nv_bfloat16* w;         // [cout][16][27] (plain convolution)
  const float* G;                 // FP32 weights of modes 1-3: [16][6][6][6], [5][5][5], [5][5][5][16]
  int parity;                     // 0: plain; 1, 2: the parity modes; 3: the stride-2 mode (below)
  int64_t total;                  // nb n0 output planes
  int cout, n0, n1, n2;
  int P2, PP, tiles, margin, npts, per, accumulate, nissue;
  uint32_t ncols;
};

// one input plane of a CTA's walk
struct Item {
  int64_t band;
  int zs;        // plane of x (periodic)
  int kl, kh;    // z taps k = kl .. kh feed output planes z_in - 1 + k
  int obase;     // range-local index of output plane z_in - 1 + kl
  int done;      // range-local output plane complete after this item (-1: none)
};

constexpr int CT_MAXITEMS = 24;         // 3 per: every segment adds two halo planes

// the input planes a CTA walks for output planes [g0, g1): per band segment
// z_lo .. z_hi - 1 of outputs, the inputs z_lo - 1 .. z_hi; returns the count
__device__ int build_items(const ConvTcArgs& a, int64_t g0, int64_t g1, Item* items) {
  int n = 0;
  for (int64_t g = g0; g < g1;) {
    const int64_t band = g / a.n0;
    const int zlo = (int)(g - band * a.n0);
    const int zhi = (int)(g1 - g < (int64_t)(a.n0 - zlo) ? zlo + (g1 - g) : a.n0);
    for (int i = 0; i < zhi - zlo + 2 && n < CT_MAXITEMS; ++i, ++n) {
      const int zin = zlo - 1 + i;
      const int lo = max(zlo, zin - 1), hi = min(zhi - 1, zin + 1);
      Item& it = items[n];
      it.band = band;
      it.zs = zin < 0 ? zin + a.n0 : (zin >= a.n0 ? zin - a.n0 : zin);
      it.kl = lo - zin + 1;
      it.kh = hi - zin + 1;
      it.obase = (int)(g - g0) + (lo - zlo);
      it.done = i >= 2 ? (int)(g - g0) + (i - 2) : -1;
    }
    g += zhi - zlo;
  }
  return n;
}

// the FP32 weight behind shared-memory element e of the B operands
// ([9 taps][4 quads][48 rows][4]): row n = 16 k + co, input channel
// ci = 4 quad + i, z tap 2 - k; the one global load of each element
__device__ __forceinline__ float weight_raw(const ConvTcArgs& a, int e) {
  const int tap = e / (4 * CT_WROWS * 4), r = e % (4 * CT_WROWS * 4);
  const int q = r / (CT_WROWS * 4), n = (r >> 2) % CT_WROWS, i = r & 3;
  const int k = n >> 4, co = n & 15, ci = 4 * q + i;
  const int e0 = 1 - k, e1 = tap / 3 - 1, e2 = tap % 3 - 1;   // coarse offset of the tap
  if (a.parity == 0)
    return co < a.cout ? __bfloat162float(a.w[(co * 16 + ci) * 27 + 9 * (2 - k) + tap]) : 0.f;
  if (a.parity == 3) {
    // output channel co, input parity ci & 7: fine offset d = 2e + p'
    const int pp = ci & 7;
    const int d0 = 2 * e0 + (pp >> 2), d1 = 2 * e1 + ((pp >> 1) & 1), d2 = 2 * e2 + (pp & 1);
    return (d0 <= 2 && d1 <= 2 && d2 <= 2) ? __ldg(a.G + (((d0 + 2) * 5 + (d1 + 2)) * 5 + (d2 + 2)) * 16 + co) : 0.f;
  }
  const int par = co & 7;
  if (a.parity == 1) {
    const int tx = (par >> 2) - 2 * e0 + 2, ty = ((par >> 1) & 1) - 2 * e1 + 2, tz = (par & 1) - 2 * e2 + 2;
    return (tx < 5 && ty < 5 && tz < 5) ? __ldg(a.G + ci * 216 + (tx * 6 + ty) * 6 + tz) : 0.f;
  }
  if (ci >= 8) return 0.f;
  // fine offset d = 2e + p' - par of input parity p' = ci
  const int d0 = 2 * e0 + (ci >> 2) - (par >> 2), d1 = 2 * e1 + ((ci >> 1) & 1) - ((par >> 1) & 1);
  const int d2 = 2 * e2 + (ci & 1) - (par & 1);
  return (d0 >= -2 && d0 <= 2 && d1 >= -2 && d1 <= 2 && d2 >= -2 && d2 <= 2)
             ? __ldg(a.G + ((d0 + 2) * 5 + (d1 + 2)) * 5 + (d2 + 2))
             : 0.f;
}

__global__ void __launch_bounds__(CT_THREADS, 2) conv16_tc_kernel(const ConvTcArgs a) {
  extern __shared__ __align__(128) unsigned char ctc_smem[];
  float* sW = reinterpret_cast<float*>(ctc_smem);              // [9 taps][4 quads][48 rows][4]
  float* Xhi = sW + CT_WFLOATS;                                 // [2 slots][4 quads][npts][4]
  float* Xlo = Xhi + 2 * 4 * a.npts * 4;
  uint64_t* done = reinterpret_cast<uint64_t*>(Xlo + 2 * 4 * a.npts * 4);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  int* sfail = reinterpret_cast<int*>(tslot + 1);
  int* snit = sfail + 1;
  Item* items = reinterpret_cast<Item*>(done + 3);           // [CT_MAXITEMS]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int n0 = a.n0, n1 = a.n1, n2 = a.n2, P2 = a.P2, PP = a.PP;
  const int64_t g0 = (int64_t)blockIdx.x * a.per, g1 = min(a.total, g0 + a.per);

  {
    // weights: all of a thread's 27 loads are issued before any is used
    // (one L2 round trip for the prologue instead of 27 in a row)
    constexpr int WPER = CT_WFLOATS / CT_THREADS;
    float wv[WPER];
#pragma unroll
    for (int u = 0; u < WPER; ++u) wv[u] = weight_raw(a, tid + u * CT_THREADS);
#pragma unroll
    for (int u = 0; u < WPER; ++u) {
      const int e = tid + u * CT_THREADS;
      const float g = wv[u];
      if (a.parity) {
        // hi part in rows 0-7 (parity modes) or K step 0 (stride mode), lo part in the rest
        const int n = (e >> 2) % CT_WROWS, ci = 4 * ((e % (4 * CT_WROWS * 4)) / (CT_WROWS * 4)) + (e & 3);
        const bool hi = a.parity == 3 ? ci < 8 : (n & 15) < 8;
        const float h = rn_tf32(g);
        sW[e] = hi ? h : rn_tf32(g - h);
      } else {
        sW[e] = g;
      }
    }
  }
  // margins of both slots and every quad: zero (only dropped halo outputs read them)
  for (int e = tid; e < 8 * 2 * a.margin; e += CT_THREADS) {
    const int sq = e / (2 * a.margin), m = e % (2 * a.margin);
    const int pt = m < a.margin ? m : a.margin + PP + (m - a.margin);
    reinterpret_cast<float4*>(Xhi)[sq * a.npts + pt] = make_float4(0.f, 0.f, 0.f, 0.f);
    reinterpret_cast<float4*>(Xlo)[sq * a.npts + pt] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  if (tid == 0) {
    mbar_init(done, a.nissue);
    mbar_fence_init();
    *sfail = 0;
    *snit = build_items(a, g0, g1, items);
  }
  if (warp == 1) {
    tmem_alloc(tslot, a.ncols);
    tmem_relinquish();
  }
  const int64_t nplane = (int64_t)n1 * n2, nvol = nplane * n0;
  // stage the input plane of `it` into slot `sl`, split hi / lo (warps 2-7):
  // a thread takes padded points r, r + 192 (one index division each) and
  // loads all 16 channels of both before it writes any
  const bool gather8 = a.parity >= 2;
  auto stage = [&](const Item& it, int sl) {
    // channel c of a plain input: x[band][c][zs]; the eight parity channels
    // p' of a fine input (2 n0, 2 n1, 2 n2): x[band][2 zs + p'0][2 ys + p'1][2 xs + p'2]
    const float* xb = gather8 ? a.x + it.band * 8 * nvol + (int64_t)(2 * it.zs) * 4 * nplane
                              : a.x + it.band * 16 * nvol + it.zs * nplane;
    for (int r0 = tid - 64; r0 < PP; r0 += 2 * CT_STAGERS) {
      float v[2][16];
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int r = r0 + j * CT_STAGERS;
        if (r < PP) {
          const int yy = r / P2, xx = r - yy * P2;
          int ys = yy - 1, xs = xx - 1;
          ys = ys < 0 ? ys + n1 : (ys >= n1 ? ys - n1 : ys);
          xs = xs < 0 ? xs + n2 : (xs >= n2 ? xs - n2 : xs);
          if (gather8) {
            const int64_t f2 = 2 * n2, fpl = 4 * nplane;
            const float* src = xb + (int64_t)(2 * ys) * f2 + 2 * xs;
#pragma unroll
            for (int c = 0; c < 8; ++c) v[j][c] = __ldg(src + (c >> 2) * fpl + ((c >> 1) & 1) * f2 + (c & 1));
          } else {
            const float* src = xb + (int64_t)ys * n2 + xs;
#pragma unroll
            for (int c = 0; c < 16; ++c) v[j][c] = __ldg(src + c * nvol);
          }
        }
      }
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int r = r0 + j * CT_STAGERS;
        if (r < PP) {
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            if (gather8 && q >= 2) break;
            float h[4], l[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              h[i] = rn_tf32(v[j][4 * q + i]);
              l[i] = rn_tf32(v[j][4 * q + i] - h[i]);
            }
            const int pt = (sl * 4 + q) * a.npts + a.margin + r;
            reinterpret_cast<float4*>(Xhi)[pt] = make_float4(h[0], h[1], h[2], h[3]);
            reinterpret_cast<float4*>(Xlo)[pt] = make_float4(l[0], l[1], l[2], l[3]);
          }
        }
      }
    }
  };
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  // store output plane `o` (range-local) of every tile (warps 4-7)
  auto epilogue = [&](int o) {
    const int64_t g = g0 + o, band = g / n0;
    const int z = (int)(g - band * n0);
    const int q4 = warp & 3;
    for (int t = 0; t < a.tiles; ++t) {
      uint32_t r[16];
      tmem_ld16(tmem + (uint32_t)(16 * (t * a.per + o)) + ((uint32_t)(32 * q4) << 16), r);
      tmem_wait_ld();
      const int lin = t * 128 + 32 * q4 + lane;          // padded point of the plane
      const int yy = lin / P2, xx = lin % P2;
      if (lin < PP && yy >= 1 && yy <= n1 && xx >= 1 && xx <= n2) {
        if (a.parity == 1 || a.parity == 2) {
          // fine grid (2 n0, 2 n1, 2 n2): point 2 J + par gets high + low part
          const int64_t f2 = 2 * n2, fpl = 4 * nplane;
          float* yp = a.y + band * 8 * nvol + (int64_t)(2 * z) * fpl + (int64_t)(2 * (yy - 1)) * f2 + 2 * (xx - 1);
#pragma unroll
          for (int par = 0; par < 8; ++par) {
            float* o = yp + (par >> 2) * fpl + ((par >> 1) & 1) * f2 + (par & 1);
            const float v = __uint_as_float(r[par]) + __uint_as_float(r[par + 8]);
            if (a.accumulate) *o += v;
            else *o = v;
          }
        } else {
          float* yp = a.y + (band * a.cout) * nvol + z * nplane + (int64_t)(yy - 1) * n2 + (xx - 1);
          for (int co = 0; co < a.cout; ++co) {
            const float v = __uint_as_float(r[co]);
            if (a.accumulate) yp[co * nvol] += v;
            else yp[co * nvol] = v;
          }
        }
      }
    }
  };
  const int nit = *snit;
  if (warp >= 4) {
    for (uint32_t c = 0; c < a.ncols; c += 16) tmem_st16_zero(tmem + c + ((uint32_t)(32 * (warp & 3)) << 16));
    tmem_wait_st();
  }
  if (warp >= 2 && nit > 0) stage(items[0], 0);
  const uint32_t idesc0 = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(128 >> 4) << 24);
  const uint32_t qstride = (uint32_t)a.npts * 16u;
  uint32_t phase = 0;
  for (int i = 0; i < nit; ++i) {
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (*sfail) break;
    if (warp < a.nissue && lane == 0) {
      // issuer w feeds tiles w, w + nissue, ... (one accumulator set per
      // tile, so each tile's MMAs come from one thread, in order); the
      // descriptors differ only in the start address (bits 0-13, 16-byte
      // units, addresses < 256 KB)
      const Item& it = items[i];
      const uint32_t N = 16u * (uint32_t)(it.kh - it.kl + 1);
      const uint32_t idesc = idesc0 | ((N >> 3) << 17);
      const uint64_t ah0 = sdesc(su32(Xhi), qstride, 128, 0u);
      const uint64_t al0 = sdesc(su32(Xlo), qstride, 128, 0u);
      const uint64_t bw0 = sdesc(su32(sW), CT_WROWS * 16, 128, 0u) + (uint64_t)(16 * it.kl);
      const uint32_t sbase = (uint32_t)((i & 1) * 4 * a.npts);
      const int rowoff[3] = {-P2, 0, P2};
      for (int t = warp; t < a.tiles; t += a.nissue) {
        const uint32_t d = tmem + (uint32_t)(16 * (t * a.per + it.obase));
        const int tb = a.margin + t * 128;
#pragma unroll
        for (int tap = 0; tap < 9; ++tap) {
          const uint32_t off = sbase + (uint32_t)(tb + rowoff[tap / 3] + (tap % 3 - 1));
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            if (c == 1 && a.parity == 2) break;   // eight input channels: one K = 8 step
            // stride mode: both K steps read the eight staged channels
            const uint64_t delta = off + (a.parity == 3 ? 0u : 2u * c * (uint32_t)a.npts);
            const uint64_t bw = bw0 + (uint64_t)(tap * 4 * CT_WROWS + c * 2 * CT_WROWS);
            mma_tf32(d, ah0 + delta, bw, idesc, 1u);
            mma_tf32(d, al0 + delta, bw, idesc, 1u);
          }
        }
      }
      mma_commit(done);
    }
    // the output plane the previous input plane completed (its columns are
    // not among those this plane's MMAs write)
    if (warp >= 4 && i > 0) {
      const int o = items[i - 1].done;
      if (o >= 0) epilogue(o);
    }
    // the next input plane goes to the slot the previous plane's MMAs read
    if (warp >= 2 && i + 1 < nit) stage(items[i + 1], (i + 1) & 1);
    // one thread waits for this plane's MMAs; the others wait at the next
    // barrier, which issues no instructions (a spinning CTA starves the
    // staging warps of issue slots)
    if (tid == 0 && !mbar_wait(done, phase)) {
      atomicCAS(&g_conv_tc_error, 0, 301);
      *sfail = 1;
    }
    phase ^= 1u;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (*sfail) {
    // MMAs may still be in flight: give them a bounded wait before the
    // accumulators are freed
    if (tid == 0) mbar_wait(done, phase ^ 1u);
  } else if (warp >= 4 && nit > 0) {
    const int o = items[nit - 1].done;
    if (o >= 0) epilogue(o);
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
static int conv_tc_launch(ConvTcArgs a, int64_t nb, int n0, int n1, int n2, cudaStream_t st, int* launched) {
  *launched = 0;
  if (a.cout < 1 || a.cout > 16 || nb < 1 || n0 < 2 || n1 < 2 || n2 < 2) return GB_OK;
  a.total = nb * n0;
  a.n0 = n0; a.n1 = n1; a.n2 = n2;
  a.P2 = n2 + 2;
  a.PP = (n1 + 2) * a.P2;
  a.tiles = (a.PP + 127) / 128;
  if (a.tiles > 16) return GB_OK;
  const int m = std::max(a.P2 + 1, a.tiles * 128 - a.PP + a.P2 + 1);
  a.margin = (m + 7) / 8 * 8;
  a.npts = a.PP + 2 * a.margin;                   // one slot of one quad
  if (a.npts > 16383) return GB_OK;
  // output planes per CTA: 16 TMEM columns each per tile, at most 256
  // columns so that two CTAs share an SM
  a.per = std::min(8, 256 / (16 * a.tiles));
  const int64_t nblk = (a.total + a.per - 1) / a.per;
  if (nblk > 0x7fffffff) return GB_OK;
  a.nissue = std::min(2, a.tiles);
  uint32_t nc = 32;
  while (nc < (uint32_t)(16 * a.tiles * a.per)) nc *= 2;
  a.ncols = nc;
  const size_t smem = (size_t)(CT_WFLOATS + 2 * 2 * 4 * a.npts * 4) * sizeof(float) + 24 +
                      CT_MAXITEMS * sizeof(Item);
  if (smem > 220 * 1024) return GB_OK;
  static size_t attr = 0;
  if (smem > attr) {
    cudaFuncSetAttribute(conv16_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr = smem;
  }
  conv16_tc_kernel<<<(unsigned)nblk, CT_THREADS, smem, st>>>(a);
  *launched = 1;
  return check_launch(a.parity ? "conv16_tc_kernel(parity)" : "conv16_tc_kernel");
}

int conv16_tc_try(const float* x, const void* w_bf16, float* y, int64_t nb, int cout, int n0, int n1, int n2,
                  int accumulate, cudaStream_t st, int* launched) {
  ConvTcArgs a{};
  a.x = x;
  a.y = y;
  a.w = reinterpret_cast<const __nv_bfloat16*>(w_bf16);
  a.cout = cout;
  a.accumulate = accumulate;
  return conv_tc_launch(a, nb, n0, n1, n2, st, launched);
}

// Parity mode (the coarse part of level 1 of the folded learned
// preconditioner, as in fold_parity16_kernel):
//   y[2J + par] += sum_c sum_{e in {-1,0,1}^3} G[c][par - 2e + 2] xc[c][J + e]
// on the coarse grid (n0, n1, n2), y the fine grid (2 n0, 2 n1, 2 n2),
// par in {0,1}^3 (axis 0 the slowest), tap index 5 (odd parity, e = -1)
// zero.  It is the 16-channel convolution above with the eight parities as
// output channels; G is FP32 (composite weights, not TF32 numbers), so B
// rows 8-15 carry the TF32 low parts of rows 0-7 and the epilogue adds the
// two accumulators: every product of the hi / lo parts of both operands is
// formed, FP32 accuracy with no extra MMA.
int conv_parity_tc_try(const float* xc, const float* G, float* y, int64_t nb, int n0, int n1, int n2,
                       cudaStream_t st, int* launched) {
  ConvTcArgs a{};
  a.x = xc;
  a.y = y;
  a.G = G;
  a.parity = 1;
  a.cout = 16;
  a.accumulate = 1;
  return conv_tc_launch(a, nb, n0, n1, n2, st, launched);
}

// The fine 5^3 stencil of the same level in parity form (mode 2):
//   y[2J + par] = sum_d F[d] xf[2J + par + d],  d in [-2, 2]^3,
// xf and y on the fine grid (2 n0, 2 n1, 2 n2).  Writing 2J + par + d =
// 2 (J + e) + p' (e in {-1,0,1}^3, p' in {0,1}^3, one way for each d) makes
// it a 3^3 convolution on the coarse grid from the eight parity sub-grids
// xf[2J + p'] (gathered while staging) to the eight output parities, with
// weights F[2e + p' - par] (zero outside [-2, 2]^3): one K = 8 step per tap.
// y is written (not accumulated).
int conv_fine5_tc_try(const float* xf, const float* F, float* y, int64_t nb, int n0, int n1, int n2,
                      cudaStream_t st, int* launched) {
  ConvTcArgs a{};
  a.x = xf;
  a.y = y;
  a.G = F;
  a.parity = 2;
  a.cout = 16;
  a.accumulate = 0;
  return conv_tc_launch(a, nb, n0, n1, n2, st, launched);
}

// The stride-2 level-1 -> level-2 stencil of the folded network (mode 3):
//   y[c][J] = sum_{d in [-2,2]^3} Q[d][c] xf[2J + d],  16 output channels,
// xf on the fine grid (2 n0, 2 n1, 2 n2), y on the coarse grid.  With
// d = 2e + p' (e in {-1,0,1}^3, p' in {0,1}^3; d = 3 has no weight) it is
// a 3^3 convolution from the eight parity sub-grids of xf to 16 channels;
// the FP32 weights enter as their TF32 high part in K step 0 and their low
// part in K step 1, both over the same staged channels.  y is written.
int conv_stride_tc_try(const float* xf, const float* Q, float* y, int64_t nb, int n0, int n1, int n2,
                       cudaStream_t st, int* launched) {
  ConvTcArgs a{};
  a.x = xf;
  a.y = y;
  a.G = Q;
  a.parity = 3;
  a.cout = 16;
  a.accumulate = 0;
  return conv_tc_launch(a, nb, n0, n1, n2, st, launched);
}

// whether conv_tc_launch takes a coarse grid of this shape
bool conv_tc_fits(int n0, int n1, int n2) {
  if (n0 < 2 || n1 < 2 || n2 < 2) return false;
  const int P2 = n2 + 2, PP = (n1 + 2) * P2, tiles = (PP + 127) / 128;
  if (tiles > 16) return false;
  const int m = std::max(P2 + 1, tiles * 128 - PP + P2 + 1);
  const int npts = PP + 2 * ((m + 7) / 8 * 8);
  if (npts > 16383) return false;
  const size_t smem = (size_t)(CT_WFLOATS + 2 * 2 * 4 * npts * 4) * sizeof(float) + 24 + CT_MAXITEMS * sizeof(Item);
  return smem <= 220 * 1024;
}

}  // namespace gb
