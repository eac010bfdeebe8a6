// Folded inference of the learned preconditioner on periodic grids (no
// reference counterpart: the network stands in for the V-cycle of
// c/fd_preconditioner.c).
//
// The network is linear, so on a periodic grid its layers compose exactly
// into three stencils over single-channel inputs plus the 16-channel
// level-2 convolution (which stays as it is):
//
//   r2[c][I] = sum_{d in [-2,2]^3} Q[c][d] r1[2I + d]           fold_stride
//              (Q = restriction o conv_a: 1 -> 16 channels, stride 2)
//   b1[p]    = sum_{d in [-2,2]^3} C1[d] r1[p + d]               fold_fine<2, 16>
//            + sum_c sum_{e in {-1,0,1}^3} G[c][(p mod 2) - 2e] a2[c][p/2 + e]
//              (C1 = conv_c o conv_a; G = conv_c o interpolation)
//   y[p]     = sum_{d in [-1,1]^3} W0[d] x[p + d]                fold_fine<1, 1>
//            + sum_{e} H[(p mod 2) - 2e] b1[p/2 + e]
//              (H = conv_p o interpolation, the step folded in)
//
// so the 16-channel level-1 tensors (and the interpolated level-0 grid) are
// never written.  Index conventions: fine point p sits on coarse point p/2
// (periodic grids of even size); G and H are stored [c][tx][ty][tz] with
// t = d + 2 in 0..5 (d = (p mod 2) - 2e in -2..3; t = 5 is zero).  The
// composite weights are extracted on the host side by applying the unfolded
// network to delta inputs, so they inherit its BF16 weights and transfer
// coefficients exactly.
//
// Level 1 runs as two launches: fold_fine_kernel<2, 0> writes the 5^3 fine
// part, then fold_parity16_kernel adds the 16-channel coarse part as a
// parity convolution (one thread per coarse point, all 8 fine points of its
// parity block from one load of each channel's 27 neighbours).
//
// The kernels read their neighbourhoods through L1 (__ldg) with the lanes
// of a warp along a grid row (coalesced), keep the weights in shared memory
// and give every thread a column of 4 output rows (fold_fine: each loaded
// input row serves all of them) or two neighbouring coarse points with all
// 16 channels (fold_stride).  FP32 throughout.
#include <algorithm>
#include "internal.cuh"

namespace gb {

// the parity convolution on the tensor cores (conv_tc.cu); *launched = 0
// when the grid does not fit its layout
int conv_parity_tc_try(const float* xc, const float* G, float* y, int64_t nb, int n0, int n1, int n2,
                       cudaStream_t st, int* launched);
int conv_fine5_tc_try(const float* xf, const float* F, float* y, int64_t nb, int n0, int n1, int n2,
                      cudaStream_t st, int* launched);
int conv_stride_tc_try(const float* xf, const float* Q, float* y, int64_t nb, int n0, int n1, int n2,
                       cudaStream_t st, int* launched);
bool conv_tc_fits(int n0, int n1, int n2);

namespace {

// periodic index for -n <= x < 2n (every offset these kernels form stays in
// that range: rows of at least PXF + 2 points are required)
__device__ __forceinline__ int pw(int x, int n) { return x < 0 ? x + n : (x >= n ? x - n : x); }

struct FoldArgs {
  const float* xf;   // (nb, n0, n1, n2)
  const float* xc;   // (nb, CC, n0/2, n1/2, n2/2)
  float* y;          // (nb, n0, n1, n2)
  const float* F;    // (2 RH + 1)^3
  const float* G;    // CC x 216
  int64_t nb;
  int n0, n1, n2;
};

constexpr int PXF = 8;   // minimum row length beyond the 2-point halo
constexpr int JB = 4;    // output rows per thread (axis 1)

// launch: block (32, 8) = 32 points of a row x 8 row blocks, grid
// (row chunks x row-block groups, planes, bands): no index divisions beyond
// one small one per thread; offsets inside a band are 32-bit
// thread = one point k of a row (lanes run along the row: coalesced loads)
// and JB consecutive rows j0 .. j0 + JB - 1 of one plane i; every input row
// it loads serves all the outputs it touches
template <int RH, int CC>
__global__ void __launch_bounds__(256, CC > 1 ? 2 : 3) fold_fine_kernel(const FoldArgs a) {
  constexpr int FW = 2 * RH + 1;
  constexpr int NR = JB + 2 * RH;          // input rows per plane
  __shared__ float sF[FW * FW * FW];
  __shared__ float sG[CC > 0 ? CC * 216 : 1];
  const int tid = threadIdx.y * 32 + threadIdx.x;
  for (int e = tid; e < FW * FW * FW; e += 256) sF[e] = a.F[e];
  if constexpr (CC > 0)
    for (int e = tid; e < CC * 216; e += 256) sG[e] = a.G[e];
  __syncthreads();
  const int n0 = a.n0, n1 = a.n1, n2 = a.n2;
  const int m0 = n0 >> 1, m1 = n1 >> 1, m2 = n2 >> 1;
  const int nkx = (n2 + 31) >> 5;
  const int k = (blockIdx.x % nkx) * 32 + threadIdx.x;
  const int j0 = ((blockIdx.x / nkx) * 8 + threadIdx.y) * JB;
  const int i = blockIdx.y;
  const int64_t b = blockIdx.z;
  if (k >= n2 || j0 >= n1) return;
  const int plane = n1 * n2, cplane = m1 * m2;
  float acc[JB];
#pragma unroll
  for (int q = 0; q < JB; ++q) acc[q] = 0.f;
  int kk[FW];
#pragma unroll
  for (int m = 0; m < FW; ++m) kk[m] = pw(k - RH + m, n2);
  const float* xb = a.xf + b * n0 * (int64_t)plane;
#pragma unroll 1
  for (int dx = -RH; dx <= RH; ++dx) {
    const float* pl = xb + pw(i + dx, n0) * plane;
    const float* f = sF + (dx + RH) * FW * FW;
    float fr[FW * FW];
#pragma unroll
    for (int t = 0; t < FW * FW; ++t) fr[t] = f[t];
#pragma unroll
    for (int rr = 0; rr < NR; ++rr) {
      const float* rp = pl + pw(j0 - RH + rr, n1) * n2;
      float v[FW];
#pragma unroll
      for (int m = 0; m < FW; ++m) v[m] = __ldg(rp + kk[m]);
#pragma unroll
      for (int q = 0; q < JB; ++q) {
        const int dy = rr - RH - q;          // compile-time after unrolling
        if (dy < -RH || dy > RH) continue;
#pragma unroll
        for (int m = 0; m < FW; ++m) acc[q] = fmaf(fr[(dy + RH) * FW + m], v[m], acc[q]);
      }
    }
  }
  // coarse part: coarse rows j0/2 - 1 .. j0/2 + JB/2, columns k/2 - 1 .. k/2 + 1;
  // the weights one (channel, plane offset) needs -- 5 row parities x 3
  // column offsets for this thread's column parity -- go to registers once
  if constexpr (CC > 0) {
  const int I0 = i >> 1, J0 = j0 >> 1, K0 = k >> 1;
  const int px = i & 1, pz = k & 1;
  int kc[3];
#pragma unroll
  for (int m = 0; m < 3; ++m) kc[m] = pw(K0 - 1 + m, m2);
  int crow[JB / 2 + 2];
#pragma unroll
  for (int rr = 0; rr < JB / 2 + 2; ++rr) crow[rr] = pw(J0 - 1 + rr, m1) * m2;
  const float* cb = a.xc + b * CC * (int64_t)m0 * cplane;
#pragma unroll 1
  for (int c = 0; c < CC; ++c) {
    const float* cc = cb + c * m0 * cplane;
    const float* gc = sG + c * 216;
#pragma unroll
    for (int ex = -1; ex <= 1; ++ex) {
      const int tx = px - 2 * ex + 2;
      if (tx > 4) continue;
      float wz[5][3];                        // [ty][ez + 1]; tz = pz - 2 ez + 2
#pragma unroll
      for (int ty = 0; ty < 5; ++ty)
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          const int tz = pz - 2 * (m - 1) + 2;
          wz[ty][m] = tz <= 4 ? gc[(tx * 6 + ty) * 6 + tz] : 0.f;
        }
      const float* cpl = cc + pw(I0 + ex, m0) * cplane;
#pragma unroll
      for (int rr = 0; rr < JB / 2 + 2; ++rr) {
        float v[3];
#pragma unroll
        for (int m = 0; m < 3; ++m) v[m] = __ldg(cpl + crow[rr] + kc[m]);
#pragma unroll
        for (int q = 0; q < JB; ++q) {
          // output row j0 + q sits on coarse row J0 + q/2 with parity q & 1
          const int ey = rr - 1 - q / 2;
          if (ey < -1 || ey > 1) continue;
          const int ty = (q & 1) - 2 * ey + 2;   // compile-time
          if (ty > 4) continue;
#pragma unroll
          for (int m = 0; m < 3; ++m) acc[q] = fmaf(wz[ty][m], v[m], acc[q]);
        }
      }
    }
  }
  }
  float* yp = a.y + b * n0 * (int64_t)plane + i * plane + k;
#pragma unroll
  for (int q = 0; q < JB; ++q)
    if (j0 + q < n1) yp[(j0 + q) * n2] = acc[q];
}

// Level 0 (rh = 1, one coarse channel), marching along axis 0.  A CTA owns
// TY full rows j0 .. j0 + TY - 1 (TY even, n1 % TY == 0) of one band over a
// chunk of planes; a thread owns the 4 points k .. k + 3 of an even row j
// and of the odd row j + 1 (8 outputs).  Each input plane p is staged once
// (cp.async into a ring of three slots: the copy of plane p + 2 is issued
// right after the single barrier of the step) and every thread adds
// W0[dx][dy][dz] x[p][.][.] over its four input rows j - 1 .. j + 2 to the
// output planes p + 1 - dx held in a register queue -- 12 shared loads and
// 216 FMAs per plane, the 27 weights in registers.  When output plane
// o = p - 1 is complete, the coarse part
// sum_e H[(o%2) - 2ex][(j%2) - 2ey][..] b1[o/2 + e] is added from staged
// coarse planes (a ring of 4; zero taps of the parities skipped; both rows
// read the same three coarse rows) and the 8 points are stored as two
// 16-byte vectors.  Row pitches FP, CP (floats) are chosen on the host so
// that the lanes of a quarter warp (fine, 16-byte loads) or half warp
// (coarse, 8-byte loads) hit distinct banks.  Requires n2 % 4 == 0 and
// periodic axes.
struct Fold0Cfg {
  int TY, FP, CP, nch;
};

__global__ void __launch_bounds__(512) fold0_pair_kernel(const FoldArgs a, const Fold0Cfg cfg) {
  __shared__ __align__(16) float sH[36 * 8];           // [tx][ty][tz 0..7]: H, tz >= 6 zero
  extern __shared__ __align__(16) float fm_smem[];
  const int n0 = a.n0, n1 = a.n1, n2 = a.n2;
  const int m0 = n0 >> 1, m1 = n1 >> 1, m2 = n2 >> 1;
  const int TY = cfg.TY, FP = cfg.FP, CP = cfg.CP;    // fine column c at 4 + c, coarse at 5 + c
  const int FR = TY + 2, CR = TY / 2 + 2;
  float* fslot = fm_smem;                              // [3][FR][FP]
  float* cslot = fm_smem + 3 * FR * FP;                // [4][CR][CP]
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int e = tid; e < 36 * 8; e += nt) sH[e] = (e & 7) < 6 ? a.G[(e >> 3) * 6 + (e & 7)] : 0.f;
  float W[27];
#pragma unroll
  for (int e = 0; e < 27; ++e) W[e] = __ldg(a.F + e);
  const int ngx = n2 >> 2;
  const int gx = tid % ngx, rp = tid / ngx;
  const int j0 = blockIdx.y * TY;
  const int j = j0 + 2 * rp, k = 4 * gx;
  const int64_t b = blockIdx.z;
  const int o_beg = (int)((int64_t)blockIdx.x * n0 / cfg.nch), o_end = (int)((int64_t)(blockIdx.x + 1) * n0 / cfg.nch);
  const float* xb = a.xf + b * n0 * (int64_t)n1 * n2;
  const float* cb = a.xc + b * (int64_t)m0 * m1 * m2;

  // the (row, 16-byte chunk) pieces of a staged plane this thread copies:
  // pieces tid, tid + nt, ... (at most 4 per thread), offsets fixed per CTA
  int f_src[4], f_dst[4];
  int nf = 0;
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int e = tid + u * nt;
    f_src[u] = 0;
    f_dst[u] = 0;
    if (e < FR * ngx) {
      const int r = e / ngx, c = e % ngx;
      f_src[u] = pw(j0 - 1 + r, n1) * n2 + 4 * c;
      f_dst[u] = r * FP + 4 + 4 * c;
      nf = u + 1;
    }
  }
  auto stage_fine = [&](int p, float* dst) {
    const float* pl = xb + (int64_t)pw(p, n0) * n1 * n2;
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (u < nf) cp_async16(dst + f_dst[u], pl + f_src[u]);
    // the two periodic halo columns of every row
    for (int e = tid; e < 2 * FR; e += nt) {
      const int r = e >> 1, row = pw(j0 - 1 + r, n1) * n2;
      if (e & 1) cp_async4(dst + r * FP + 4 + n2, pl + row);       // column n2
      else cp_async4(dst + r * FP + 3, pl + row + n2 - 1);         // column -1
    }
  };
  // the coarse elements (row r, column c = -1 .. m2) this thread copies
  int c_src[4], c_dst[4];
  int ncp = 0;
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int e = tid + u * nt;
    c_src[u] = 0;
    c_dst[u] = 0;
    if (e < CR * (m2 + 2)) {
      const int r = e / (m2 + 2), c = e % (m2 + 2) - 1;
      c_src[u] = pw((j0 >> 1) - 1 + r, m1) * m2 + pw(c, m2);
      c_dst[u] = r * CP + 5 + c;
      ncp = u + 1;
    }
  }
  auto stage_coarse = [&](int C, float* dst) {
    const float* pl = cb + (int64_t)pw(C, m0) * m1 * m2;
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (u < ncp) cp_async4(dst + c_dst[u], pl + c_src[u]);
  };
  auto cidx = [](int C) { return (C + 4) & 3; };

  // prologue: planes o_beg - 1 and o_beg, coarse planes around o_beg / 2
  int c_last = (o_beg >> 1) + 1;
  stage_fine(o_beg - 1, fslot);
  for (int C = (o_beg >> 1) - 1; C <= c_last; ++C) stage_coarse(C, cslot + cidx(C) * CR * CP);
  cp_async_commit();
  stage_fine(o_beg, fslot + FR * FP);
  cp_async_commit();

  // output planes p - 1, p, p + 1 (rows j, j + 1) of the step with input p
  float qa[2][4], qb[2][4], qc[2][4];
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int q = 0; q < 4; ++q) qa[r][q] = qb[r][q] = qc[r][q] = 0.f;
  const bool act = rp < TY / 2;

  const int nsteps = o_end - o_beg + 2;
  for (int st = 0; st < nsteps; ++st) {
    const int p = o_beg - 1 + st;
    cp_async_wait<1>();
    __syncthreads();
    // refill: fine plane p + 2 into the slot step st - 1 used, and the coarse
    // plane the output completed two steps later needs
    if (p + 2 <= o_end) {
      stage_fine(p + 2, fslot + ((st + 2) % 3) * FR * FP);
      const int Cn = ((p + 1) >> 1) + 1;
      if (Cn > c_last) {
        stage_coarse(Cn, cslot + cidx(Cn) * CR * CP);
        c_last = Cn;
      }
    }
    cp_async_commit();
    if (act) {
      const float* F = fslot + (st % 3) * FR * FP;
#pragma unroll
      for (int R = 0; R < 4; ++R) {
        // input row j - 1 + R: dy = R for row j, R - 1 for row j + 1
        const float* rpp = F + (2 * rp + R) * FP + 4 + k;
        const float4 l4 = *reinterpret_cast<const float4*>(rpp - 4);
        const float4 m4 = *reinterpret_cast<const float4*>(rpp);
        const float4 r4 = *reinterpret_cast<const float4*>(rpp + 4);
        const float v[6] = {l4.w, m4.x, m4.y, m4.z, m4.w, r4.x};
#pragma unroll
        for (int dx = 0; dx < 3; ++dx) {
          // plane p is x[o + dx - 1] of output o = p + 1 - dx
          float(&Q)[2][4] = dx == 2 ? qa : (dx == 1 ? qb : qc);
#pragma unroll
          for (int dz = 0; dz < 3; ++dz) {
            if (R <= 2) {
              const float w = W[dx * 9 + R * 3 + dz];
#pragma unroll
              for (int q = 0; q < 4; ++q) Q[0][q] = fmaf(w, v[q + dz], Q[0][q]);
            }
            if (R >= 1) {
              const float w = W[dx * 9 + (R - 1) * 3 + dz];
#pragma unroll
              for (int q = 0; q < 4; ++q) Q[1][q] = fmaf(w, v[q + dz], Q[1][q]);
            }
          }
        }
      }
      const int o = p - 1;
      if (o >= o_beg) {
        // coarse part of output plane o; coarse row of j and j + 1: j / 2
        const int px = o & 1, I0 = o >> 1, K0 = k >> 1;
#pragma unroll
        for (int ex = -1; ex <= 1; ++ex) {
          const int tx = px - 2 * ex + 2;
          if (tx > 4) continue;
          const float* Cs = cslot + cidx(I0 + ex) * CR * CP;
          float c[3][4];                                  // coarse rows J - 1 .. J + 1, cols K0 - 1 .. K0 + 2
#pragma unroll
          for (int e = 0; e < 3; ++e) {
            const float* cr = Cs + (rp + e) * CP + 4 + K0;
            const float2 u = *reinterpret_cast<const float2*>(cr), w = *reinterpret_cast<const float2*>(cr + 2);
            c[e][0] = u.x; c[e][1] = u.y; c[e][2] = w.x; c[e][3] = w.y;
          }
          const float* gt = sH + tx * 48;
#pragma unroll
          for (int e = 0; e < 5; ++e) {
            // e = 0, 1, 2: row j (tyy = 4, 2, 0 for ey = -1, 0, 1); e = 3, 4:
            // row j + 1 (tyy = 3, 1 for ey = 0, 1)
            const int r = e < 3 ? 0 : 1;
            const int ey = e < 3 ? e - 1 : e - 3;
            const int tyy = e < 3 ? 4 - 2 * e : 3 - 2 * (e - 3);
            const float4 g03 = *reinterpret_cast<const float4*>(gt + tyy * 8);
            const float g4 = gt[tyy * 8 + 4];
            const float* cv = c[ey + 1];
            qa[r][0] = fmaf(g4, cv[0], fmaf(g03.z, cv[1], fmaf(g03.x, cv[2], qa[r][0])));
            qa[r][1] = fmaf(g03.w, cv[1], fmaf(g03.y, cv[2], qa[r][1]));
            qa[r][2] = fmaf(g4, cv[1], fmaf(g03.z, cv[2], fmaf(g03.x, cv[3], qa[r][2])));
            qa[r][3] = fmaf(g03.w, cv[2], fmaf(g03.y, cv[3], qa[r][3]));
          }
        }
        float* yp = a.y + ((b * n0 + o) * (int64_t)n1 + j) * n2 + k;
        *reinterpret_cast<float4*>(yp) = make_float4(qa[0][0], qa[0][1], qa[0][2], qa[0][3]);
        *reinterpret_cast<float4*>(yp + n2) = make_float4(qa[1][0], qa[1][1], qa[1][2], qa[1][3]);
      }
#pragma unroll
      for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          qa[r][q] = qb[r][q];
          qb[r][q] = qc[r][q];
          qc[r][q] = 0.f;
        }
    }
  }
  cp_async_wait<0>();
}

// smallest pitch >= lo, a multiple of 4 (16-byte rows), congruent to r
// modulo m where that is possible (else lo rounded up to 4)
static int bank_pitch(int lo, int r, int m) {
  for (int p = (lo + 3) / 4 * 4; p < lo + m + 4; p += 4)
    if (p % m == r % m) return p;
  return (lo + 3) / 4 * 4;
}

// r2[b][c][I] = sum_d Q[d][c] r1[b][2I + d], d in [-2, 2]^3, 16 channels
struct StrideArgs {
  const float* x;    // (nb, n0, n1, n2) fine (level-1) grid
  float* y;          // (nb, 16, n0/2, n1/2, n2/2)
  const float* Q;    // [125][16]
  int64_t nb;
  int n0, n1, n2;
};

// thread = two neighbouring coarse points (K, K + 1) of a row, all 16
// channels: the 7 fine columns they read and every weight load are shared
__global__ void __launch_bounds__(256) fold_stride_kernel(const StrideArgs a) {
  __shared__ __align__(16) float sQ[125 * 16];
  for (int e = threadIdx.x; e < 125 * 16; e += blockDim.x) sQ[e] = a.Q[e];
  __syncthreads();
  const int n0 = a.n0, n1 = a.n1, n2 = a.n2;
  const int m0 = n0 >> 1, m1 = n1 >> 1, m2 = n2 >> 1;
  const int mh = (m2 + 1) / 2;                      // point pairs per coarse row
  const int64_t mpts = (int64_t)m0 * m1 * m2;
  const int64_t plane = (int64_t)n1 * n2;
  const int64_t total = a.nb * m0 * (int64_t)m1 * mh;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int K = (int)(e % mh) * 2;
    int64_t r = e / mh;
    const int J = (int)(r % m1);
    r /= m1;
    const int I = (int)(r % m0);
    const int64_t b = r / m0;
    const bool two = K + 1 < m2;
    float acc0[16], acc1[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) { acc0[c] = 0.f; acc1[c] = 0.f; }
    int kk[7];
#pragma unroll
    for (int m = 0; m < 7; ++m) kk[m] = pw(2 * K - 2 + m, n2);
    const float* xb = a.x + b * n0 * plane;
#pragma unroll 1
    for (int dx = 0; dx < 5; ++dx) {
      const float* pl = xb + pw(2 * I + dx - 2, n0) * plane;
#pragma unroll 1
      for (int dy = 0; dy < 5; ++dy) {
        const float* rp = pl + (int64_t)pw(2 * J + dy - 2, n1) * n2;
        float w[7];
#pragma unroll
        for (int m = 0; m < 7; ++m) w[m] = __ldg(rp + kk[m]);
        const float4* q4 = reinterpret_cast<const float4*>(sQ + ((dx * 5 + dy) * 5) * 16);
#pragma unroll
        for (int dz = 0; dz < 5; ++dz) {
#pragma unroll
          for (int c4 = 0; c4 < 4; ++c4) {
            const float4 q = q4[dz * 4 + c4];
            acc0[4 * c4] = fmaf(q.x, w[dz], acc0[4 * c4]);
            acc0[4 * c4 + 1] = fmaf(q.y, w[dz], acc0[4 * c4 + 1]);
            acc0[4 * c4 + 2] = fmaf(q.z, w[dz], acc0[4 * c4 + 2]);
            acc0[4 * c4 + 3] = fmaf(q.w, w[dz], acc0[4 * c4 + 3]);
            acc1[4 * c4] = fmaf(q.x, w[dz + 2], acc1[4 * c4]);
            acc1[4 * c4 + 1] = fmaf(q.y, w[dz + 2], acc1[4 * c4 + 1]);
            acc1[4 * c4 + 2] = fmaf(q.z, w[dz + 2], acc1[4 * c4 + 2]);
            acc1[4 * c4 + 3] = fmaf(q.w, w[dz + 2], acc1[4 * c4 + 3]);
          }
        }
      }
    }
    float* yb = a.y + b * 16 * mpts + ((int64_t)I * m1 + J) * m2 + K;
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      yb[c * mpts] = acc0[c];
      if (two) yb[c * mpts + 1] = acc1[c];
    }
  }
}

// The 16-channel coarse part of level 1 as a parity convolution:
//   y[2J + par] += sum_c sum_e G[c][par - 2e + 2] a2[c][J + e],
// par in {0,1}^3, e in {-1,0,1}^3 (tap t = par - 2e + 2 per axis; t = 5, an
// odd parity with e = -1, is zero).  One thread per coarse point J loads the
// 27 neighbours of a channel once and feeds all 8 fine points of its parity
// block: 125 FMAs per 27 loads, against one output per gathered
// neighbourhood in fold_fine_kernel.  A CTA owns one coarse plane of one band;
// every CTA stages G reordered into the order the unrolled loops consume it
// (channel, parity, tap), 128 floats per channel, so each 16-byte broadcast
// shared load serves four FMAs.
__host__ __device__ __forceinline__ constexpr int par_taps(int p) { return p ? 2 : 3; }
// e of the j-th tap of parity p: p = 0 -> -1, 0, 1; p = 1 -> 0, 1
__host__ __device__ __forceinline__ constexpr int par_e(int p, int j) { return p ? j : j - 1; }

// index into G[c][6][6][6] of the k-th weight in (parity, tap) order, the
// order of the unrolled loops below: (3 + 2)^3 = 125 over the 8 parities,
// then -1
struct ParityTaps {
  int v[128];
};
constexpr ParityTaps make_parity_taps() {
  ParityTaps t{};
  int k = 0;
  for (int par = 0; par < 8; ++par) {
    const int px = par >> 2, py = (par >> 1) & 1, pz = par & 1;
    for (int jx = 0; jx < par_taps(px); ++jx)
      for (int jy = 0; jy < par_taps(py); ++jy)
        for (int jz = 0; jz < par_taps(pz); ++jz) {
          const int tx = px - 2 * par_e(px, jx) + 2, ty = py - 2 * par_e(py, jy) + 2;
          const int tz = pz - 2 * par_e(pz, jz) + 2;
          t.v[k++] = (tx * 6 + ty) * 6 + tz;
        }
  }
  for (; k < 128; ++k) t.v[k] = -1;
  return t;
}
__constant__ ParityTaps kParityTaps = make_parity_taps();

__global__ void __launch_bounds__(256) fold_parity16_kernel(const FoldArgs a) {
  __shared__ __align__(16) float sW[16 * 128];
  const int tid = threadIdx.x;
  // reorder G[c][tx][ty][tz] (t in 0..5) into (c, parity, tap) order
  for (int e = tid; e < 16 * 128; e += blockDim.x) {
    const int src = kParityTaps.v[e & 127];
    sW[e] = src >= 0 ? __ldg(a.G + (e >> 7) * 216 + src) : 0.f;
  }
  __syncthreads();
  const int m0 = a.n0 >> 1, m1 = a.n1 >> 1, m2 = a.n2 >> 1;
  const int m12 = m1 * m2, m012 = m12 * m0;
  const int I = blockIdx.x;
  const int64_t b = blockIdx.y;
  const float* cb = a.xc + b * 16 * (int64_t)m012;
  float* yb = a.y + b * 8 * (int64_t)m012;
  const int n2 = a.n2, n12 = a.n1 * a.n2;
  int po[3];
#pragma unroll
  for (int e = 0; e < 3; ++e) po[e] = pw(I - 1 + e, m0) * m12;
  for (int q = tid; q < m12; q += blockDim.x) {
    const int J1 = q / m2, J2 = q - J1 * m2;
    int ro[3], co[3];
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      ro[e] = pw(J1 - 1 + e, m1) * m2;
      co[e] = pw(J2 - 1 + e, m2);
    }
    float acc[8];
#pragma unroll
    for (int p = 0; p < 8; ++p) acc[p] = 0.f;
#pragma unroll 1
    for (int c = 0; c < 16; ++c) {
      const float* xc = cb + c * m012;
      float v[3][3][3];
#pragma unroll
      for (int e0 = 0; e0 < 3; ++e0)
#pragma unroll
        for (int e1 = 0; e1 < 3; ++e1)
#pragma unroll
          for (int e2 = 0; e2 < 3; ++e2) v[e0][e1][e2] = __ldg(xc + po[e0] + ro[e1] + co[e2]);
      const float4* w4 = reinterpret_cast<const float4*>(sW + c * 128);
      int k = 0;
#pragma unroll
      for (int par = 0; par < 8; ++par) {
        const int px = par >> 2, py = (par >> 1) & 1, pz = par & 1;
#pragma unroll
        for (int jx = 0; jx < par_taps(px); ++jx)
#pragma unroll
          for (int jy = 0; jy < par_taps(py); ++jy)
#pragma unroll
            for (int jz = 0; jz < par_taps(pz); ++jz, ++k) {
              const float4 w = w4[k >> 2];
              const float wk = (k & 3) == 0 ? w.x : ((k & 3) == 1 ? w.y : ((k & 3) == 2 ? w.z : w.w));
              acc[par] = fmaf(wk, v[par_e(px, jx) + 1][par_e(py, jy) + 1][par_e(pz, jz) + 1], acc[par]);
            }
      }
    }
    float* yp = yb + (int64_t)(2 * I) * n12 + (2 * J1) * n2 + 2 * J2;
#pragma unroll
    for (int par = 0; par < 8; ++par) {
      float* o = yp + (par >> 2) * n12 + ((par >> 1) & 1) * n2 + (par & 1);
      *o += acc[par];
    }
  }
}

template <typename KernelT>
int launch_fine(KernelT k, const FoldArgs& a, const char* what, cudaStream_t st) {
  const int nkx = (a.n2 + 31) / 32;
  const int njb = (a.n1 + JB - 1) / JB;
  const dim3 grid((unsigned)(nkx * ((njb + 7) / 8)), (unsigned)a.n0, (unsigned)a.nb);
  k<<<grid, dim3(32, 8), 0, st>>>(a);
  return check_launch(what);
}

template <typename KernelT, typename ArgsT>
int launch_grid(KernelT k, const ArgsT& a, int64_t work, const char* what, cudaStream_t st) {
  const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, (int64_t)sm_count() * 16));
  k<<<(unsigned)blocks, 256, 0, st>>>(a);
  return check_launch(what);
}

}  // namespace
}  // namespace gb

using namespace gb;

extern "C" {

int gb_learned_fold_fine(const float* xf, const float* F, int rh, const float* xc, const float* G, int cc,
                         float* y, int64_t nb, const int64_t n_c[3], void* stream) {
  GB_REQUIRE(xf && F && y && n_c && nb >= 0, "gb_learned_fold_fine: bad arguments");
  if (nb == 0) return GB_OK;
  GB_REQUIRE(n_c[2] >= PXF + 2, "gb_learned_fold_fine: rows shorter than 10 points");
  GB_REQUIRE(n_c[0] >= 2 && n_c[1] >= 2 && n_c[2] >= 2 && n_c[0] % 2 == 0 && n_c[1] % 2 == 0 &&
                 n_c[2] % 2 == 0 && n_c[0] < (1 << 20) && n_c[1] < (1 << 20) && n_c[2] < (1 << 20),
             "gb_learned_fold_fine: needs even grid sizes (periodic coarsening)");
  GB_REQUIRE(xc && G, "gb_learned_fold_fine: missing coarse input or weights");
  GB_REQUIRE(nb < 65536 && n_c[0] * n_c[1] * n_c[2] * (cc > 1 ? cc : 1) < ((int64_t)1 << 31),
             "gb_learned_fold_fine: too many grids or points per grid");
  {
    // y is written (fine part) before the coarse part reads xc and adds
    // into y, so an output overlapping either input gives wrong results
    const uint64_t nf = (uint64_t)nb * n_c[0] * n_c[1] * n_c[2] * sizeof(float);
    const uint64_t nco = (uint64_t)nb * (cc > 1 ? cc : 1) * (n_c[0] / 2) * (n_c[1] / 2) * (n_c[2] / 2) *
                         sizeof(float);
    auto overlap = [](const void* a, uint64_t na, const void* b, uint64_t nb_) {
      const uint64_t pa = (uint64_t)(uintptr_t)a, pb = (uint64_t)(uintptr_t)b;
      return pa < pb + nb_ && pb < pa + na;
    };
    GB_REQUIRE(!overlap(y, nf, xf, nf) && !overlap(y, nf, xc, nco),
               "gb_learned_fold_fine: the output overlaps an input");
  }
  FoldArgs a{xf, xc, y, F, G, nb, (int)n_c[0], (int)n_c[1], (int)n_c[2]};
  cudaStream_t st = (cudaStream_t)stream;
  if (rh == 1 && cc == 1) {
    // a quarter warp spans <= 2 row pairs: consecutive 16-byte chunks when
    // a row pair advances the chunk index by ngx (mod 8); likewise the
    // coarse 8-byte loads (mod 16) of a half warp
    const int ngx = (int)(n_c[2] / 4);
    Fold0Cfg cfg;
    cfg.FP = bank_pitch((int)n_c[2] + 8, (int)(n_c[2] / 2), 16);
    cfg.CP = bank_pitch((int)(n_c[2] / 2) + 8, (int)(n_c[2] / 2), 32);
    auto smem_of = [&](int t) {
      return (size_t)(3 * (t + 2) * cfg.FP + 4 * (t / 2 + 2) * cfg.CP) * sizeof(float);
    };
    static size_t attr = 0;
    if (attr == 0) {
      cudaFuncSetAttribute(fold0_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
      attr = 1;
    }
    // rows per CTA: the even divisor of n1 (<= 512 threads of 2 rows x 4
    // points, plane pieces <= 4 per thread) with the most resident warps
    // doing work per SM; ties to more rows (less halo)
    int TY = 0;
    double best = 0.0;
    for (int t = (int)n_c[1]; t >= 2; t -= 2) {
      const int thr = ngx * t / 2;
      if (n_c[1] % t || thr > 512 || (t + 2) * ngx > 4 * thr || (t / 2 + 2) * (n_c[2] / 2 + 2) > 4 * thr ||
          smem_of(t) > 200 * 1024)
        continue;
      int blk = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blk, fold0_pair_kernel, thr, smem_of(t));
      const double busy = (double)blk * thr;
      if (busy > best * 1.001) {
        best = busy;
        TY = t;
      }
    }
    if (TY && n_c[2] % 4 == 0 && n_c[0] >= 2) {
      cfg.TY = TY;
      const int threads = ngx * TY / 2;
      const size_t smem = smem_of(TY);
      // plane chunks of about 12 planes (two halo planes each)
      cfg.nch = (int)std::max<int64_t>(1, n_c[0] / 12);
      const dim3 grid((unsigned)cfg.nch, (unsigned)(n_c[1] / TY), (unsigned)nb);
      fold0_pair_kernel<<<grid, (unsigned)threads, smem, st>>>(a, cfg);
      return check_launch("fold0_pair_kernel");
    }
    return launch_fine(fold_fine_kernel<1, 1>, a, "fold_fine_kernel<1,1>", st);
  }
  if (rh == 2 && cc == 16) {
    // fine 5^3 part, then the coarse part added as a parity convolution:
    // both on the tensor cores when the coarse plane fits their layout
    const int m0 = (int)(n_c[0] / 2), m1 = (int)(n_c[1] / 2), m2 = (int)(n_c[2] / 2);
    if (conv_tc_fits(m0, m1, m2)) {
      int launched = 0;
      int rc = conv_fine5_tc_try(xf, F, y, nb, m0, m1, m2, st, &launched);
      if (rc) return rc;
      if (!launched) return fail(GB_E_INVALID, "gb_learned_fold_fine: tensor-core plan refused a fitting grid");
      rc = conv_parity_tc_try(xc, G, y, nb, m0, m1, m2, st, &launched);
      if (rc) return rc;
      if (!launched) return fail(GB_E_INVALID, "gb_learned_fold_fine: tensor-core plan refused a fitting grid");
      return GB_OK;
    }
    int rc = launch_fine(fold_fine_kernel<2, 0>, a, "fold_fine_kernel<2,0>", st);
    if (rc) return rc;
    const int m12 = (int)(n_c[1] / 2 * (n_c[2] / 2));
    const unsigned threads = (unsigned)std::min(256, (m12 + 31) / 32 * 32);
    fold_parity16_kernel<<<dim3((unsigned)(n_c[0] / 2), (unsigned)nb), threads, 0, st>>>(a);
    return check_launch("fold_parity16_kernel");
  }
  return fail(GB_E_UNSUPPORTED, "gb_learned_fold_fine: (rh, cc) not in {(1, 1), (2, 16)}");
}

int gb_learned_fold_stride(const float* x, const float* Q, float* y, int64_t nb, const int64_t n_c[3],
                           void* stream) {
  GB_REQUIRE(x && Q && y && n_c && nb >= 0, "gb_learned_fold_stride: bad arguments");
  if (nb == 0) return GB_OK;
  GB_REQUIRE(n_c[0] >= 2 && n_c[1] >= 2 && n_c[2] >= 2 && n_c[0] % 2 == 0 && n_c[1] % 2 == 0 &&
                 n_c[2] % 2 == 0 && n_c[0] < (1 << 20) && n_c[1] < (1 << 20) && n_c[2] < (1 << 20),
             "gb_learned_fold_stride: needs even grid sizes (periodic coarsening)");
  // on the tensor cores when the coarse plane fits their layout
  const int m0 = (int)(n_c[0] / 2), m1 = (int)(n_c[1] / 2), m2 = (int)(n_c[2] / 2);
  if (conv_tc_fits(m0, m1, m2)) {
    int launched = 0;
    const int rc = conv_stride_tc_try(x, Q, y, nb, m0, m1, m2, (cudaStream_t)stream, &launched);
    if (rc || launched) return rc;
  }
  StrideArgs a{x, y, Q, nb, (int)n_c[0], (int)n_c[1], (int)n_c[2]};
  const int64_t work = nb * (n_c[0] / 2) * (n_c[1] / 2) * ((n_c[2] / 2 + 1) / 2);
  return launch_grid(fold_stride_kernel, a, work, "fold_stride_kernel", (cudaStream_t)stream);
}

}  // extern "C"
