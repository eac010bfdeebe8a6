// FD star stencil, TMA + warp-specialised pipeline (the default path on
// sm_100a whenever the layout allows it; fd_stencil.cu keeps the cp.async
// kernel for the other cases: odd row pitches, Bloch phases, radius > 4).
//
// Tile = a band of T1 full rows of the (axis1, axis2) plane: because a CTA
// holds whole rows, the axis-2 halo of a periodic grid is read from the other
// end of the same shared-memory row (no wrap-around copies), and only the
// axis-1 halo rows of the first / last tile need a second TMA box.  One
// producer warp streams planes (tile + halo rows) into a ring of NS slots
// with cp.async.bulk.tensor; zero boundaries come from the TMA out-of-bounds
// fill on every axis (planes -H..-1 and n0.., rows outside 0..n1-1, and the
// padding columns of each 128-byte-pitched shared-memory row), so the
// consumers run without boundary branches.  Consumer warps keep the axis-0
// neighbours in a register queue whose rotation is resolved at compile time
// (the plane loop is unrolled by 2H+1), read the in-plane neighbours from the
// slot with 16-byte loads at offsets fixed per thread, take the stencil
// coefficients from the kernel-parameter bank, and hand each slot back
// through an mbarrier when its last reader is done.  All waits are bounded
// (tma.cuh).
#include <algorithm>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <type_traits>
#include <cudaTypedefs.h>
#include "internal.cuh"
#include "tma.cuh"

namespace gb {

__device__ int g_dev_error = 0;

__device__ void raise_device_error(int code) { atomicCAS(&g_dev_error, 0, code); }

int device_error_flag(int clear) {
  int v = 0;
  cudaMemcpyFromSymbol(&v, g_dev_error, sizeof(int));
  if (clear && v) {
    int z = 0;
    cudaMemcpyToSymbol(g_dev_error, &z, sizeof(int));
  }
  return v;
}

bool encode_tensor_map_4d(CUtensorMap* map, CUtensorMapDataType dt, void* base, const uint64_t dims[4],
                          const uint64_t strides_bytes[3], const uint32_t box[4]) {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess || !p)
      return false;
    fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  cuuint64_t d[4] = {dims[0], dims[1], dims[2], dims[3]};
  cuuint64_t s[3] = {strides_bytes[0], strides_bytes[1], strides_bytes[2]};
  cuuint32_t b[4] = {box[0], box[1], box[2], box[3]};
  cuuint32_t e[4] = {1, 1, 1, 1};
  CUresult r = fn(map, dt, 4, base, d, s, b, e, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

static thread_local const char* g_tma_reason = "";
// autotuner state: layout key -> chosen rows-per-thread-row count (ty)
static std::mutex g_tune_mutex;
static std::map<std::string, int> g_tune;
// GPAW_B200_AUTOTUNE=0 turns timing off (the model's choice is launched):
// makes the launch sequence of a run reproducible, e.g. for a profiler
static int autotune_enabled() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("GPAW_B200_AUTOTUNE");
    v = (e && e[0] == '0') ? 0 : 1;
  }
  return v;
}
constexpr int NS_MAX = 16;      // ring slots (mbarrier pairs live in the first 256 bytes)

struct TmaArgs {
  void* out;
  const void* y;
  const void* vpot;
  int64_t nbatch;
  int n0, n1, n2;
  int pbc0, pbc1, pbc2;
  int TY, TZ, NTC, T1, ROWS, ytiles, NS;
  int T1L;          // rows of the last row tile of a periodic axis 1 (<= T1)
  int pitch;        // bytes per shared-memory row (multiple of 128, >= n2 * sizeof(T))
  int slot_bytes;   // ROWS * pitch
  double c0;
  double c0diff;    // c0 + sum of the neighbour coefficients (difference form)
  double a[3][2 * HMAX + 1];
  float c0f, c0difff;
  float af[3][2 * HMAX + 1];
  double alpha, beta, gamma;
};

// coefficients straight from the kernel-parameter bank (no registers held)
template <typename R>
__device__ __forceinline__ R coef(const TmaArgs& a, int c, int m) {
  if constexpr (sizeof(R) == 8) return a.a[c][m];
  else return a.af[c][m];
}

// Slot layout: ROWS rows of `pitch` bytes, logical row r = grid row y0 - H + r
// (wrapped on a periodic axis 1).  Columns [n2, pitch) of every row are TMA
// out-of-bounds fill (zeros); on a zero-boundary axis 2 the pitch keeps at
// least 16 such bytes, and the halo chunks left of column 0 / right of column
// n2 - 1 read them, so the consumers have no boundary branches at all.
// shared-memory vector loads of VB bytes (16: float4, 8: float2)
template <typename T, int N, int VB>
__device__ __forceinline__ void ldv(const T* p, T (&v)[N]) {
  if constexpr (VB == 16) {
    lds_vec<T, N>(p, v);
  } else {
    constexpr int V = 8 / (int)sizeof(T);
    static_assert(N % V == 0, "");
#pragma unroll
    for (int i = 0; i < N / V; ++i) {
      const float2 x = *reinterpret_cast<const float2*>(p + i * V);
      const T* e = reinterpret_cast<const T*>(&x);
#pragma unroll
      for (int k = 0; k < V; ++k) v[i * V + k] = e[k];
    }
  }
}

// N consecutive elements from global memory: 16-byte loads when N elements
// make whole 16-byte chunks (the caller guarantees the alignment), else
// element loads
template <typename V, int N>
__device__ __forceinline__ void ldg_run(const V* __restrict__ p, V (&v)[N]) {
  if constexpr ((N * sizeof(V)) % 16 == 0) {
    constexpr int E = 16 / (int)sizeof(V);
#pragma unroll
    for (int h = 0; h < N / E; ++h) {
      const float4 x = __ldg(reinterpret_cast<const float4*>(p) + h);
      const V* e = reinterpret_cast<const V*>(&x);
#pragma unroll
      for (int k = 0; k < E; ++k) v[h * E + k] = e[k];
    }
  } else {
#pragma unroll
    for (int c = 0; c < N; ++c) v[c] = p[c];
  }
}

// FP32 taps on two neighbouring points at once (packed f32x2 arithmetic,
// sm_100): one pair of offsets +k / -k with coefficients cp / cm.  SYM = 1
// (cp == cm, the Laplacian): c ((vp + vm) - 2 xc), 3 packed operations and
// exactly zero on a constant; SYM = -1 (cp == -cm, first derivatives):
// c (vp - vm); SYM = 0: the difference form c (v - xc) per offset.
template <int SYM>
__device__ __forceinline__ float2 tap2(float2 acc, float cp, float cm, float2 vp, float2 vm, float2 xc) {
  const float2 m1 = make_float2(-1.f, -1.f);
  if constexpr (SYM == 1) {
    const float2 d = __ffma2_rn(make_float2(-2.f, -2.f), xc, __fadd2_rn(vp, vm));
    return __ffma2_rn(make_float2(cp, cp), d, acc);
  } else if constexpr (SYM == -1) {
    return __ffma2_rn(make_float2(cp, cp), __ffma2_rn(vm, m1, vp), acc);
  } else {
    acc = __ffma2_rn(make_float2(cp, cp), __ffma2_rn(xc, m1, vp), acc);
    return __ffma2_rn(make_float2(cm, cm), __ffma2_rn(xc, m1, vm), acc);
  }
}

template <typename T, int H, int R1, int R2, int VB, int SYM = 0>
__global__ void __launch_bounds__(512) star_tma_kernel(const __grid_constant__ CUtensorMap tmA,
                                                        const __grid_constant__ CUtensorMap tmH,
                                                        const __grid_constant__ CUtensorMap tmB,
                                                        const __grid_constant__ CUtensorMap tmL,
                                                        const __grid_constant__ TmaArgs a) {
  using R = typename Elem<T>::R;
  constexpr int VEC = VB / (int)sizeof(T);   // elements per vector access
  constexpr int HZ = ((H + VEC - 1) / VEC) * VEC;
  constexpr int NQ = 2 * H + 1;
  static_assert(R2 % VEC == 0, "");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + NS_MAX;
  unsigned char* slots = smem + 256;

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int NWC = (a.NTC + 31) >> 5;       // consumer warps
  const int NS = a.NS;
  const int n0 = a.n0, n1 = a.n1, n2 = a.n2;
  const int T1 = a.T1;
  const int64_t n12 = (int64_t)n1 * n2;
  const int64_t total = a.nbatch * a.ytiles * n0;
  const int64_t s_begin = total * blockIdx.x / gridDim.x;
  const int64_t s_end = total * (blockIdx.x + 1) / gridDim.x;

  if (tid == 0) {
    for (int i = 0; i < NS; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], NWC);
    }
    mbar_fence_init();
  }
  __syncthreads();

  if (warp == NWC) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      tma_prefetch_desc(&tmA);
      tma_prefetch_desc(&tmH);
      tma_prefetch_desc(&tmB);
      tma_prefetch_desc(&tmL);
      const int tile_kind_first = a.pbc1 ? 1 : 0;
      // ring position and the parity of the empty barrier to wait on (no wait
      // during the first pass over the ring)
      int slot = 0;
      uint32_t eph = 0;
      bool first_pass = true;
      int64_t s = s_begin;
      while (s < s_end) {
        const int64_t col = s / n0;
        const int p_start = (int)(s % n0);
        const int p_end = (int)((s_end - s) < (int64_t)(n0 - p_start) ? p_start + (s_end - s) : n0);
        s += p_end - p_start;
        const int band = (int)(col / a.ytiles);
        const int y0 = (int)(col % a.ytiles) * T1;
        // 0: one box; 1: first tile of a periodic axis 1; 2: last tile of it
        const int kind = (tile_kind_first && y0 == 0) ? 1 : (a.pbc1 && y0 + T1 >= n1) ? 2 : 0;
        // the last tile of a periodic axis 1 may be shorter (T1L rows)
        const uint32_t bytes = kind == 2 ? (uint32_t)((a.T1L + 2 * H) * a.pitch) : (uint32_t)a.slot_bytes;
        const int L = p_end - p_start + 2 * H;
        for (int t = 0; t < L; ++t) {
          if (!first_pass && !mbar_wait(&empty[slot], eph)) {
            raise_device_error(101);
            return;
          }
          int sp = p_start - H + t;
          // periodic axis 0 wraps; a zero-boundary axis 0 reads planes -H..-1
          // and n0..n0+H-1 as TMA out-of-bounds fill (zeros)
          if (a.pbc0) sp = sp < 0 ? sp + n0 : (sp >= n0 ? sp - n0 : sp);
          unsigned char* dst = slots + (int64_t)slot * a.slot_bytes;
          mbar_arrive_expect_tx(&full[slot], bytes);
          if (kind == 0) {
            tma_load_4d(dst, &tmA, &full[slot], 0, y0 - H, sp, band);
          } else if (kind == 1) {
            tma_load_4d(dst, &tmH, &full[slot], 0, n1 - H, sp, band);
            tma_load_4d(dst + H * a.pitch, &tmB, &full[slot], 0, 0, sp, band);
          } else {
            tma_load_4d(dst, &tmL, &full[slot], 0, y0 - H, sp, band);
            tma_load_4d(dst + (a.T1L + H) * a.pitch, &tmH, &full[slot], 0, 0, sp, band);
          }
          if (++slot == NS) {
            slot = 0;
            if (first_pass) first_pass = false;
            else eph ^= 1u;
          }
        }
      }
    }
    return;
  }

  // -------------------------------------------------------------- consumers
  // threads beyond NTC (last warp only) mirror thread 0's reads and skip the
  // stores, so that every consumer lane runs the same barrier protocol
  const bool active = tid < a.NTC;
  const int ctid = active ? tid : 0;
  const int ty = ctid / a.TZ, tz = ctid % a.TZ;
  const int pitch = a.pitch;
  const int own_row = (H + ty * R1) * pitch;
  const int own_col = tz * R2 * (int)sizeof(T);
  int lcol[HZ / VEC], rcol[HZ / VEC];
#pragma unroll
  for (int ch = 0; ch < HZ / VEC; ++ch) {
    int zl = tz * R2 - HZ + ch * VEC;
    if (zl < 0) zl = a.pbc2 ? zl + n2 : n2;
    int zr = tz * R2 + R2 + ch * VEC;
    if (zr >= n2) zr = a.pbc2 ? zr - n2 : n2;
    lcol[ch] = own_row + zl * (int)sizeof(T);
    rcol[ch] = own_row + zr * (int)sizeof(T);
  }
  // FP32: the difference form sum_p c_p (x_p - x_c) + (sum c) x_c keeps the
  // operator exactly constant-annihilating after the coefficients are rounded
  // (otherwise every eigenvalue shifts by ~|c0| 2^-24)
  constexpr bool DIFF = sizeof(R) == 4;
  constexpr bool PACK = std::is_same<T, float>::value && R2 % 2 == 0;
  const bool epi = a.alpha != 1.0 || a.beta != 0.0 || a.y != nullptr || a.vpot != nullptr;
  const R* __restrict__ vpot = reinterpret_cast<const R*>(a.vpot);

  T q[NQ][R1][R2];
  int slot = 0;          // ring slot of the current step
  uint32_t fph = 0;      // parity of its full barrier
  int64_t s = s_begin;
  while (s < s_end) {
    const int64_t col = s / n0;
    const int p_start = (int)(s % n0);
    const int p_end = (int)((s_end - s) < (int64_t)(n0 - p_start) ? p_start + (s_end - s) : n0);
    s += p_end - p_start;
    const int64_t band = col / a.ytiles;
    const int y0 = (int)(col % a.ytiles) * T1;
    const int L = p_end - p_start + 2 * H;
    T* dst = reinterpret_cast<T*>(a.out) + band * n12 * n0;
    const T* ybase = a.y ? reinterpret_cast<const T*>(a.y) + band * n12 * n0 : nullptr;
    const int yrow = y0 + ty * R1;

    for (int tb = 0; tb < L; tb += NQ) {
#pragma unroll
      for (int u = 0; u < NQ; ++u) {
        const int t = tb + u;
        if (t < L) {
        int cslot = slot - H;  // slot of the centre plane (step t - H)
        if (cslot < 0) cslot += NS;
        if (!mbar_wait(&full[slot], fph)) {
          raise_device_error(102);
          return;
        }
        const unsigned char* P = slots + (int64_t)slot * a.slot_bytes;
#pragma unroll
        for (int r = 0; r < R1; ++r)
          ldv<T, R2, VB>(reinterpret_cast<const T*>(P + own_row + r * pitch + own_col), q[u][r]);

        if (t >= 2 * H) {
          const int cu = (u + NQ - H) % NQ;     // centre plane in the queue (static after unrolling)
          const int cpl = p_start + t - 2 * H;
          const unsigned char* Pc = slots + (int64_t)cslot * a.slot_bytes;
          T acc[R1][R2];
          if constexpr (PACK) {
          // FP32: two points per instruction (f32x2), pairs of columns
          float2 acc2[R1][R2 / 2];
          // centre + axis 0 (register queue)
#pragma unroll
          for (int r = 0; r < R1; ++r)
#pragma unroll
            for (int p = 0; p < R2 / 2; ++p) {
              const float2 xc = make_float2(q[cu][r][2 * p], q[cu][r][2 * p + 1]);
              float2 x = __fmul2_rn(make_float2(a.c0difff, a.c0difff), xc);
#pragma unroll
              for (int k = 1; k <= H; ++k) {
                const int mp = (u + 1 + H + k) % NQ, mm = (u + 1 + H - k) % NQ;
                x = tap2<SYM>(x, coef<R>(a, 0, HMAX + k), coef<R>(a, 0, HMAX - k),
                              make_float2(q[mp][r][2 * p], q[mp][r][2 * p + 1]),
                              make_float2(q[mm][r][2 * p], q[mm][r][2 * p + 1]), xc);
              }
              acc2[r][p] = x;
            }
          // axis 2: the row with its halo chunks
#pragma unroll
          for (int r = 0; r < R1; ++r) {
            float w[HZ + R2 + HZ];
#pragma unroll
            for (int ch = 0; ch < HZ / VEC; ++ch) {
              T tl[VEC], tr[VEC];
              ldv<T, VEC, VB>(reinterpret_cast<const T*>(Pc + lcol[ch] + r * pitch), tl);
              ldv<T, VEC, VB>(reinterpret_cast<const T*>(Pc + rcol[ch] + r * pitch), tr);
#pragma unroll
              for (int v = 0; v < VEC; ++v) {
                w[ch * VEC + v] = tl[v];
                w[HZ + R2 + ch * VEC + v] = tr[v];
              }
            }
#pragma unroll
            for (int c = 0; c < R2; ++c) w[HZ + c] = q[cu][r][c];
#pragma unroll
            for (int p = 0; p < R2 / 2; ++p) {
              const int c = HZ + 2 * p;
              const float2 xc = make_float2(w[c], w[c + 1]);
              float2 x = acc2[r][p];
#pragma unroll
              for (int k = 1; k <= H; ++k)
                x = tap2<SYM>(x, coef<R>(a, 2, HMAX + k), coef<R>(a, 2, HMAX - k),
                              make_float2(w[c + k], w[c + 1 + k]), make_float2(w[c - k], w[c + 1 - k]), xc);
              acc2[r][p] = x;
            }
          }
          // axis 1: rows of the centre slot, streamed (difference form)
#pragma unroll
          for (int rr = -H; rr < R1 + H; ++rr) {
            T v[R2];
            if (rr >= 0 && rr < R1) {
#pragma unroll
              for (int c = 0; c < R2; ++c) v[c] = q[cu][rr][c];
            } else {
              ldv<T, R2, VB>(reinterpret_cast<const T*>(Pc + own_row + rr * pitch + own_col), v);
            }
#pragma unroll
            for (int r = 0; r < R1; ++r) {
              const int d = rr - r;
              if (d < -H || d > H || d == 0) continue;
              const float cc = coef<R>(a, 1, HMAX + d);
#pragma unroll
              for (int p = 0; p < R2 / 2; ++p) {
                const float2 xc = make_float2(q[cu][r][2 * p], q[cu][r][2 * p + 1]);
                const float2 dv = __ffma2_rn(xc, make_float2(-1.f, -1.f), make_float2(v[2 * p], v[2 * p + 1]));
                acc2[r][p] = __ffma2_rn(make_float2(cc, cc), dv, acc2[r][p]);
              }
            }
          }
#pragma unroll
          for (int r = 0; r < R1; ++r)
#pragma unroll
            for (int p = 0; p < R2 / 2; ++p) {
              acc[r][2 * p] = acc2[r][p].x;
              acc[r][2 * p + 1] = acc2[r][p].y;
            }
          } else {
          // centre + axis 0 (register queue)
#pragma unroll
          for (int r = 0; r < R1; ++r)
#pragma unroll
            for (int c = 0; c < R2; ++c) {
              const T xc = q[cu][r][c];
              T x = scale(DIFF ? (R)a.c0difff : (R)a.c0, xc);
#pragma unroll
              for (int m = 0; m < NQ; ++m) {
                if (m == H) continue;
                const T v = q[(u + 1 + m) % NQ][r][c];
                x = fmadd(x, coef<R>(a, 0, m + HMAX - H), DIFF ? sub(v, xc) : v);
              }
              acc[r][c] = x;
            }
          // axis 2 (halo chunks of the own rows)
#pragma unroll
          for (int r = 0; r < R1; ++r) {
            T wl[HZ], wr[HZ];
#pragma unroll
            for (int ch = 0; ch < HZ / VEC; ++ch) {
              T tl[VEC], tr[VEC];
              ldv<T, VEC, VB>(reinterpret_cast<const T*>(Pc + lcol[ch] + r * pitch), tl);
              ldv<T, VEC, VB>(reinterpret_cast<const T*>(Pc + rcol[ch] + r * pitch), tr);
#pragma unroll
              for (int v = 0; v < VEC; ++v) {
                wl[ch * VEC + v] = tl[v];
                wr[ch * VEC + v] = tr[v];
              }
            }
#pragma unroll
            for (int c = 0; c < R2; ++c) {
              const T xc = q[cu][r][c];
#pragma unroll
              for (int m = 0; m < NQ; ++m) {
                if (m == H) continue;
                const int cc = c + m - H;
                const T v = cc < 0 ? wl[HZ + cc] : (cc >= R2 ? wr[cc - R2] : q[cu][r][cc]);
                acc[r][c] = fmadd(acc[r][c], coef<R>(a, 2, m + HMAX - H), DIFF ? sub(v, xc) : v);
              }
            }
          }
          // axis 1 (rows of the centre slot)
#pragma unroll
          for (int rr = -H; rr < R1 + H; ++rr) {
            T v[R2];
            if (rr >= 0 && rr < R1) {
#pragma unroll
              for (int c = 0; c < R2; ++c) v[c] = q[cu][rr][c];
            } else {
              ldv<T, R2, VB>(reinterpret_cast<const T*>(Pc + own_row + rr * pitch + own_col), v);
            }
#pragma unroll
            for (int r = 0; r < R1; ++r) {
              const int m = rr - r + H;
              if (m < 0 || m > 2 * H || m == H) continue;
#pragma unroll
              for (int c = 0; c < R2; ++c)
                acc[r][c] = fmadd(acc[r][c], coef<R>(a, 1, m + HMAX - H), DIFF ? sub(v[c], q[cu][r][c]) : v[c]);
            }
          }
          }  // PACK
          // epilogue + streaming stores
          if (active) {
            const int64_t pbase = (int64_t)cpl * n12 + (int64_t)yrow * n2 + tz * R2;
#pragma unroll
            for (int r = 0; r < R1; ++r) {
              if (yrow + r >= n1) continue;
              const int64_t p = pbase + (int64_t)r * n2;
              if (epi) {
                if constexpr (sizeof(T) == 4) {
                  // FP32: y and the potential as 16-byte loads of this
                  // thread's R2 points (p is a multiple of R2, both bases
                  // 16-byte aligned); the FP64 kernels run faster, epilogue
                  // or not, with the element loads below
                  T yv[R2];
                  R vv[R2];
                  if (ybase) ldg_run<T, R2>(ybase + p, yv);
                  if (vpot) ldg_run<R, R2>(vpot + p, vv);
                  if constexpr (PACK) {
                    const float2 al = make_float2((float)a.alpha, (float)a.alpha);
                    const float2 be = make_float2((float)a.beta, (float)a.beta);
                    const float2 ga = make_float2((float)a.gamma, (float)a.gamma);
#pragma unroll
                    for (int c = 0; c < R2; c += 2) {
                      const float2 xc = make_float2(q[cu][r][c], q[cu][r][c + 1]);
                      float2 v = __ffma2_rn(be, xc, __fmul2_rn(al, make_float2(acc[r][c], acc[r][c + 1])));
                      if (ybase) v = __ffma2_rn(ga, make_float2(yv[c], yv[c + 1]), v);
                      if (vpot) v = __ffma2_rn(make_float2(vv[c], vv[c + 1]), xc, v);
                      acc[r][c] = v.x;
                      acc[r][c + 1] = v.y;
                    }
                  } else {
#pragma unroll
                  for (int c = 0; c < R2; ++c) {
                    T v = fmadd(scale((R)a.alpha, acc[r][c]), (R)a.beta, q[cu][r][c]);
                    if (ybase) v = fmadd(v, (R)a.gamma, yv[c]);
                    if (vpot) v = fmadd(v, vv[c], q[cu][r][c]);
                    acc[r][c] = v;
                  }
                  }
                } else {
#pragma unroll
                  for (int c = 0; c < R2; ++c) {
                    T v = fmadd(scale((R)a.alpha, acc[r][c]), (R)a.beta, q[cu][r][c]);
                    if (ybase) v = fmadd(v, (R)a.gamma, ybase[p + c]);
                    if (vpot) v = fmadd(v, vpot[p + c], q[cu][r][c]);
                    acc[r][c] = v;
                  }
                }
              }
#pragma unroll
              for (int c = 0; c < R2; c += VEC) {
                if constexpr (VB == 16) {
                  float4 w4;
                  T* e = reinterpret_cast<T*>(&w4);
#pragma unroll
                  for (int v = 0; v < VEC; ++v) e[v] = acc[r][c + v];
                  __stcs(reinterpret_cast<float4*>(dst + p + c), w4);
                } else {
                  float2 w2;
                  T* e = reinterpret_cast<T*>(&w2);
#pragma unroll
                  for (int v = 0; v < VEC; ++v) e[v] = acc[r][c + v];
                  __stcs(reinterpret_cast<float2*>(dst + p + c), w2);
                }
              }
            }
          }
        }
        // hand back the slot read as centre plane (its last reader was this step)
        if (t >= H) {
          __syncwarp();
          if (lane == 0) mbar_arrive(&empty[cslot]);
        }
        if (++slot == NS) {
          slot = 0;
          fph ^= 1u;
        }
        }
      }
    }
    // segment end: release the slots of the last H planes (axis-0 neighbours only)
    for (int d = H; d >= 1; --d) {
      int rs = slot - d;
      if (rs < 0) rs += NS;
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[rs]);
    }
  }
}

// ------------------------------------------------------------------ host
template <typename T, int H, int R1, int R2, int VB = 16, int SYM = 0>
static int launch_tma_cfg(const gb_operator* op, const void* in, void* out, int64_t nin, cudaStream_t st,
                          const Epilogue& ep) {
  using R = typename Elem<T>::R;
  const int n0 = (int)op->n[0], n1 = (int)op->n[1], n2 = (int)op->n[2];
  const int TZ = n2 / R2;
  auto kern = star_tma_kernel<T, H, R1, R2, VB, SYM>;
  static int regs = -1;
  if (regs < 0) {
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, kern) != cudaSuccess) { g_tma_reason = "cudaFuncGetAttributes failed"; return 1; }
    regs = fa.numRegs;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
  }
  // shared-memory row pitch: 128-byte multiple; a zero-boundary axis 2 keeps
  // at least 16 bytes of out-of-bounds fill (zeros) after the last column
  const int rowb = n2 * (int)sizeof(T);
  const int pitch = ((rowb + (op->pbc[2] ? 0 : 16) + 127) / 128) * 128;
  if (pitch / (int)sizeof(R) > 256) { g_tma_reason = "row longer than a TMA box"; return 1; }
  // candidate (rows per tile, CTAs per SM, ring depth): score = resident
  // consumer warps (up to 24) x halo efficiency x prefetch depth (up to 4 planes)
  struct Cand { double score; int ty, ctas, ns; };
  Cand cands[256];
  int ncand = 0;
  const int SMEM_SM = 228 * 1024, SMEM_CTA = 227 * 1024;
  for (int ty = 1; ty * TZ <= 512 - 32 && ncand < 250; ++ty) {
    const int T1 = ty * R1;
    if (T1 < H || T1 + 2 * H > 256) continue;
    // periodic axis 1: at least two tiles, the last one at least H rows
    if (op->pbc[1] && (ceil_div(n1, T1) < 2 || n1 - (ceil_div(n1, T1) - 1) * T1 < H)) continue;
    if (!op->pbc[1] && T1 > n1 + R1 - 1) continue;
    const int threads = ((ty * TZ + 31) / 32) * 32 + 32;
    const int regs_cta = threads * ((regs + 7) / 8 * 8);
    const int by_regs = 65536 / regs_cta;
    const int slot = (T1 + 2 * H) * pitch;
    for (int ctas = 1; ctas <= by_regs && ctas <= 4; ++ctas) {
      const int per_cta = std::min(SMEM_SM / ctas - 1024, SMEM_CTA) - 256 - 128;
      const int ns = std::min(NS_MAX, per_cta / slot);
      if (ns < H + 3) continue;
      const double cw = std::min(24.0, ctas * ((ty * TZ + 31) / 32.0));
      // useful rows per staged row: halo rows and the empty part of a short
      // last tile both count against a tile height
      const double eff = (double)n1 / ((double)ceil_div(n1, T1) * (T1 + 2.0 * H));
      const double pf = std::min(1.0, (ns - H - 1) / 4.0);
      cands[ncand++] = {cw * eff * pf, ty, ctas, ns};
    }
  }
  std::sort(cands, cands + ncand, [](const Cand& x, const Cand& y) { return x.score > y.score; });
  // the occupancy-checked candidates kept for tuning (distinct row-tile
  // heights): the model's best three, the best tile height that divides n1
  // (no short last tile), and the best configuration with several CTAs per SM
  constexpr int NOK = 6;
  Cand ok[NOK];
  int occ_of[NOK];
  int nok = 0;
  auto try_add = [&](const Cand& cd) -> bool {
    for (int i = 0; i < nok; ++i)
      if (ok[i].ty == cd.ty) return false;
    const int th = ((cd.ty * TZ + 31) / 32) * 32 + 32;
    const size_t sm = 256 + 128 + (size_t)cd.ns * (cd.ty * R1 + 2 * H) * pitch;
    int o = 0;
    if (nok < NOK && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, th, sm) == cudaSuccess &&
        o >= cd.ctas) {
      ok[nok] = cd;
      occ_of[nok++] = o;
      return true;
    }
    return false;
  };
  for (int c = 0; c < ncand && nok < 3; ++c) try_add(cands[c]);
  for (int c = 0; c < ncand; ++c)
    if (n1 % (cands[c].ty * R1) == 0 && try_add(cands[c])) break;
  for (int c = 0; c < ncand; ++c)
    if (cands[c].ctas > 1 && try_add(cands[c])) break;
  cudaGetLastError();
  if (nok == 0) {
    g_tma_reason = ncand ? "zero occupancy" : "no row tile fits the grid";
    return 1;
  }

  // one launch of candidate c
  auto launch = [&](int c) -> int {
    const Cand cb = ok[c];
    TmaArgs a{};
    a.out = out; a.y = ep.y; a.vpot = ep.vpot; a.nbatch = nin;
    a.n0 = n0; a.n1 = n1; a.n2 = n2;
    a.pbc0 = op->pbc[0]; a.pbc1 = op->pbc[1]; a.pbc2 = op->pbc[2];
    a.TY = cb.ty; a.TZ = TZ; a.NTC = cb.ty * TZ; a.T1 = cb.ty * R1; a.ROWS = a.T1 + 2 * H;
    a.ytiles = ceil_div(n1, a.T1);
    a.T1L = n1 - (a.ytiles - 1) * a.T1;
    a.NS = cb.ns;
    a.pitch = pitch;
    a.slot_bytes = a.ROWS * pitch;
    a.c0 = op->center;
    a.c0diff = op->center;
    for (int cc = 0; cc < 3; ++cc)
      for (int m = 0; m < 2 * HMAX + 1; ++m) a.c0diff += op->a[cc][m];
    memcpy(a.a, op->a, sizeof(a.a));
    a.c0f = (float)a.c0;
    a.c0difff = (float)a.c0diff;
    for (int cc = 0; cc < 3; ++cc)
      for (int m = 0; m < 2 * HMAX + 1; ++m) a.af[cc][m] = (float)op->a[cc][m];
    a.alpha = ep.alpha; a.beta = ep.beta; a.gamma = ep.gamma;
    const size_t smem = 256 + 128 + (size_t)a.NS * a.slot_bytes;
    // tensor maps over (n2 scalars, n1, n0, nbatch); the box spans the whole
    // padded pitch, so the columns past n2 arrive as zeros
    const int scal = Elem<T>::cplx ? 2 : 1;
    const CUtensorMapDataType dt = sizeof(R) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const uint64_t es = sizeof(R);
    const uint64_t dims[4] = {(uint64_t)n2 * scal, (uint64_t)n1, (uint64_t)n0, (uint64_t)nin};
    const uint64_t strides[3] = {dims[0] * es, dims[0] * dims[1] * es, dims[0] * dims[1] * dims[2] * es};
    const uint32_t bx = (uint32_t)(pitch / (int)es);
    CUtensorMap tmA, tmH, tmB, tmL;
    const uint32_t boxA[4] = {bx, (uint32_t)a.ROWS, 1, 1};
    const uint32_t boxH[4] = {bx, (uint32_t)H, 1, 1};
    const uint32_t boxB[4] = {bx, (uint32_t)(a.T1 + H), 1, 1};
    const uint32_t boxL[4] = {bx, (uint32_t)(a.T1L + H), 1, 1};
    void* base = const_cast<void*>(in);
    if (!encode_tensor_map_4d(&tmA, dt, base, dims, strides, boxA) ||
        !encode_tensor_map_4d(&tmH, dt, base, dims, strides, boxH) ||
        !encode_tensor_map_4d(&tmB, dt, base, dims, strides, boxB) ||
        !encode_tensor_map_4d(&tmL, dt, base, dims, strides, boxL)) {
      g_tma_reason = "cuTensorMapEncodeTiled rejected the layout";
      return 1;
    }
    const int threads = ((a.NTC + 31) / 32) * 32 + 32;
    const int64_t total = nin * (int64_t)a.ytiles * n0;
    int64_t blocks = (int64_t)sm_count() * std::min(occ_of[c], cb.ctas);
    blocks = std::min<int64_t>(blocks, std::max<int64_t>(1, total / (4 * H + 4)));
    kern<<<(unsigned)blocks, threads, smem, st>>>(tmA, tmH, tmB, tmL, a);
    return check_launch("star_tma_kernel");
  };

  // autotuning: the first call for a layout (grid, boundaries, dtype, radius,
  // epilogue kind, batch) times the candidates with CUDA events on its own
  // data -- every launch writes the same output, so the call stays exact --
  // and later calls launch the winner.  Inside a stream capture, or if timing
  // fails, the model's best candidate is used without tuning.
  const int epi_kind = (ep.vpot ? 4 : 0) | (ep.y ? 2 : 0) | ((ep.alpha != 1.0 || ep.beta != 0.0) ? 1 : 0);
  char keyb[160];
  snprintf(keyb, sizeof keyb, "%d:%d:%d:%d:%d:%d:%d:%d:%d:%d:%d:%lld", (int)sizeof(T), Elem<T>::cplx ? 1 : 0, H, n0,
           n1, n2, op->pbc[0] * 4 + op->pbc[1] * 2 + op->pbc[2], epi_kind, (int)VB, R2, SYM, (long long)nin);
  const std::string key(keyb);
  int choice = -1;
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto f = g_tune.find(key);
    if (f != g_tune.end())
      for (int c = 0; c < nok; ++c)
        if (ok[c].ty == f->second) choice = c;
  }
  if (choice < 0 && nok > 1 && autotune_enabled()) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st, &cs);
    if (cs == cudaStreamCaptureStatusNone) {
      // one warm-up round, then three rounds that time every candidate once
      // each, interleaved, keeping each candidate's fastest launch: clock
      // ramps and the cache state left by the previous launch affect every
      // candidate alike
      cudaEvent_t e0, e1;
      if (cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess) {
        float t_c[16];
        bool bad_c[16];
        for (int c = 0; c < nok; ++c) {
          t_c[c] = 1e30f;
          bad_c[c] = launch(c) != 0;
        }
        for (int round = 0; round < 3; ++round)
          for (int c = 0; c < nok; ++c) {
            if (bad_c[c]) continue;
            cudaEventRecord(e0, st);
            bad_c[c] = launch(c) != 0;
            cudaEventRecord(e1, st);
            float ms = 0.f;
            if (!bad_c[c] && cudaEventSynchronize(e1) == cudaSuccess &&
                cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess)
              t_c[c] = std::min(t_c[c], ms);
          }
        float best_ms = 1e30f;
        for (int c = 0; c < nok; ++c)
          if (!bad_c[c] && t_c[c] < best_ms) {
            best_ms = t_c[c];
            choice = c;
          }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
      }
      cudaGetLastError();
      if (choice >= 0) {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        g_tune[key] = ok[choice].ty;
      }
    }
  }
  if (choice < 0) choice = 0;
  return launch(choice);
}

static int g_stencil_path = 0;   // 0 auto, 1 cp.async only, 2 TMA required
const char* tma_reason() { return g_tma_reason; }

int star_tma_apply(const gb_operator* op, const void* in, void* out, int64_t nin, int dtype, const double* ph,
                   cudaStream_t st, const Epilogue& ep, int nk) {
  g_tma_reason = "";
  if (g_stencil_path == 1) { g_tma_reason = "cp.async path forced"; return 1; }
  if (!op->cfd || op->H > 4) { g_tma_reason = "stencil not on axes or radius > 4"; return 1; }
  if (ph) {
    for (int i = 0; i < 6 * (nk > 1 ? nk : 1); ++i)
      if (ph[2 * i] != 1.0 || ph[2 * i + 1] != 0.0) { g_tma_reason = "Bloch phases"; return 1; }
  }
  const size_t es = dtype_size(dtype);
  const int n2 = (int)op->n[2];
  if ((n2 * es) % 16 != 0 || n2 * es / (dtype_complex(dtype) ? es / 2 : es) > 256) {
    g_tma_reason = "row pitch not a multiple of 16 bytes or row longer than a TMA box";
    return 1;
  }
  if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15) { g_tma_reason = "unaligned data"; return 1; }
  if (ep.y && (reinterpret_cast<uintptr_t>(ep.y) & 15)) { g_tma_reason = "unaligned y"; return 1; }
  if (ep.vpot && (reinterpret_cast<uintptr_t>(ep.vpot) & 15)) { g_tma_reason = "unaligned potential"; return 1; }
  if (op->n[0] < op->H || op->n[1] < op->H || op->n[2] < 8) { g_tma_reason = "grid shorter than the stencil"; return 1; }
  switch (dtype) {
    case GB_DTYPE_F64:
      switch (op->H) {
        case 1: return launch_tma_cfg<double, 1, 2, 2>(op, in, out, nin, st, ep);
        case 2: return launch_tma_cfg<double, 2, 2, 2>(op, in, out, nin, st, ep);
        case 3: return launch_tma_cfg<double, 3, 2, 2>(op, in, out, nin, st, ep);
        default: return launch_tma_cfg<double, 4, 2, 2>(op, in, out, nin, st, ep);
      }
    case GB_DTYPE_F32: {
      // coefficient symmetry of every axis, in FP32: symmetric pairs (the
      // Laplacian) and antisymmetric pairs (derivatives) take fewer
      // operations in the packed kernel
      bool sym = true, anti = true;
      for (int c = 0; c < 3; ++c)
        for (int k = 1; k <= HMAX; ++k) {
          const float p = (float)op->a[c][HMAX + k], m = (float)op->a[c][HMAX - k];
          sym = sym && p == m;
          anti = anti && p == -m;
        }
      const int kind = sym ? 1 : (anti ? -1 : 0);
#define GB_F32_TMA(HH)                                                                      \
  return kind == 1 ? launch_tma_cfg<float, HH, 2, 4, 16, 1>(op, in, out, nin, st, ep)       \
                   : kind == -1 ? launch_tma_cfg<float, HH, 2, 4, 16, -1>(op, in, out, nin, st, ep) \
                                : launch_tma_cfg<float, HH, 2, 4, 16, 0>(op, in, out, nin, st, ep)
      switch (op->H) {
        case 1: GB_F32_TMA(1);
        case 2: GB_F32_TMA(2);
        case 3: GB_F32_TMA(3);
        default: GB_F32_TMA(4);
      }
#undef GB_F32_TMA
    }
    case GB_DTYPE_C128:
      switch (op->H) {
        case 1: return launch_tma_cfg<double2, 1, 2, 1>(op, in, out, nin, st, ep);
        case 2: return launch_tma_cfg<double2, 2, 2, 1>(op, in, out, nin, st, ep);
        case 3: return launch_tma_cfg<double2, 3, 2, 1>(op, in, out, nin, st, ep);
        default: return launch_tma_cfg<double2, 4, 2, 1>(op, in, out, nin, st, ep);
      }
    default:
      switch (op->H) {
        case 1: return launch_tma_cfg<float2, 1, 2, 2>(op, in, out, nin, st, ep);
        case 2: return launch_tma_cfg<float2, 2, 2, 2>(op, in, out, nin, st, ep);
        case 3: return launch_tma_cfg<float2, 3, 2, 2>(op, in, out, nin, st, ep);
        default: return launch_tma_cfg<float2, 4, 2, 2>(op, in, out, nin, st, ep);
      }
  }
}

void set_stencil_path(int mode) { g_stencil_path = mode; }
int stencil_path() { return g_stencil_path; }

}  // namespace gb

extern "C" {

int gb_set_stencil_path(int mode) {
  if (mode < 0 || mode > 2) return gb::fail(GB_E_INVALID, "gb_set_stencil_path: mode must be 0, 1 or 2");
  gb::set_stencil_path(mode);
  return GB_OK;
}

int gb_device_errors(int clear, int* code) {
  if (!code) return gb::fail(GB_E_INVALID, "gb_device_errors: null pointer");
  *code = gb::device_error_flag(clear);
  const int tc = gb::band_tc_error_flag(clear);
  if (!*code) *code = tc;
  const int ctc = gb::conv_tc_error_flag(clear);
  if (!*code) *code = ctc;
  return GB_OK;
}

}  // extern "C"
