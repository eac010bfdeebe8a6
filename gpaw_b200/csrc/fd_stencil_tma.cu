// FD star stencil, TMA + warp-specialised pipeline (the default path on
// sm_100a whenever the layout allows it; fd_stencil.cu keeps the cp.async
// kernel for the other cases: odd row pitches, Bloch phases, radius > 4).
//
// Tile = a band of T1 full rows of the (axis1, axis2) plane: because a CTA
// holds whole rows, the axis-2 halo of a periodic grid is read from the other
// end of the same shared-memory row (no wrap-around copies), and only the
// axis-1 halo rows of the first / last tile need a second TMA box.  One
// producer warp streams planes (tile + halo rows) into a ring of NS slots
// with cp.async.bulk.tensor (zero boundaries come from the TMA out-of-bounds
// fill); consumer warps keep the axis-0 register queue of the cp.async kernel
// and hand each slot back through an mbarrier when its last reader is done.
// All waits are bounded (tma.cuh).
#include <algorithm>
#include <cstring>
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
struct TmaArgs {
  void* out;
  const void* y;
  int64_t nbatch;
  int n0, n1, n2;
  int pbc0, pbc1, pbc2;
  int TY, TZ, NTC, T1, ROWS, ytiles;
  int slot_bytes;
  double c0;
  double c0diff;   // c0 + sum of the neighbour coefficients (difference form)
  double a[3][2 * HMAX + 1];
  double alpha, beta, gamma;
  const void* vpot;
};

template <typename T, int H, int R1, int R2, int NS>
__global__ void star_tma_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmH,
                                const __grid_constant__ CUtensorMap tmB, const TmaArgs a) {
  using R = typename Elem<T>::R;
  constexpr int VEC = 16 / (int)sizeof(T);
  constexpr int HZ = ((H + VEC - 1) / VEC) * VEC;
  static_assert(R2 % VEC == 0, "");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // 128-byte aligned base for the TMA destinations
  unsigned char* smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + NS;
  unsigned char* slots = smem + 128;

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int NWC = (a.NTC + 31) >> 5;       // consumer warps
  const int n0 = a.n0, n1 = a.n1, n2 = a.n2;
  const int T1 = a.T1, ROWS = a.ROWS;
  const int64_t rowb = (int64_t)n2 * sizeof(T);
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

  // split row of a tile's slot layout (rows < rs in part 0, the rest in part 1)
  auto split_row = [&](int y0) -> int {
    if (a.pbc1 && y0 == 0) return H;
    if (a.pbc1 && y0 + T1 == n1) return T1 + H;
    return ROWS;
  };
  auto part1_off = [&](int rs) -> int64_t { return ((rs * rowb + 127) / 128) * 128; };

  if (warp == NWC) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      tma_prefetch_desc(&tmA);
      tma_prefetch_desc(&tmH);
      tma_prefetch_desc(&tmB);
      long long k = 0;
      int64_t s = s_begin;
      while (s < s_end) {
        const int64_t col = s / n0;
        const int p_start = (int)(s % n0);
        const int p_end = (int)((s_end - s) < (int64_t)(n0 - p_start) ? p_start + (s_end - s) : n0);
        s += p_end - p_start;
        const int band = (int)(col / a.ytiles);
        const int y0 = (int)(col % a.ytiles) * T1;
        const int rs = split_row(y0);
        for (int j = p_start - H; j < p_end + H; ++j, ++k) {
          const int slot = (int)(k % NS);
          if (k >= NS && !mbar_wait(&empty[slot], (uint32_t)(((k / NS) - 1) & 1))) {
            raise_device_error(101);
            return;
          }
          int sp = j;
          if (j < 0 || j >= n0) sp = a.pbc0 ? (j < 0 ? j + n0 : j - n0) : -1;
          if (sp < 0) {
            mbar_arrive(&full[slot]);
            continue;
          }
          unsigned char* dst = slots + (int64_t)slot * a.slot_bytes;
          if (rs == ROWS) {
            mbar_arrive_expect_tx(&full[slot], (uint32_t)(ROWS * rowb));
            tma_load_4d(dst, &tmA, &full[slot], 0, y0 - H, sp, band);
          } else if (rs == H) {        // first tile of a periodic axis 1
            mbar_arrive_expect_tx(&full[slot], (uint32_t)(ROWS * rowb));
            tma_load_4d(dst, &tmH, &full[slot], 0, n1 - H, sp, band);
            tma_load_4d(dst + part1_off(H), &tmB, &full[slot], 0, 0, sp, band);
          } else {                     // last tile of a periodic axis 1
            mbar_arrive_expect_tx(&full[slot], (uint32_t)(ROWS * rowb));
            tma_load_4d(dst, &tmB, &full[slot], 0, y0 - H, sp, band);
            tma_load_4d(dst + part1_off(T1 + H), &tmH, &full[slot], 0, 0, sp, band);
          }
        }
      }
    }
    return;
  }

  // -------------------------------------------------------------- consumers
  const bool active = tid < a.NTC;
  const int ty = active ? tid / a.TZ : 0, tz = active ? tid % a.TZ : 0;
  // FP32: the difference form sum_p c_p (x_p - x_c) + (sum c) x_c keeps the
  // operator exactly constant-annihilating after the coefficients are rounded
  // (otherwise every eigenvalue shifts by ~|c0| 2^-24)
  constexpr bool DIFF = sizeof(R) == 4;
  const R c0 = DIFF ? (R)a.c0diff : (R)a.c0;
  R a0[2 * H + 1], a1[2 * H + 1], a2[2 * H + 1];
#pragma unroll
  for (int m = 0; m <= 2 * H; ++m) {
    a0[m] = (R)a.a[0][m - H + HMAX];
    a1[m] = (R)a.a[1][m - H + HMAX];
    a2[m] = (R)a.a[2][m - H + HMAX];
  }
  const bool epi = a.alpha != 1.0 || a.beta != 0.0 || a.y != nullptr || a.vpot != nullptr;
  const R* __restrict__ vpot = reinterpret_cast<const R*>(a.vpot);
  const R ealpha = (R)a.alpha, ebeta = (R)a.beta, egamma = (R)a.gamma;

  long long k = 0;
  int64_t s = s_begin;
  while (s < s_end) {
    const int64_t col = s / n0;
    const int p_start = (int)(s % n0);
    const int p_end = (int)((s_end - s) < (int64_t)(n0 - p_start) ? p_start + (s_end - s) : n0);
    s += p_end - p_start;
    const int64_t band = col / a.ytiles;
    const int y0 = (int)(col % a.ytiles) * T1;
    const int rs = split_row(y0);
    const int64_t off1 = part1_off(rs);
    T* dst = reinterpret_cast<T*>(a.out) + band * n12 * n0;
    const T* ybase = a.y ? reinterpret_cast<const T*>(a.y) + band * n12 * n0 : nullptr;
    // address of (row, col) in a slot
    auto cell = [&](const unsigned char* base, int row, int c) -> const T* {
      const int64_t rb = row < rs ? row * rowb : off1 + (row - rs) * rowb;
      return reinterpret_cast<const T*>(base + rb) + c;
    };

    T q[2 * H + 1][R1][R2];
#pragma unroll
    for (int m = 0; m <= 2 * H; ++m)
#pragma unroll
      for (int r = 0; r < R1; ++r)
#pragma unroll
        for (int c = 0; c < R2; ++c) q[m][r][c] = zero<T>();

    const int j0 = p_start - H, j1 = p_end + H;
    const long long k0 = k;
    for (int j = j0; j < j1; ++j, ++k) {
      const int slot = (int)(k % NS);
      if (!mbar_wait(&full[slot], (uint32_t)((k / NS) & 1))) {
        raise_device_error(102);
        return;
      }
      const bool zplane = (j < 0 || j >= n0) && !a.pbc0;
      const unsigned char* P = slots + (int64_t)slot * a.slot_bytes;
#pragma unroll
      for (int m = 0; m < 2 * H; ++m)
#pragma unroll
        for (int r = 0; r < R1; ++r)
#pragma unroll
          for (int c = 0; c < R2; ++c) q[m][r][c] = q[m + 1][r][c];
#pragma unroll
      for (int r = 0; r < R1; ++r) {
        T v[R2];
        if (!zplane && active) {
          lds_vec<T, R2>(cell(P, H + ty * R1 + r, tz * R2), v);
        } else {
#pragma unroll
          for (int c = 0; c < R2; ++c) v[c] = zero<T>();
        }
#pragma unroll
        for (int c = 0; c < R2; ++c) q[2 * H][r][c] = v[c];
      }
      const int cpl = j - H;
      if (cpl >= p_start && active) {
        const unsigned char* Pc = slots + (int64_t)((k - H) % NS) * a.slot_bytes;
        T acc[R1][R2];
        const int zl = tz * R2 - HZ, zr = tz * R2 + R2;
#pragma unroll
        for (int r = 0; r < R1; ++r) {
          const int row = H + ty * R1 + r;
          T wl[HZ], wr[HZ];
#pragma unroll
          for (int cch = 0; cch < HZ / VEC; ++cch) {
            int zc = zl + cch * VEC;
            T tmp[VEC];
            if (zc < 0 && !a.pbc2) {
#pragma unroll
              for (int v = 0; v < VEC; ++v) tmp[v] = zero<T>();
            } else {
              if (zc < 0) zc += n2;
              lds_vec<T, VEC>(cell(Pc, row, zc), tmp);
            }
#pragma unroll
            for (int v = 0; v < VEC; ++v) wl[cch * VEC + v] = tmp[v];
            int zc2 = zr + cch * VEC;
            if (zc2 >= n2 && !a.pbc2) {
#pragma unroll
              for (int v = 0; v < VEC; ++v) tmp[v] = zero<T>();
            } else {
              if (zc2 >= n2) zc2 -= n2;
              lds_vec<T, VEC>(cell(Pc, row, zc2), tmp);
            }
#pragma unroll
            for (int v = 0; v < VEC; ++v) wr[cch * VEC + v] = tmp[v];
          }
#pragma unroll
          for (int c = 0; c < R2; ++c) {
            T x = scale(c0, q[H][r][c]);
#pragma unroll
            for (int m = 0; m <= 2 * H; ++m)
              if (m != H) x = fmadd(x, a0[m], DIFF ? sub(q[m][r][c], q[H][r][c]) : q[m][r][c]);
#pragma unroll
            for (int m = 0; m <= 2 * H; ++m) {
              if (m == H) continue;
              const int cc = c + m - H;
              T v;
              if (cc < 0) v = wl[HZ + cc];
              else if (cc >= R2) v = wr[cc - R2];
              else v = q[H][r][cc];
              x = fmadd(x, a2[m], DIFF ? sub(v, q[H][r][c]) : v);
            }
            acc[r][c] = x;
          }
        }
#pragma unroll
        for (int rr = -H; rr < R1 + H; ++rr) {
          T v[R2];
          if (rr >= 0 && rr < R1) {
#pragma unroll
            for (int c = 0; c < R2; ++c) v[c] = q[H][rr][c];
          } else {
            lds_vec<T, R2>(cell(Pc, H + ty * R1 + rr, tz * R2), v);
          }
#pragma unroll
          for (int r = 0; r < R1; ++r) {
            const int m = rr - r + H;
            if (m < 0 || m > 2 * H || m == H) continue;
#pragma unroll
            for (int c = 0; c < R2; ++c)
              acc[r][c] = fmadd(acc[r][c], a1[m], DIFF ? sub(v[c], q[H][r][c]) : v[c]);
          }
        }
        T* outp = dst + (int64_t)cpl * n12;
        const T* yp = ybase ? ybase + (int64_t)cpl * n12 : nullptr;
#pragma unroll
        for (int r = 0; r < R1; ++r) {
          const int yy = y0 + ty * R1 + r;
          if (yy >= n1) continue;
          T* o = outp + (int64_t)yy * n2 + tz * R2;
          if (epi) {
#pragma unroll
            for (int c = 0; c < R2; ++c) {
              T v = fmadd(scale(ealpha, acc[r][c]), ebeta, q[H][r][c]);
              if (yp) v = fmadd(v, egamma, yp[(int64_t)yy * n2 + tz * R2 + c]);
              if (vpot) v = fmadd(v, vpot[(int64_t)cpl * n12 + (int64_t)yy * n2 + tz * R2 + c], q[H][r][c]);
              acc[r][c] = v;
            }
          }
#pragma unroll
          for (int c = 0; c < R2; c += VEC) {
            float4 w4;
            T* e = reinterpret_cast<T*>(&w4);
#pragma unroll
            for (int v = 0; v < VEC; ++v) e[v] = acc[r][c + v];
            __stcs(reinterpret_cast<float4*>(o + c), w4);
          }
        }
      }
      // hand back the slot of plane j - H (its last reader was this step)
      if (j - H >= j0) {
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[(int)((k - H) % NS)]);
      }
    }
    // segment end: release the slots of the last H planes
    for (long long kk = (k - H > k0 ? k - H : k0); kk < k; ++kk) {
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[(int)(kk % NS)]);
    }
  }
}

// ------------------------------------------------------------------ host
template <typename T, int H, int R1, int R2>
static int launch_tma_cfg(const gb_operator* op, const void* in, void* out, int64_t nin, cudaStream_t st,
                          const Epilogue& ep) {
  constexpr int NS = H + 3;
  const int n0 = (int)op->n[0], n1 = (int)op->n[1], n2 = (int)op->n[2];
  const int TZ = n2 / R2;
  auto kern = star_tma_kernel<T, H, R1, R2, NS>;
  static int regs = -1;
  if (regs < 0) {
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, kern) != cudaSuccess) { g_tma_reason = "cudaFuncGetAttributes failed"; return 1; }
    regs = fa.numRegs;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
  }
  // rows per tile: periodic axis 1 needs T1 | n1 and at least two tiles;
  // pick the tile that keeps the most consumer threads resident per SM
  // (registers and shared memory both limit the CTAs per SM).
  // candidate tiles, best score first; the first one the occupancy
  // calculator accepts is used
  struct Cand { double score; int ty; };
  Cand cands[64];
  int ncand = 0;
  const int64_t rowb0 = (int64_t)n2 * sizeof(T);
  for (int ty = 1; ty * TZ <= 1024 - 32 && ncand < 64; ++ty) {
    const int T1 = ty * R1;
    if (T1 < H || T1 + 2 * H > 256) continue;
    if (op->pbc[1] && (n1 % T1 != 0 || n1 / T1 < 2)) continue;
    if (!op->pbc[1] && T1 > n1 + R1 - 1) continue;
    const int threads = ((ty * TZ + 31) / 32) * 32 + 32;
    const int regs_cta = threads * ((regs + 7) / 8 * 8);
    const int by_regs = 65536 / regs_cta;
    const int64_t slot = ((T1 + 2 * H) * rowb0 + 128 + 127) / 128 * 128;
    const int64_t smem_cta = 256 + NS * slot;
    if (smem_cta > 220 * 1024) continue;
    const int by_smem = (int)((228 * 1024) / (smem_cta + 1024));
    const int ctas = std::min(by_regs, by_smem);
    if (ctas < 1) continue;
    // resident consumer threads, discounted by the halo re-read overhead
    cands[ncand++] = {(double)ctas * ty * TZ * T1 / (T1 + 2.0 * H), ty};
  }
  std::sort(cands, cands + ncand, [](const Cand& x, const Cand& y) { return x.score > y.score; });
  int best_ty = -1, occ = 0, threads = 0;
  size_t smem = 0;
  for (int c = 0; c < ncand && best_ty < 0; ++c) {
    const int ty = cands[c].ty;
    const int T1 = ty * R1;
    const int slotb = (int)((((T1 + 2 * H) * rowb0 + 128) + 127) / 128 * 128);
    const size_t sm = 256 + (size_t)NS * slotb;
    const int th = ((ty * TZ + 31) / 32) * 32 + 32;
    int o = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, th, sm) == cudaSuccess && o >= 1) {
      best_ty = ty; occ = o; threads = th; smem = sm;
    }
  }
  cudaGetLastError();
  if (best_ty < 0) {
    g_tma_reason = ncand ? "zero occupancy" : "no row tile fits the grid (periodic axis 1 needs T1 | n1)";
    return 1;
  }
  TmaArgs a{};
  a.out = out; a.y = ep.y; a.nbatch = nin;
  a.n0 = n0; a.n1 = n1; a.n2 = n2;
  a.pbc0 = op->pbc[0]; a.pbc1 = op->pbc[1]; a.pbc2 = op->pbc[2];
  a.TY = best_ty; a.TZ = TZ; a.NTC = best_ty * TZ; a.T1 = best_ty * R1; a.ROWS = a.T1 + 2 * H;
  a.ytiles = ceil_div(n1, a.T1);
  const int64_t rowb = (int64_t)n2 * sizeof(T);
  a.slot_bytes = (int)(((a.ROWS * rowb + 128) + 127) / 128 * 128);
  a.c0 = op->center;
  a.c0diff = op->center;
  for (int c = 0; c < 3; ++c)
    for (int m = 0; m < 2 * HMAX + 1; ++m) a.c0diff += op->a[c][m];
  memcpy(a.a, op->a, sizeof(a.a));
  a.alpha = ep.alpha; a.beta = ep.beta; a.gamma = ep.gamma; a.vpot = ep.vpot;
  if (smem > 220 * 1024 || a.ROWS > 256) { g_tma_reason = "tile too large"; return 1; }
  // tensor maps over (n2 scalars, n1, n0, nbatch)
  const int scal = Elem<T>::cplx ? 2 : 1;
  const CUtensorMapDataType dt = sizeof(typename Elem<T>::R) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                                                  : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const uint64_t es = sizeof(typename Elem<T>::R);
  const uint64_t dims[4] = {(uint64_t)n2 * scal, (uint64_t)n1, (uint64_t)n0, (uint64_t)nin};
  const uint64_t strides[3] = {dims[0] * es, dims[0] * dims[1] * es, dims[0] * dims[1] * dims[2] * es};
  CUtensorMap tmA, tmH, tmB;
  const uint32_t boxA[4] = {(uint32_t)dims[0], (uint32_t)a.ROWS, 1, 1};
  const uint32_t boxH[4] = {(uint32_t)dims[0], (uint32_t)H, 1, 1};
  const uint32_t boxB[4] = {(uint32_t)dims[0], (uint32_t)(a.T1 + H), 1, 1};
  void* base = const_cast<void*>(in);
  if (!encode_tensor_map_4d(&tmA, dt, base, dims, strides, boxA) ||
      !encode_tensor_map_4d(&tmH, dt, base, dims, strides, boxH) ||
      !encode_tensor_map_4d(&tmB, dt, base, dims, strides, boxB)) {
    g_tma_reason = "cuTensorMapEncodeTiled rejected the layout";
    return 1;
  }
  const int64_t total = nin * (int64_t)a.ytiles * n0;
  int64_t blocks = (int64_t)sm_count() * occ;
  blocks = std::min<int64_t>(blocks, std::max<int64_t>(1, total / (4 * H + 4)));
  kern<<<(unsigned)blocks, threads, smem, st>>>(tmA, tmH, tmB, a);
  const int rc = check_launch("star_tma_kernel");
  return rc;
}

static int g_stencil_path = 0;   // 0 auto, 1 cp.async only, 2 TMA required
const char* tma_reason() { return g_tma_reason; }

int star_tma_apply(const gb_operator* op, const void* in, void* out, int64_t nin, int dtype, const double* ph,
                   cudaStream_t st, const Epilogue& ep) {
  g_tma_reason = "";
  if (g_stencil_path == 1) { g_tma_reason = "cp.async path forced"; return 1; }
  if (!op->cfd || op->H > 4) { g_tma_reason = "stencil not on axes or radius > 4"; return 1; }
  if (ph) {
    for (int i = 0; i < 6; ++i)
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
  if (op->n[0] < op->H || op->n[1] < op->H) { g_tma_reason = "grid shorter than the stencil"; return 1; }
  switch (dtype) {
    case GB_DTYPE_F64:
      switch (op->H) {
        case 1: return launch_tma_cfg<double, 1, 2, 2>(op, in, out, nin, st, ep);
        case 2: return launch_tma_cfg<double, 2, 2, 2>(op, in, out, nin, st, ep);
        case 3: return launch_tma_cfg<double, 3, 2, 2>(op, in, out, nin, st, ep);
        default: return launch_tma_cfg<double, 4, 2, 2>(op, in, out, nin, st, ep);
      }
    case GB_DTYPE_F32:
      switch (op->H) {
        case 1: return launch_tma_cfg<float, 1, 2, 4>(op, in, out, nin, st, ep);
        case 2: return launch_tma_cfg<float, 2, 2, 4>(op, in, out, nin, st, ep);
        case 3: return launch_tma_cfg<float, 3, 2, 4>(op, in, out, nin, st, ep);
        default: return launch_tma_cfg<float, 4, 2, 4>(op, in, out, nin, st, ep);
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
  return GB_OK;
}

}  // extern "C"
