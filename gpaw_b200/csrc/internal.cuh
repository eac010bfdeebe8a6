// Internal (non-ABI) declarations shared by the .cu files of libgpawb200.
#pragma once
#include <vector>
#include "common.cuh"

namespace gb {
static constexpr int HMAX = 6;   // largest axis radius handled by star_kernel

// Bloch phases: a launch covers nk equal groups of bands (k-points), each
// with its own phase_cd set; ph[k][axis][side][re/im].  Kernels pick the
// set of a band as band / per_k.
static constexpr int KMAX = 8;
struct PhaseSets {
  double ph[KMAX][3][2][2];
  int nk;            // sets in use (1 for a single k-point or real data)
  int64_t per_k;     // bands per set
  int any;           // some phase differs from 1
};
// fill from nk x 12 doubles ((c, side, re/im) per set; null: all 1)
void fill_phase_sets(PhaseSets& p, const double* src, int nk, int64_t nbatch);
__host__ __device__ inline int phase_set_of(const PhaseSets& p, int64_t band) {
  if (p.nk <= 1) return 0;
  const int64_t k = band / p.per_k;
  return (int)(k < p.nk ? k : p.nk - 1);
}

// out = alpha * Op(in) + beta * in + gamma * y + vpot * in
// (y may be null; vpot is an optional real grid of the operator's shape,
// broadcast over bands, in the element precision: the local potential)
struct Epilogue {
  double alpha = 1.0, beta = 0.0, gamma = 0.0;
  const void* y = nullptr;
  const void* vpot = nullptr;
};

}  // namespace gb

// operator object
struct gb_operator {
  int np;
  std::vector<double> coef;
  std::vector<int> off;    // np x 3
  int64_t n[3];
  int range;
  int pbc[3];
  int real;
  int cfd;                 // all offsets on axes -> star kernel
  int H;                   // largest axis offset
  double center;
  double a[3][2 * gb::HMAX + 1];
  double diag;
};


struct gb_transformer {
  int64_t nin_c[3], nout_c[3];
  int k;              // 2 * nn
  int interpolate;
  int real;
  int pbc[3];
  // restriction: fine centre of coarse i is 2 i + off[c];
  // interpolation: fine local f has global parity f + skip0[c], coarse local
  // index of fine global F (even) is F/2 - cbeg[c]
  int off[3];
  int skip0[3], skip1[3];
  int cbeg[3];
};

namespace gb {
// 16-byte vector load of N contiguous elements from shared memory
template <typename T, int N>
__device__ __forceinline__ void lds_vec(const T* p, T (&v)[N]) {
  constexpr int VEC = 16 / sizeof(T);
  static_assert(N % VEC == 0, "");
#pragma unroll
  for (int i = 0; i < N / VEC; ++i) {
    float4 x = *reinterpret_cast<const float4*>(p + i * VEC);
    const T* e = reinterpret_cast<const T*>(&x);
#pragma unroll
    for (int k = 0; k < VEC; ++k) v[i * VEC + k] = e[k];
  }
}


// ph: nk phase sets of 12 doubles (null for real data); the batch is split
// into nk equal groups of bands, one set each
int op_apply(const gb_operator* op, const void* in, void* out, int64_t nin, int dtype,
             const double* ph, cudaStream_t st, const Epilogue& ep, int nk = 1);
int tr_apply(const gb_transformer* t, const void* in, void* out, int64_t nin, int dtype,
             const double* ph, cudaStream_t st, double alpha, const void* y, double gamma, int nk = 1);
// TMA stencil path: returns 1 when the request is not eligible (caller falls back)
int star_tma_apply(const gb_operator* op, const void* in, void* out, int64_t nin, int dtype,
                   const double* ph, cudaStream_t st, const Epilogue& ep, int nk = 1);
void set_stencil_path(int mode);
const char* tma_reason();
int stencil_path();
}  // namespace gb
