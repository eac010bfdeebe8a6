// Density accumulation (replaces _gpaw.add_to_density: c/utilities.c:313-,
// called once per band by gpaw/wavefunctions/fd.py:95-100).  One launch for
// all bands: nt_G[G] += sum_n f_n |psit_n(G)|^2, accumulated in FP64 for
// every wave-function precision.  One thread per grid point walks the bands
// (coalesced band-by-band reads; the sum over bands stays in a register).
#include <algorithm>
#include "internal.cuh"

namespace gb {

__device__ __forceinline__ double abs2(double v) { return v * v; }
__device__ __forceinline__ double abs2(float v) { return (double)v * (double)v; }
__device__ __forceinline__ double abs2(double2 v) { return v.x * v.x + v.y * v.y; }
__device__ __forceinline__ double abs2(float2 v) { return (double)v.x * v.x + (double)v.y * v.y; }

template <typename T>
__global__ void add_to_density_kernel(const double* __restrict__ f_n, const T* __restrict__ psit, int64_t nb,
                                      int64_t nG, double* __restrict__ nt) {
  for (int64_t G = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; G < nG; G += (int64_t)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int64_t n = 0; n < nb; ++n) acc = fma(f_n[n], abs2(psit[n * nG + G]), acc);
    nt[G] += acc;
  }
}

}  // namespace gb

extern "C" int gb_add_to_density(int64_t nb, const double* f_n, const void* psit_nG, int dtype, int64_t nG,
                                 double* nt_G, void* stream) {
  GB_REQUIRE(nb >= 0 && nG >= 0 && gb::dtype_valid(dtype), "gb_add_to_density: bad arguments");
  if (nb == 0 || nG == 0) return GB_OK;
  GB_REQUIRE(f_n && psit_nG && nt_G, "gb_add_to_density: null pointer");
  const int threads = 256;
  const int64_t blocks = std::min<int64_t>((nG + threads - 1) / threads, (int64_t)gb::sm_count() * 8);
  cudaStream_t st = (cudaStream_t)stream;
  switch (dtype) {
    case GB_DTYPE_F64:
      gb::add_to_density_kernel<double><<<(unsigned)blocks, threads, 0, st>>>(f_n, (const double*)psit_nG, nb, nG, nt_G);
      break;
    case GB_DTYPE_F32:
      gb::add_to_density_kernel<float><<<(unsigned)blocks, threads, 0, st>>>(f_n, (const float*)psit_nG, nb, nG, nt_G);
      break;
    case GB_DTYPE_C128:
      gb::add_to_density_kernel<double2><<<(unsigned)blocks, threads, 0, st>>>(f_n, (const double2*)psit_nG, nb, nG, nt_G);
      break;
    default:
      gb::add_to_density_kernel<float2><<<(unsigned)blocks, threads, 0, st>>>(f_n, (const float2*)psit_nG, nb, nG, nt_G);
  }
  return gb::check_launch("add_to_density_kernel");
}
