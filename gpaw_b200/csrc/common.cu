// Error state, device queries and version for libgpawb200.
#include <string>
#include "internal.cuh"

namespace gb {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(GB_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return GB_OK;
}

int sm_count() {
  static int cached[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  if (cached[dev] == 0) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    cached[dev] = n > 0 ? n : 1;
  }
  return cached[dev];
}

void fill_phase_sets(PhaseSets& p, const double* src, int nk, int64_t nbatch) {
  p.nk = nk < 1 ? 1 : nk;
  p.per_k = p.nk > 1 ? nbatch / p.nk : nbatch;
  if (p.per_k < 1) p.per_k = 1;
  p.any = 0;
  for (int k = 0; k < KMAX; ++k)
    for (int c = 0; c < 3; ++c)
      for (int d = 0; d < 2; ++d) {
        const bool have = src && k < p.nk;
        p.ph[k][c][d][0] = have ? src[k * 12 + (c * 2 + d) * 2] : 1.0;
        p.ph[k][c][d][1] = have ? src[k * 12 + (c * 2 + d) * 2 + 1] : 0.0;
        if (p.ph[k][c][d][0] != 1.0 || p.ph[k][c][d][1] != 0.0) p.any = 1;
      }
}

}  // namespace gb

extern "C" {

const char* gb_last_error(void) { return gb::g_last_error.c_str(); }

const char* gb_version(void) { return "gpawb200 0.1 (sm_100a)"; }

int gb_device_sm_count(int* n) {
  if (!n) return gb::fail(GB_E_INVALID, "gb_device_sm_count: null pointer");
  *n = gb::sm_count();
  return GB_OK;
}

}  // extern "C"
