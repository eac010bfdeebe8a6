// Multigrid V-cycle without any device allocation (no reference counterpart).
//
// gb_fd_precond needs seven work grids that its caller allocates.  Some
// callers cannot allocate device memory while they run: a host program that
// drives the solver from C or Fortran and owns only the residual and result
// buffers it hands in, or a service whose device-memory budget is fixed when
// it starts and which must not grow afterwards.  gb_fd_precond_noalloc takes
// the same operators, residuals and output as gb_fd_precond and carves the
// work grids out of one fixed array that lives in the library itself.
//
// The array: g_precond_scratch below, PRECOND_SCRATCH_BYTES (64 MiB), a
// file-scope __device__ array, so every GPU that loads this library holds it
// until the process exits.  Host code cannot use its name as a device
// address; the first call on each device looks the address up with
// cudaGetSymbolAddress while that device is current and keeps it.  Make that
// first call before any stream capture begins on the device.  With CUDA's
// lazy module loading (CUDA_MODULE_LOADING=LAZY, the default since 12.2) the
// array is only placed in device memory by that first look-up, so a caller
// whose budget is fixed at start-up makes one call at start-up: a call with
// nin = 0 does the look-up and launches nothing.  The kept address belongs
// to the device's primary context: after cudaDeviceReset (or a reset of the
// primary context) it is stale, and this entry point must not be called on
// that device again in the same process.
//
// Size: q0 (one level-0 grid per band), r1, d1, q1 (level 1) and r2, d2
// (level 2), each rounded up to 256 bytes -- about 1.41 x nin x level-0
// points x element size.  A call that needs more fails with GB_E_INVALID
// and launches nothing; split the bands over several calls.
//
// Contents: every work grid is written in full by the launch that produces
// it before any launch reads it, so nothing in the array has to start at
// zero and what an earlier call left there is never read.  All calls share
// the one array: two calls whose launches can overlap on the GPU (different
// streams, or different host threads without ordering) overwrite each
// other's work grids.  Issue them on one stream or order them otherwise.
#include <mutex>

#include "internal.cuh"

using namespace gb;

namespace {

constexpr size_t PRECOND_SCRATCH_BYTES = size_t(64) << 20;

static __device__ __align__(256) unsigned char g_precond_scratch[PRECOND_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_scratch_mutex;
void* g_scratch_ptr[MAX_DEVICES] = {};

// device address of g_precond_scratch on the current device (looked up once)
int scratch_address(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(GB_E_CUDA, std::string("gb_fd_precond_noalloc: cudaGetDevice: ") +
                                                   cudaGetErrorString(e));
  if (dev < 0 || dev >= MAX_DEVICES) return fail(GB_E_UNSUPPORTED, "gb_fd_precond_noalloc: device index too large");
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_precond_scratch);
    if (e != cudaSuccess || !p)
      return fail(GB_E_CUDA, std::string("gb_fd_precond_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return GB_OK;
}

size_t round256(size_t b) { return (b + 255) / 256 * 256; }

}  // namespace

extern "C" int gb_fd_precond_noalloc(const gb_transformer* rest0, const gb_transformer* rest1,
                                     const gb_transformer* intp1, const gb_transformer* intp2,
                                     const gb_operator* kin0, const gb_operator* kin1, const gb_operator* kin2,
                                     void* d0, const void* residuals, double step, int64_t nin, int dtype,
                                     const double* phase_cd, void* stream) {
  GB_REQUIRE(kin0 && kin1 && kin2, "gb_fd_precond_noalloc: null operator");
  GB_REQUIRE(dtype_valid(dtype) && nin >= 0, "gb_fd_precond_noalloc: bad dtype or batch");
  void* base = nullptr;
  if (nin == 0) return scratch_address(&base);  // set-up only
  GB_REQUIRE(d0 && residuals, "gb_fd_precond_noalloc: null residuals or output");
  const size_t es = dtype_size(dtype);
  const size_t points0 = (size_t)(kin0->n[0] * kin0->n[1] * kin0->n[2]);
  // a batch whose level-0 grids alone exceed the array is refused before any
  // product that could wrap around
  if (points0 == 0 || (size_t)nin > PRECOND_SCRATCH_BYTES / (points0 * es))
    return fail(GB_E_INVALID, "gb_fd_precond_noalloc: " + std::to_string(nin) +
                                  " grids need more work space than the fixed " +
                                  std::to_string(PRECOND_SCRATCH_BYTES) + " bytes; pass fewer grids per call");
  auto level_bytes = [&](const gb_operator* k) {
    return round256((size_t)nin * (size_t)(k->n[0] * k->n[1] * k->n[2]) * es);
  };
  const size_t b0 = level_bytes(kin0), b1 = level_bytes(kin1), b2 = level_bytes(kin2);
  const size_t need = b0 + 3 * b1 + 2 * b2;
  if (need > PRECOND_SCRATCH_BYTES)
    return fail(GB_E_INVALID, "gb_fd_precond_noalloc: " + std::to_string(nin) + " grids need " +
                                  std::to_string(need) + " bytes of work space, more than the fixed " +
                                  std::to_string(PRECOND_SCRATCH_BYTES) + " bytes; pass fewer grids per call");
  int rc = scratch_address(&base);
  if (rc) return rc;
  unsigned char* p = static_cast<unsigned char*>(base);
  void* q0 = p;
  void* r1 = p + b0;
  void* d1 = p + b0 + b1;
  void* q1 = p + b0 + 2 * b1;
  void* r2 = p + b0 + 3 * b1;
  void* d2 = p + b0 + 3 * b1 + b2;
  // q2 is not touched by the V-cycle; d2 stands in for the pointer
  return gb_fd_precond(rest0, rest1, intp1, intp2, kin0, kin1, kin2, d0, q0, r1, d1, q1, r2, d2, d2, residuals,
                       nullptr, step, nin, dtype, phase_cd, stream);
}
