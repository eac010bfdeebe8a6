// Shared device/host helpers for libgpawb200 (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include "../../include/gpawb200.h"

namespace gb {

// ---------------------------------------------------------------- errors
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int check_launch(const char* what);

#define GB_REQUIRE(cond, msg)                                   \
  do {                                                          \
    if (!(cond)) return ::gb::fail(GB_E_INVALID, (msg));        \
  } while (0)

// ---------------------------------------------------------------- element types
// Complex values are stored interleaved; on the device they are float2/double2.
template <typename T> struct Elem;
template <> struct Elem<double>  { using R = double; static constexpr bool cplx = false; };
template <> struct Elem<float>   { using R = float;  static constexpr bool cplx = false; };
template <> struct Elem<double2> { using R = double; static constexpr bool cplx = true;  };
template <> struct Elem<float2>  { using R = float;  static constexpr bool cplx = true;  };

__host__ __device__ inline size_t dtype_size(int dtype) {
  return dtype == GB_DTYPE_F64 ? 8 : dtype == GB_DTYPE_F32 ? 4 : dtype == GB_DTYPE_C128 ? 16 : 8;
}
inline bool dtype_complex(int dtype) { return dtype == GB_DTYPE_C128 || dtype == GB_DTYPE_C64; }
inline bool dtype_valid(int dtype) { return dtype >= 0 && dtype <= 3; }

// arithmetic over real/complex element types with real scalars
__device__ __forceinline__ double  zero_of(double)  { return 0.0; }
__device__ __forceinline__ float   zero_of(float)   { return 0.f; }
__device__ __forceinline__ double2 zero_of(double2) { return make_double2(0.0, 0.0); }
__device__ __forceinline__ float2  zero_of(float2)  { return make_float2(0.f, 0.f); }

template <typename T> __device__ __forceinline__ T zero() { return zero_of(T()); }

// a + s*b  (s real)
__device__ __forceinline__ double  fmadd(double a, double s, double b) { return fma(s, b, a); }
__device__ __forceinline__ float   fmadd(float a, float s, float b)    { return fmaf(s, b, a); }
__device__ __forceinline__ double2 fmadd(double2 a, double s, double2 b) {
  return make_double2(fma(s, b.x, a.x), fma(s, b.y, a.y));
}
__device__ __forceinline__ float2 fmadd(float2 a, float s, float2 b) {
  return make_float2(fmaf(s, b.x, a.x), fmaf(s, b.y, a.y));
}
__device__ __forceinline__ double  scale(double s, double a) { return s * a; }
__device__ __forceinline__ float   scale(float s, float a)   { return s * a; }
__device__ __forceinline__ double2 scale(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
__device__ __forceinline__ float2  scale(float s, float2 a)   { return make_float2(s * a.x, s * a.y); }
__device__ __forceinline__ double  add(double a, double b) { return a + b; }
__device__ __forceinline__ float   add(float a, float b)   { return a + b; }
__device__ __forceinline__ double2 add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2  add(float2 a, float2 b)   { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double  sub(double a, double b) { return a - b; }
__device__ __forceinline__ float   sub(float a, float b)   { return a - b; }
__device__ __forceinline__ double2 sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2  sub(float2 a, float2 b)   { return make_float2(a.x - b.x, a.y - b.y); }

// multiplication by a complex phase (re, im) held in double precision;
// identity for real element types (the reference ignores phases for real
// arrays, c/operators.c:270-273).
__device__ __forceinline__ double  phase_mul(double a, double, double)  { return a; }
__device__ __forceinline__ float   phase_mul(float a, double, double)   { return a; }
__device__ __forceinline__ double2 phase_mul(double2 a, double pr, double pi) {
  return make_double2(a.x * pr - a.y * pi, a.x * pi + a.y * pr);
}
__device__ __forceinline__ float2 phase_mul(float2 a, double pr, double pi) {
  float r = (float)pr, i = (float)pi;
  return make_float2(a.x * r - a.y * i, a.x * i + a.y * r);
}

// ---------------------------------------------------------------- async copies
// cp.async (LDGSTS) global->shared, L2-only (.cg) for 16 B, .ca for 4/8 B.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(sdst)), "l"(gsrc));
}
__device__ __forceinline__ void cp_async8(void* sdst, const void* gsrc) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_u32(sdst)), "l"(gsrc));
}
__device__ __forceinline__ void cp_async4(void* sdst, const void* gsrc) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_u32(sdst)), "l"(gsrc));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <typename T>
__device__ __forceinline__ void cp_async_elem(T* sdst, const T* gsrc) {
  if constexpr (sizeof(T) == 16) cp_async16(sdst, gsrc);
  else if constexpr (sizeof(T) == 8) cp_async8(sdst, gsrc);
  else cp_async4(sdst, gsrc);
}

// streaming (evict-first) stores for outputs that are not re-read soon
__device__ __forceinline__ void st_cs(double* p, double v) { __stcs(p, v); }
__device__ __forceinline__ void st_cs(float* p, float v) { __stcs(p, v); }
__device__ __forceinline__ void st_cs(double2* p, double2 v) { __stcs(p, v); }
__device__ __forceinline__ void st_cs(float2* p, float2 v) { __stcs(p, v); }

inline int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

int sm_count();

}  // namespace gb
