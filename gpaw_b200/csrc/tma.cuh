// TMA (cp.async.bulk.tensor) and mbarrier helpers for sm_100a, written as
// inline PTX.  Every wait is bounded: after WAIT_LIMIT polls the caller gets
// `false`, records an error code in a device flag and leaves, so a fault in
// the pipeline protocol can never hang the GPU.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace gb {

constexpr long long WAIT_LIMIT = 1LL << 25;   // ~ seconds of polling

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"((uint32_t)__cvta_generic_to_shared(bar)),
               "r"(count));
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"((uint32_t)__cvta_generic_to_shared(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"((uint32_t)__cvta_generic_to_shared(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait on phase `parity`; false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (long long i = 0; i < WAIT_LIMIT; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// 4-D tiled TMA load into shared memory, completion on `bar`
__device__ __forceinline__ void tma_load_4d(void* smem_dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1,
                                            int c2, int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5, %6}], [%2];\n" ::"r"((uint32_t)__cvta_generic_to_shared(smem_dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"((uint32_t)__cvta_generic_to_shared(bar)), "r"(c0), "r"(c1),
      "r"(c2), "r"(c3)
      : "memory");
}

__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// device-side error flag (set by timed-out waits); read with gb_device_errors()
int device_error_flag(int clear);
int band_tc_error_flag(int clear);   // the tensor-core band GEMMs' flag
int conv_tc_error_flag(int clear);   // the tensor-core convolution's flag
__device__ void raise_device_error(int code);

// host: encode a 4-D tiled tensor map (dims innermost first, strides in bytes)
bool encode_tensor_map_4d(CUtensorMap* map, CUtensorMapDataType dt, void* base, const uint64_t dims[4],
                          const uint64_t strides_bytes[3], const uint32_t box[4]);

}  // namespace gb
