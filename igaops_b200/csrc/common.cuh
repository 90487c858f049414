// Shared device/host helpers of libigab200 (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdarg.h>

#include "igab200.h"
#include "fastdiv.cuh"

namespace iga {

// ---------------------------------------------------------------- errors
void set_error(const char* fmt, ...);
void clear_error();

#define IGA_CHECK_ARG(cond, ...)                                  \
  do {                                                            \
    if (!(cond)) {                                                \
      ::iga::set_error(__VA_ARGS__);                              \
      return IGA_ERR_INVALID_ARG;                                 \
    }                                                             \
  } while (0)

#define IGA_CUDA_TRY(expr)                                              \
  do {                                                                  \
    cudaError_t e__ = (expr);                                           \
    if (e__ != cudaSuccess) {                                           \
      ::iga::set_error("%s failed: %s", #expr, cudaGetErrorString(e__)); \
      return IGA_ERR_CUDA;                                              \
    }                                                                   \
  } while (0)

// Launch check: reports configuration errors of the last launch.
#define IGA_LAUNCH_CHECK()                                                  \
  do {                                                                      \
    cudaError_t e__ = cudaGetLastError();                                   \
    if (e__ != cudaSuccess) {                                               \
      ::iga::set_error("kernel launch failed (%s:%d): %s", __FILE__, __LINE__, \
                       cudaGetErrorString(e__));                            \
      return IGA_ERR_CUDA;                                                  \
    }                                                                       \
  } while (0)

inline cudaStream_t as_stream(iga_stream s) { return reinterpret_cast<cudaStream_t>(s); }

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// ---------------------------------------------------------- device misc
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Bound of every device-side spin wait (nanoseconds).
constexpr uint64_t kWaitLimitNs = 1000ull * 1000ull * 1000ull;

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait on an mbarrier phase; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait_bounded_ns(uint32_t bar, uint32_t parity,
                                                     uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_timer_ns();
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_timer_ns() - t0 > limit_ns) return false;
  }
}
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
  return mbar_wait_bounded_ns(bar, parity, kWaitLimitNs);
}

// Limit of the first waits of a launch whose wait test hook is set: the
// withheld copy never lands, so the wait runs out after this long.
constexpr uint64_t kWaitTestLimitNs = 1000ull * 1000ull;

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Named barrier among `nthreads` threads (barrier id 1; id 0 is __syncthreads).
__device__ __forceinline__ void named_sync(uint32_t id, uint32_t nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// 1D bulk async copy global -> shared (TMA engine), completion on `bar`.
// dst/src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes,
                                         uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

template <typename T>
__device__ __forceinline__ T ldg(const T* p) {
  return __ldg(p);
}

}  // namespace iga
