// Division by a CTA-invariant divisor as one multiply-high (host and device).
// Plain header (no CUDA runtime includes) so that host tests can compile it.
#pragma once

#include <stdint.h>

#ifndef __CUDACC__
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
#ifndef __forceinline__
#define __forceinline__ inline
#endif
#endif

namespace iga {

// Quotient of a non-negative index by a divisor that is fixed for the whole
// CTA, as one multiply-high: floor(e / d) = umulhi(e, m) with
// m = floor(2^32 / d) + 1, exact whenever e * d < 2^32 (division by an
// invariant integer through a rounded-up reciprocal, Granlund & Montgomery,
// PLDI 1994). The kernels use it for tile-local indices (e, d < 2^16).
struct FastDiv {
  uint32_t d, m;
  __host__ __device__ __forceinline__ explicit FastDiv(int dv) : d((uint32_t)dv), m(0u) {
    if (d > 1u) {
      // floor(2^32 / d) from 32-bit arithmetic: (2^32 - 1) / d, plus one
      // when d divides 2^32 (a power of two)
      m = 0xFFFFFFFFu / d + ((d & (d - 1u)) == 0u ? 1u : 0u) + 1u;
    }
  }
  __host__ __device__ __forceinline__ int div(int e) const {
#ifdef __CUDA_ARCH__
    return d <= 1u ? e : (int)__umulhi((uint32_t)e, m);
#else
    return d <= 1u ? e : (int)(((uint64_t)(uint32_t)e * m) >> 32);
#endif
  }
};

}  // namespace iga
