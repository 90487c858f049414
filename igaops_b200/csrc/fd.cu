// Fast-diagonalisation (FD) preconditioner apply.
//
// P^{-1} v = (U_d (x) ... (x) U_1) Lambda^{-1} (U_d (x) ... (x) U_1)^T v on
// the free nodes, zero on the Dirichlet nodes (SpaceFD.apply,
// src/igaops/fastdiag/utils/space_precond.py:273-320).  The free nodes of a
// direction are a contiguous index range [lo_d, lo_d + m_d) (Dirichlet only
// removes the first and/or last control point, space_precond.py:159-168), so
// the free set is a box of the control-point tensor: gather and scatter are
// index arithmetic, fused with the first and last mode products' inputs.
//
// This file holds the SIMT path (FP64 / FP32 mode products); the BF16
// tensor-core (tcgen05) mode products live in fd_tc.cu.
#include "common.cuh"

namespace iga {

struct Box {
  int32_t ndim;
  int32_t n[4];   // full extents, direction 1 first
  int32_t lo[4];  // first free index per direction
  int32_t m[4];   // free extents
};

// dst[f*ncols + k] = src[g(f)*ncols + k] (gather) or the reverse (scatter):
// f enumerates the box (direction 1 fastest), g(f) its position in the full
// tensor.
template <typename T, bool SCATTER>
__global__ void __launch_bounds__(256) box_copy_kernel(Box b, int64_t ncols, const T* __restrict__ src,
                                                       T* __restrict__ dst) {
  int64_t mfree = 1;
  for (int d = 0; d < b.ndim; ++d) mfree *= b.m[d];
  const int64_t total = mfree * ncols;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = idx % ncols;
    int64_t f = idx / ncols;
    int64_t g = 0, stride = 1;
    for (int d = 0; d < b.ndim; ++d) {
      const int64_t i = f % b.m[d];
      f /= b.m[d];
      g += (i + b.lo[d]) * stride;
      stride *= b.n[d];
    }
    if (SCATTER)
      dst[g * ncols + k] = src[idx];
    else
      dst[idx] = src[g * ncols + k];
  }
}

}  // namespace iga

using namespace iga;

extern "C" {

iga_status iga_mode_product(int dtype, const iga_factor* M, int64_t outer, int64_t inner,
                            const void* x, void* y, int accumulate, iga_stream stream);
iga_status iga_pointwise_scale(int dtype, int64_t nq, int64_t ncols, const void* coef,
                               int64_t coef_stride, const void* u, void* out, int accumulate,
                               iga_stream stream);

iga_status iga_box_copy(int dtype, int ndim, const int32_t* n, const int32_t* lo,
                        const int32_t* m, int64_t ncols, const void* src, void* dst, int scatter,
                        iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(ndim >= 1 && ndim <= 4, "ndim %d out of range", ndim);
  IGA_CHECK_ARG(n && lo && m && src && dst && ncols >= 1, "bad argument");
  IGA_CHECK_ARG(dtype == IGA_F64 || dtype == IGA_F32, "dtype %d not supported", dtype);
  Box b;
  b.ndim = ndim;
  int64_t M = 1;
  for (int d = 0; d < 4; ++d) {
    b.n[d] = d < ndim ? n[d] : 1;
    b.lo[d] = d < ndim ? lo[d] : 0;
    b.m[d] = d < ndim ? m[d] : 1;
    IGA_CHECK_ARG(b.lo[d] >= 0 && b.m[d] >= 0 && b.lo[d] + b.m[d] <= b.n[d],
                  "box of direction %d out of range", d);
    M *= b.m[d];
  }
  if (M == 0) return IGA_OK;
  int64_t blocks = ceil_div(M * ncols, 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  cudaStream_t st = as_stream(stream);
  if (dtype == IGA_F64) {
    if (scatter)
      box_copy_kernel<double, true><<<(unsigned)blocks, 256, 0, st>>>(b, ncols, (const double*)src,
                                                                      (double*)dst);
    else
      box_copy_kernel<double, false><<<(unsigned)blocks, 256, 0, st>>>(b, ncols, (const double*)src,
                                                                       (double*)dst);
  } else {
    if (scatter)
      box_copy_kernel<float, true><<<(unsigned)blocks, 256, 0, st>>>(b, ncols, (const float*)src,
                                                                     (float*)dst);
    else
      box_copy_kernel<float, false><<<(unsigned)blocks, 256, 0, st>>>(b, ncols, (const float*)src,
                                                                      (float*)dst);
  }
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

iga_status iga_fd_apply(int dtype, int ndim, const int32_t* n, const int32_t* lo, const int32_t* m,
                        const void* const* U, const void* inv_lambda, int64_t ncols, const void* x,
                        void* y, void* work0, void* work1, iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(ndim >= 1 && ndim <= 4, "ndim %d out of range", ndim);
  IGA_CHECK_ARG(n && lo && m && U && inv_lambda && x && y && work0 && work1, "null argument");
  IGA_CHECK_ARG(ncols >= 1, "ncols must be >= 1");
  IGA_CHECK_ARG(dtype == IGA_F64 || dtype == IGA_F32, "dtype %d not supported", dtype);
  Box b;
  b.ndim = ndim;
  int64_t N = 1, M = 1;
  for (int d = 0; d < 4; ++d) {
    b.n[d] = d < ndim ? n[d] : 1;
    b.lo[d] = d < ndim ? lo[d] : 0;
    b.m[d] = d < ndim ? m[d] : 1;
    IGA_CHECK_ARG(b.lo[d] >= 0 && b.m[d] >= 0 && b.lo[d] + b.m[d] <= b.n[d],
                  "free box of direction %d out of range", d);
    N *= b.n[d];
    M *= b.m[d];
  }
  cudaStream_t st = as_stream(stream);
  const size_t esz = dtype == IGA_F64 ? 8 : 4;
  IGA_CUDA_TRY(cudaMemsetAsync(y, 0, (size_t)N * ncols * esz, st));
  if (M == 0) return IGA_OK;
  int64_t blocks = ceil_div(M * ncols, 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (dtype == IGA_F64)
    box_copy_kernel<double, false><<<(unsigned)blocks, 256, 0, st>>>(b, ncols, (const double*)x,
                                                                     (double*)work0);
  else
    box_copy_kernel<float, false><<<(unsigned)blocks, 256, 0, st>>>(b, ncols, (const float*)x,
                                                                    (float*)work0);
  IGA_LAUNCH_CHECK();
  void* buf[2] = {work0, work1};
  int cur = 0;
  // tensor modes, slowest first: mode k <-> direction ndim-1-k
  for (int pass = 0; pass < 2; ++pass) {
    for (int k = 0; k < ndim; ++k) {
      const int d = ndim - 1 - k;
      iga_factor F;
      F.kind = 1;
      F.rows = F.cols = m[d];
      if (pass == 0) {  // U^T
        F.ld_row = 1;
        F.ld_col = m[d];
      } else {
        F.ld_row = m[d];
        F.ld_col = 1;
      }
      F.dense = U[d];
      int64_t outer = 1, inner = ncols;
      for (int j = ndim - 1; j > d; --j) outer *= m[j];
      for (int j = d - 1; j >= 0; --j) inner *= m[j];
      iga_status rc = iga_mode_product(dtype, &F, outer, inner, buf[cur], buf[cur ^ 1], 0, stream);
      if (rc) return rc;
      cur ^= 1;
    }
    if (pass == 0) {
      iga_status rc = iga_pointwise_scale(dtype, M, ncols, inv_lambda, 1, buf[cur], buf[cur ^ 1],
                                          0, stream);
      if (rc) return rc;
      cur ^= 1;
    }
  }
  if (dtype == IGA_F64)
    box_copy_kernel<double, true><<<(unsigned)blocks, 256, 0, st>>>(b, ncols,
                                                                    (const double*)buf[cur],
                                                                    (double*)y);
  else
    box_copy_kernel<float, true><<<(unsigned)blocks, 256, 0, st>>>(b, ncols,
                                                                   (const float*)buf[cur],
                                                                   (float*)y);
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

}  // extern "C"
