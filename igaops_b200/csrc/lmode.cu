// L-mode (n-mode) products and the generic pointwise step.
//
// These kernels back MatrixFree.apply / tensor_matrix_product
// (src/igaops/operators/utils/matrix_free.py:39-119) for arbitrary factor
// lists (banded B-spline/WQ factors or dense matrices such as the
// fast-diagonalisation eigenvectors), and the unfused matrix-free operator
// path used for quadrature rules the fused kernel does not cover.
#include <string.h>

#include "common.cuh"

namespace iga {

// ------------------------------------------------------------- errors
static thread_local char g_err[512] = {0};

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}
void clear_error() { g_err[0] = 0; }

// ------------------------------------------------- banded mode product
// y[o, r, i] (+)= sum_t vals[r*w + t] * x[o, start[r] + t, i]
template <typename T>
__global__ void __launch_bounds__(256) band_mode_kernel(int64_t outer, int32_t rows, int32_t cols,
                                                         int64_t inner, int32_t w,
                                                         const int32_t* __restrict__ start,
                                                         const T* __restrict__ vals,
                                                         const T* __restrict__ x, T* __restrict__ y,
                                                         int accumulate) {
  const int64_t total = outer * rows * inner;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = idx % inner;
    const int64_t t2 = idx / inner;
    const int32_t r = (int32_t)(t2 % rows);
    const int64_t o = t2 / rows;
    const int32_t s = __ldg(start + r);
    const T* xp = x + (o * cols) * inner + i;
    const T* vp = vals + (int64_t)r * w;
    T acc = T(0);
    for (int t = 0; t < w; ++t) {
      const int32_t c = s + t;
      if (c >= 0 && c < cols) acc += __ldg(vp + t) * __ldg(xp + (int64_t)c * inner);
    }
    T* yp = y + idx;
    *yp = accumulate ? (*yp + acc) : acc;
  }
}

// ----------------------------------------- strided batched SIMT GEMM
// C[b][m][n] (+)= sum_k A[b][m][k] B[b][k][n], arbitrary element strides.
template <typename T, int BM, int BN, int BK>
__global__ void __launch_bounds__(256) gemm_strided_kernel(
    int32_t M, int32_t N, int32_t K, const T* __restrict__ A, int64_t sam, int64_t sak, int64_t sab,
    const T* __restrict__ B, int64_t sbk, int64_t sbn, int64_t sbb, T* __restrict__ C, int64_t scm,
    int64_t scn, int64_t scb, int accumulate) {
  static_assert(BM == 64 && BN == 64, "thread layout assumes a 64x64 tile");
  __shared__ T As[BK][BM + 1];
  __shared__ T Bs[BK][BN + 1];
  const int tid = threadIdx.x;
  const int tm = tid / 16;  // 0..15 -> rows tm*4 .. +3
  const int tn = tid % 16;  // 0..15 -> cols tn*4 .. +3
  const int64_t b = blockIdx.z;
  const int32_t m0 = blockIdx.y * BM;
  const int32_t n0 = blockIdx.x * BN;
  A += b * sab;
  B += b * sbb;
  C += b * scb;
  T acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = T(0);

  for (int32_t k0 = 0; k0 < K; k0 += BK) {
    // load A tile (BM x BK) and B tile (BK x BN)
    for (int e = tid; e < BM * BK; e += 256) {
      const int mm = e % BM, kk = e / BM;
      const int32_t gm = m0 + mm, gk = k0 + kk;
      As[kk][mm] = (gm < M && gk < K) ? A[gm * sam + gk * sak] : T(0);
    }
    for (int e = tid; e < BK * BN; e += 256) {
      const int nn = e % BN, kk = e / BN;
      const int32_t gn = n0 + nn, gk = k0 + kk;
      Bs[kk][nn] = (gn < N && gk < K) ? B[gk * sbk + gn * sbn] : T(0);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      T a[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][tm * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Bs[kk][tn * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] += a[i] * bv[j];
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int32_t gm = m0 + tm * 4 + i;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int32_t gn = n0 + tn * 4 + j;
      if (gn >= N) continue;
      T* cp = C + gm * scm + gn * scn;
      *cp = accumulate ? (*cp + acc[i][j]) : acc[i][j];
    }
  }
}

template <typename T>
static iga_status launch_gemm(int32_t M, int32_t N, int32_t K, int64_t batch, const T* A,
                              int64_t sam, int64_t sak, int64_t sab, const T* B, int64_t sbk,
                              int64_t sbn, int64_t sbb, T* C, int64_t scm, int64_t scn,
                              int64_t scb, int accumulate, cudaStream_t st) {
  if (M == 0 || N == 0 || batch == 0) return IGA_OK;
  IGA_CHECK_ARG(batch <= 65535, "gemm batch %lld exceeds 65535", (long long)batch);
  dim3 grid((unsigned)ceil_div(N, 64), (unsigned)ceil_div(M, 64), (unsigned)batch);
  IGA_CHECK_ARG(grid.y <= 65535, "gemm M=%d too large", M);
  gemm_strided_kernel<T, 64, 64, 16><<<grid, 256, 0, st>>>(M, N, K, A, sam, sak, sab, B, sbk, sbn,
                                                           sbb, C, scm, scn, scb, accumulate);
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

template <typename T>
static iga_status mode_product_t(const iga_factor* M, int64_t outer, int64_t inner, const T* x,
                                 T* y, int accumulate, cudaStream_t st) {
  const int32_t rows = M->rows, cols = M->cols;
  if (outer == 0 || inner == 0 || rows == 0) return IGA_OK;
  if (M->kind == 0) {
    const iga_band& b = M->band;
    IGA_CHECK_ARG(b.rows == rows && b.cols == cols, "band shape mismatch");
    IGA_CHECK_ARG(b.start && b.vals && b.width > 0, "band has null arrays");
    const int64_t total = outer * rows * inner;
    int64_t blocks = ceil_div(total, 256);
    if (blocks > 148 * 64) blocks = 148 * 64;
    band_mode_kernel<T><<<(unsigned)blocks, 256, 0, st>>>(outer, rows, cols, inner, b.width,
                                                          b.start, (const T*)b.vals, x, y,
                                                          accumulate);
    IGA_LAUNCH_CHECK();
    return IGA_OK;
  }
  IGA_CHECK_ARG(M->kind == 1 && M->dense, "dense factor has null data");
  const T* D = (const T*)M->dense;
  if (inner >= 16) {
    // per o: C(rows x inner) = M(rows x cols) X_o(cols x inner)
    IGA_CHECK_ARG(outer <= 65535, "outer %lld too large", (long long)outer);
    return launch_gemm<T>(rows, (int32_t)inner, cols, outer, D, M->ld_row, M->ld_col, 0, x, inner,
                          1, (int64_t)cols * inner, y, inner, 1, (int64_t)rows * inner,
                          accumulate, st);
  }
  // per i: C(outer x rows) = X_i(outer x cols) M^T
  IGA_CHECK_ARG(outer <= 0x7fffffff, "outer too large");
  return launch_gemm<T>((int32_t)outer, rows, cols, inner, x, (int64_t)cols * inner, inner, 1, D,
                        M->ld_col, M->ld_row, 0, y, (int64_t)rows * inner, inner, 1, accumulate,
                        st);
}

// ------------------------------------------------------- pointwise scale
template <typename T>
__global__ void __launch_bounds__(256) pointwise_scale_kernel(int64_t nq, int64_t ncols,
                                                               const T* __restrict__ coef,
                                                               int64_t cs, const T* __restrict__ u,
                                                               T* __restrict__ out, int accumulate) {
  const int64_t total = nq * ncols;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t q = idx / ncols;
    const T v = __ldg(coef + q * cs) * __ldg(u + idx);
    out[idx] = accumulate ? out[idx] + v : v;
  }
}

// y = alpha*x + beta*y (beta == 0 ignores the old y, so NaN garbage in y is
// not propagated)
template <typename T>
__global__ void __launch_bounds__(256) axpby_kernel(int64_t n, T alpha, const T* __restrict__ x,
                                                     T beta, T* __restrict__ y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const T v = alpha * x[i];
    y[i] = (beta == T(0)) ? v : v + beta * y[i];
  }
}

}  // namespace iga

using namespace iga;

extern "C" {

int iga_abi_version(void) { return 1; }

const char* iga_last_error(void) { return g_err; }

iga_status iga_mode_product(int dtype, const iga_factor* M, int64_t outer, int64_t inner,
                            const void* x, void* y, int accumulate, iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(M && x && y, "null argument");
  IGA_CHECK_ARG(outer >= 0 && inner >= 0, "negative size");
  cudaStream_t st = as_stream(stream);
  if (dtype == IGA_F64)
    return mode_product_t<double>(M, outer, inner, (const double*)x, (double*)y, accumulate, st);
  if (dtype == IGA_F32)
    return mode_product_t<float>(M, outer, inner, (const float*)x, (float*)y, accumulate, st);
  set_error("dtype %d not supported by iga_mode_product", dtype);
  return IGA_ERR_UNSUPPORTED;
}

iga_status iga_lmode_apply(int dtype, int ndim, const iga_factor* factors, int64_t ncols,
                           const void* x, void* y, void* work0, void* work1, iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(ndim >= 1 && ndim <= 8, "ndim %d out of range", ndim);
  IGA_CHECK_ARG(factors && x && y && ncols >= 1, "null argument");
  IGA_CHECK_ARG(dtype == IGA_F64 || dtype == IGA_F32, "dtype %d not supported", dtype);
  IGA_CHECK_ARG(ndim == 1 || (work0 && work1), "work buffers required for ndim > 1");
  // tensor dims, slowest first: dims[0] = direction ndim, ..., dims[ndim-1] = direction 1
  int64_t dims[8];
  for (int k = 0; k < ndim; ++k) dims[k] = factors[ndim - 1 - k].cols;
  const void* src = x;
  void* bufs[2] = {work0, work1};
  int which = 0;
  // same order as the reference: the slowest direction first
  for (int m = 0; m < ndim; ++m) {
    const iga_factor* F = &factors[ndim - 1 - m];
    IGA_CHECK_ARG(F->cols == dims[m], "factor %d has %d columns, tensor mode has %lld",
                  ndim - 1 - m, F->cols, (long long)dims[m]);
    int64_t outer = 1, inner = ncols;
    for (int k = 0; k < m; ++k) outer *= dims[k];
    for (int k = m + 1; k < ndim; ++k) inner *= dims[k];
    void* dst = (m == ndim - 1) ? y : bufs[which];
    iga_status rc = iga_mode_product(dtype, F, outer, inner, src, dst, 0, stream);
    if (rc != IGA_OK) return rc;
    dims[m] = F->rows;
    src = dst;
    which ^= 1;
  }
  return IGA_OK;
}

iga_status iga_pointwise_scale(int dtype, int64_t nq, int64_t ncols, const void* coef,
                               int64_t coef_stride, const void* u, void* out, int accumulate,
                               iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(coef && u && out && nq >= 0 && ncols >= 1, "bad argument");
  const int64_t total = nq * ncols;
  if (total == 0) return IGA_OK;
  int64_t blocks = ceil_div(total, 256);
  if (blocks > 148 * 32) blocks = 148 * 32;
  cudaStream_t st = as_stream(stream);
  if (dtype == IGA_F64)
    pointwise_scale_kernel<double><<<(unsigned)blocks, 256, 0, st>>>(
        nq, ncols, (const double*)coef, coef_stride, (const double*)u, (double*)out, accumulate);
  else if (dtype == IGA_F32)
    pointwise_scale_kernel<float><<<(unsigned)blocks, 256, 0, st>>>(
        nq, ncols, (const float*)coef, coef_stride, (const float*)u, (float*)out, accumulate);
  else {
    set_error("dtype %d not supported", dtype);
    return IGA_ERR_UNSUPPORTED;
  }
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

iga_status iga_axpby(int dtype, int64_t n, double alpha, const void* x, double beta, void* y,
                     iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(x && y && n >= 0, "bad argument");
  if (n == 0) return IGA_OK;
  int64_t blocks = ceil_div(n, 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  cudaStream_t st = as_stream(stream);
  if (dtype == IGA_F64)
    axpby_kernel<double><<<(unsigned)blocks, 256, 0, st>>>(n, alpha, (const double*)x, beta,
                                                           (double*)y);
  else if (dtype == IGA_F32)
    axpby_kernel<float><<<(unsigned)blocks, 256, 0, st>>>(n, (float)alpha, (const float*)x,
                                                          (float)beta, (float*)y);
  else {
    set_error("dtype %d not supported", dtype);
    return IGA_ERR_UNSUPPORTED;
  }
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

}  // extern "C"
