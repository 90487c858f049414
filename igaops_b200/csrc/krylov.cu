// Device primitives of the Krylov solvers (Arnoldi / CGS2, GCRO-DR).
//
// The reference keeps its Krylov bases as (m, n) numpy arrays and combines
// them with dot products and matrix products (src/igaops/solvers/
// linear_solver.py:438-525, src/igaops/solvers/deflated/gcrodr.py:257-363,
// helpers.py:13-146).  Here the bases stay on the device as rows of length n
// and two kernels cover every large operation:
//   gram    : G = A^H B for m1 rows of A and m2 rows of B (dot products,
//             Gram-Schmidt projections, W^H V overlaps), FP64 accumulation,
//             two-stage reduction in a fixed order (deterministic);
//   combine : out_k = beta*out_k + alpha * sum_j c_{jk} A_j (Gram-Schmidt
//             update, x = Z y, basis rotations C = W Q).
// Element types: FP64 or FP32 real, or FP64 complex (interleaved re/im).
#include <mutex>

#include "common.cuh"

namespace iga {

constexpr int kGramThreads = 256;
constexpr int kGramMaxPairs = 16;  // accumulators per thread

template <typename T>
struct Elem;
template <>
struct Elem<double> {
  static constexpr int W = 1;
};
template <>
struct Elem<float> {
  static constexpr int W = 1;
};

// CPLX: values are (re, im) pairs of T = double
template <typename T, bool CPLX>
__global__ void __launch_bounds__(kGramThreads) gram_stage1(int64_t n, int m1, const T* __restrict__ A,
                                                            int64_t lda, int m2,
                                                            const T* __restrict__ B, int64_t ldb,
                                                            int ti, double* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int C = CPLX ? 2 : 1;
  T* As = reinterpret_cast<T*>(smem_raw);  // [m1][ti*C]
  T* Bs = As + (size_t)m1 * ti * C;        // [m2][ti*C]
  const int npairs = m1 * m2;
  const int64_t nblk = gridDim.x;
  const int64_t chunk = (n + nblk - 1) / nblk;
  const int64_t i0 = blockIdx.x * chunk;
  const int64_t i1 = min(n, i0 + chunk);
  double acc_re[kGramMaxPairs], acc_im[kGramMaxPairs];
#pragma unroll
  for (int p = 0; p < kGramMaxPairs; ++p) acc_re[p] = acc_im[p] = 0.0;
  for (int64_t base = i0; base < i1; base += ti) {
    const int len = (int)((i1 - base) < (int64_t)ti ? (i1 - base) : (int64_t)ti);
    for (int e = threadIdx.x; e < m1 * len * C; e += blockDim.x) {
      const int j = e / (len * C), t = e - j * (len * C);
      As[j * ti * C + t] = A[j * lda * C + base * C + t];
    }
    for (int e = threadIdx.x; e < m2 * len * C; e += blockDim.x) {
      const int j = e / (len * C), t = e - j * (len * C);
      Bs[j * ti * C + t] = B[j * ldb * C + base * C + t];
    }
    __syncthreads();
#pragma unroll
    for (int p = 0; p < kGramMaxPairs; ++p) {
      const int pair = threadIdx.x + p * blockDim.x;
      if (pair >= npairs) break;
      const int j1 = pair / m2, j2 = pair - j1 * m2;
      const T* a = As + j1 * ti * C;
      const T* b = Bs + j2 * ti * C;
      double sr = 0.0, si = 0.0;
      for (int t = 0; t < len; ++t) {
        if (CPLX) {
          const double ar = a[2 * t], ai = a[2 * t + 1], br = b[2 * t], bi = b[2 * t + 1];
          sr += ar * br + ai * bi;  // conj(a) * b
          si += ar * bi - ai * br;
        } else {
          sr += (double)a[t] * (double)b[t];
        }
      }
      acc_re[p] += sr;
      acc_im[p] += si;
    }
    __syncthreads();
  }
#pragma unroll
  for (int p = 0; p < kGramMaxPairs; ++p) {
    const int pair = threadIdx.x + p * blockDim.x;
    if (pair >= npairs) break;
    double* dst = partial + ((int64_t)blockIdx.x * npairs + pair) * C;
    dst[0] = acc_re[p];
    if (CPLX) dst[1] = acc_im[p];
  }
}

template <bool CPLX>
__global__ void gram_stage2(int npairs, int nblk, const double* __restrict__ partial,
                            double* __restrict__ out) {
  constexpr int C = CPLX ? 2 : 1;
  const int pair = blockIdx.x * blockDim.x + threadIdx.x;
  if (pair >= npairs) return;
  double sr = 0.0, si = 0.0;
  for (int b = 0; b < nblk; ++b) {
    sr += partial[((int64_t)b * npairs + pair) * C];
    if (CPLX) si += partial[((int64_t)b * npairs + pair) * C + 1];
  }
  out[pair * C] = sr;
  if (CPLX) out[pair * C + 1] = si;
}

// One row set against one vector (real): partial[b*m + j] = sum over block
// b's index range of A_j[i] * x[i], streamed straight from global memory
// (the CGS projections and norms of Arnoldi, m <= kGramRowsMax).  MB (4, 8,
// 16 or 32) >= m bounds the unrolled accumulator set.
constexpr int kGramRowsMax = 32;

template <typename T, int MB>
__global__ void __launch_bounds__(kGramThreads)
    gram_rows_stage1(int64_t n, int m, const T* __restrict__ A, int64_t lda,
                     const T* __restrict__ x, double* __restrict__ partial) {
  const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const int64_t i0 = (int64_t)blockIdx.x * chunk;
  const int64_t i1 = min(n, i0 + chunk);
  double acc[MB];
#pragma unroll
  for (int j = 0; j < MB; ++j) acc[j] = 0.0;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += kGramThreads) {
    const double xv = (double)x[i];
#pragma unroll
    for (int j = 0; j < MB; ++j)
      if (j < m) acc[j] += (double)A[j * lda + i] * xv;
  }
  __shared__ double red[kGramThreads / 32][MB];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < MB; ++j) {
    if (j >= m) break;
    double v = acc[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp][j] = v;
  }
  __syncthreads();
  if (threadIdx.x < m) {
    double v = 0.0;
#pragma unroll
    for (int w = 0; w < kGramThreads / 32; ++w) v += red[w][threadIdx.x];
    partial[(int64_t)blockIdx.x * m + threadIdx.x] = v;
  }
}

// Second stage for nv <= kGramThreads values per block, one CTA:
// out[v] = sum over blocks of partial[b*nv + v].  G = the largest power of
// two <= kGramThreads / nv row groups; group g sums blocks g, g+G, ..., then
// a halving tree over the groups (addition order fixed by nv and nblk).
__global__ void __launch_bounds__(kGramThreads)
    gram_stage2_tree(int nv, int nblk, const double* __restrict__ partial,
                     double* __restrict__ out) {
  __shared__ double red[kGramThreads];
  int G = 1;
  while (2 * G * nv <= kGramThreads) G *= 2;
  const int t = threadIdx.x, g = t / nv, v = t - g * nv;
  double s = 0.0;
  if (g < G)
    for (int b = g; b < nblk; b += G) s += partial[(int64_t)b * nv + v];
  red[t] = s;
  __syncthreads();
  for (int h = G / 2; h > 0; h >>= 1) {
    if (g < h) red[t] += red[t + h * nv];
    __syncthreads();
  }
  if (t < nv) out[t] = red[t];
}

// out_k[i] = beta*out_k[i] + alpha * sum_j coef[j*kout + k] * A_j[i]
template <typename T, bool CPLX>
__global__ void __launch_bounds__(256) combine_kernel(int64_t n, int m_in, const T* __restrict__ A,
                                                      int64_t lda, int kout,
                                                      const double* __restrict__ coef,
                                                      double alpha, double beta, T* __restrict__ out,
                                                      int64_t ldo) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int C = CPLX ? 2 : 1;
  double* cs = reinterpret_cast<double*>(smem_raw);  // [m_in*kout*C]
  for (int e = threadIdx.x; e < m_in * kout * C; e += blockDim.x) cs[e] = coef[e];
  __syncthreads();
  constexpr int KB = 8;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    for (int k0 = 0; k0 < kout; k0 += KB) {
      double ar[KB], ai[KB];
#pragma unroll
      for (int kk = 0; kk < KB; ++kk) ar[kk] = ai[kk] = 0.0;
      for (int j = 0; j < m_in; ++j) {
        double vr, vi = 0.0;
        if (CPLX) {
          vr = A[(j * lda + i) * 2];
          vi = A[(j * lda + i) * 2 + 1];
        } else {
          vr = (double)A[j * lda + i];
        }
#pragma unroll
        for (int kk = 0; kk < KB; ++kk) {
          const int k = k0 + kk;
          if (k < kout) {
            const double cr = cs[(j * kout + k) * C];
            if (CPLX) {
              const double ci = cs[(j * kout + k) * C + 1];
              ar[kk] += cr * vr - ci * vi;
              ai[kk] += cr * vi + ci * vr;
            } else {
              ar[kk] += cr * vr;
            }
          }
        }
      }
#pragma unroll
      for (int kk = 0; kk < KB; ++kk) {
        const int k = k0 + kk;
        if (k >= kout) break;
        if (CPLX) {
          double* o = reinterpret_cast<double*>(out) + (k * ldo + i) * 2;
          const double orr = beta == 0.0 ? 0.0 : beta * o[0];
          const double oi = beta == 0.0 ? 0.0 : beta * o[1];
          o[0] = orr + alpha * ar[kk];
          o[1] = oi + alpha * ai[kk];
        } else {
          T* o = out + k * ldo + i;
          const double old = beta == 0.0 ? 0.0 : beta * (double)(*o);
          *o = (T)(old + alpha * ar[kk]);
        }
      }
    }
  }
}

// x[i] *= s (or /= s) with s read from device memory
template <typename T>
__global__ void scale_dev_kernel(int64_t n, T* __restrict__ x, const double* __restrict__ s,
                                 int invert, int cplx) {
  double f;
  if (invert == 2) {  // x /= sqrt(s): normalise by a squared norm; zero norm -> 0
    const double r = sqrt(fmax(s[0], 0.0));
    f = r > 0.0 ? 1.0 / r : 0.0;
  } else {
    f = invert ? 1.0 / s[0] : s[0];
  }
  const int64_t m = cplx ? 2 * n : n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] = (T)((double)x[i] * f);
}

template <typename T>
__global__ void mask_kernel(int64_t nidx, const int64_t* __restrict__ idx, T* __restrict__ x) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nidx;
       i += (int64_t)gridDim.x * blockDim.x)
    x[idx[i]] = T(0);
}

template <typename T>
__global__ void cast_kernel(int64_t n, const T* __restrict__ src, double* __restrict__ dst_d,
                            float* __restrict__ dst_f) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (dst_d) dst_d[i] = (double)src[i];
    if (dst_f) dst_f[i] = (float)src[i];
  }
}

// complex <-> (re, im) planes
__global__ void cplx_split_kernel(int64_t n, const double* __restrict__ z, double* __restrict__ re,
                                  double* __restrict__ im) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    re[i] = z[2 * i];
    im[i] = z[2 * i + 1];
  }
}
__global__ void cplx_merge_kernel(int64_t n, const double* __restrict__ re,
                                  const double* __restrict__ im, double* __restrict__ z) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    z[2 * i] = re[i];
    z[2 * i + 1] = im[i];
  }
}

static unsigned grid_for(int64_t n, int64_t cap = 148 * 8) {
  int64_t b = ceil_div(n, 256);
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (unsigned)b;
}

}  // namespace iga

using namespace iga;

extern "C" {

iga_status iga_gram_workspace(int64_t n, int m1, int m2, int cplx, int* nblk, int64_t* elems) {
  clear_error();
  IGA_CHECK_ARG(nblk && elems && m1 >= 1 && m2 >= 1 && n >= 0, "bad argument");
  IGA_CHECK_ARG((int64_t)m1 * m2 <= (int64_t)kGramThreads * kGramMaxPairs,
                "m1*m2 = %lld exceeds %d", (long long)m1 * m2, kGramThreads * kGramMaxPairs);
  int64_t b = ceil_div(n, 2048);
  if (b < 1) b = 1;
  if (b > 148 * 2) b = 148 * 2;
  *nblk = (int)b;
  *elems = b * (int64_t)m1 * m2 * (cplx ? 2 : 1);
  return IGA_OK;
}

iga_status iga_gram(int dtype, int cplx, int64_t n, int m1, const void* A, int64_t lda, int m2,
                    const void* B, int64_t ldb, double* out, double* partial, int nblk,
                    iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(A && B && out && partial && nblk >= 1 && m1 >= 1 && m2 >= 1, "bad argument");
  IGA_CHECK_ARG((int64_t)m1 * m2 <= (int64_t)kGramThreads * kGramMaxPairs,
                "m1*m2 = %lld exceeds %d", (long long)m1 * m2, kGramThreads * kGramMaxPairs);
  IGA_CHECK_ARG(!cplx || dtype == IGA_F64, "complex gram needs FP64");
  cudaStream_t st = as_stream(stream);
  const int C = cplx ? 2 : 1;
  const int npairs = m1 * m2;
  if (dtype != IGA_F64 && dtype != IGA_F32) {
    set_error("dtype %d not supported", dtype);
    return IGA_ERR_UNSUPPORTED;
  }
  if (!cplx && (m2 == 1 || m1 == 1) && npairs <= kGramRowsMax) {
    // real A^T x (or a^T B): out[j] is the dot product of row j of the
    // row set with the single vector; pair index j1*m2 + j2 = j either way
    const void* R = m2 == 1 ? A : B;
    const void* v = m2 == 1 ? B : A;
    const int64_t ldr = m2 == 1 ? lda : ldb;
    const int m = npairs;
#define IGA_GRAM_ROWS(MB)                                                             \
  do {                                                                                \
    if (dtype == IGA_F64)                                                             \
      gram_rows_stage1<double, MB><<<nblk, kGramThreads, 0, st>>>(                    \
          n, m, (const double*)R, ldr, (const double*)v, partial);                    \
    else                                                                              \
      gram_rows_stage1<float, MB><<<nblk, kGramThreads, 0, st>>>(                     \
          n, m, (const float*)R, ldr, (const float*)v, partial);                      \
  } while (0)
    if (m <= 4)
      IGA_GRAM_ROWS(4);
    else if (m <= 8)
      IGA_GRAM_ROWS(8);
    else if (m <= 16)
      IGA_GRAM_ROWS(16);
    else
      IGA_GRAM_ROWS(32);
#undef IGA_GRAM_ROWS
    IGA_LAUNCH_CHECK();
    gram_stage2_tree<<<1, kGramThreads, 0, st>>>(m, nblk, partial, out);
    IGA_LAUNCH_CHECK();
    return IGA_OK;
  }
  const size_t esz = dtype == IGA_F64 ? 8 : 4;
  int ti = (int)(40 * 1024 / ((size_t)(m1 + m2) * C * esz));
  if (ti > 64) ti = 64;
  if (ti < 1) ti = 1;
  const size_t smem = (size_t)(m1 + m2) * ti * C * esz;
  if (smem > 48 * 1024) {
    // wide row sets (m1 + m2 above 2560 real / 1280 complex FP64 rows) need
    // more than the default dynamic shared-memory window even at one row
    // per tile
    if (dtype == IGA_F64 && cplx)
      IGA_CUDA_TRY(cudaFuncSetAttribute(gram_stage1<double, true>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    else if (dtype == IGA_F64)
      IGA_CUDA_TRY(cudaFuncSetAttribute(gram_stage1<double, false>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    else
      IGA_CUDA_TRY(cudaFuncSetAttribute(gram_stage1<float, false>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  }
  if (dtype == IGA_F64) {
    if (cplx)
      gram_stage1<double, true><<<nblk, kGramThreads, smem, st>>>(n, m1, (const double*)A, lda, m2,
                                                                 (const double*)B, ldb, ti,
                                                                 partial);
    else
      gram_stage1<double, false><<<nblk, kGramThreads, smem, st>>>(
          n, m1, (const double*)A, lda, m2, (const double*)B, ldb, ti, partial);
  } else {
    gram_stage1<float, false><<<nblk, kGramThreads, smem, st>>>(n, m1, (const float*)A, lda, m2,
                                                               (const float*)B, ldb, ti, partial);
  }
  IGA_LAUNCH_CHECK();
  if (npairs * C <= kGramThreads)
    gram_stage2_tree<<<1, kGramThreads, 0, st>>>(npairs * C, nblk, partial, out);
  else if (cplx)
    gram_stage2<true><<<(unsigned)ceil_div(npairs, 128), 128, 0, st>>>(npairs, nblk, partial, out);
  else
    gram_stage2<false><<<(unsigned)ceil_div(npairs, 128), 128, 0, st>>>(npairs, nblk, partial, out);
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

// ---------------------------------------------------------------------
// iga_gram_noalloc: iga_gram for callers that cannot allocate device memory.
//
// The partial sums of the two-stage reduction live in this file-scope device
// array instead of caller scratch.  Every GPU that loads the library holds it
// (kNoAllocPartials doubles = 512 KiB) until the process exits.  Host code
// cannot pass `g_gram_partials` itself to a kernel (in host code that name is
// a host-side stand-in, not a device address), so the device address is
// looked up with cudaGetSymbolAddress, with the device current, on the first
// call made on it.  The address belongs to the device's current context: the
// cache keeps the context it was looked up in (cuCtxGetCurrent, reached
// through the runtime's driver entry point, so the library does not link
// libcuda) and looks the address up again when a call finds another context
// current (after a cudaDeviceReset, say).
constexpr int64_t kNoAllocPartials = 1 << 16;
static __device__ __align__(256) double g_gram_partials[kNoAllocPartials];

static double* noalloc_partials_for_current_device(iga_status* rc) {
  constexpr int kMaxDevices = 64;
  static double* addr[kMaxDevices] = {nullptr};
  static void* addr_ctx[kMaxDevices] = {nullptr};
  static std::mutex mu;
  using ctx_get_fn = int (*)(void**);
  static ctx_get_fn ctx_get = nullptr;
  static bool ctx_get_tried = false;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    set_error("iga_gram_noalloc: no usable current device (%s)", cudaGetErrorString(e));
    *rc = IGA_ERR_CUDA;
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (!ctx_get_tried) {
    ctx_get_tried = true;
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      ctx_get = reinterpret_cast<ctx_get_fn>(fn);
  }
  // the context current on this thread (null when the runtime has not bound
  // one yet: the symbol lookup below binds the device's primary context)
  void* ctx = nullptr;
  if (ctx_get && ctx_get(&ctx) != 0) ctx = nullptr;
  if (!addr[dev] || !ctx || ctx != addr_ctx[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_gram_partials);
    if (e != cudaSuccess || !p) {
      set_error("iga_gram_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
      *rc = IGA_ERR_CUDA;
      return nullptr;
    }
    addr[dev] = static_cast<double*>(p);
    ctx = nullptr;
    if (ctx_get && ctx_get(&ctx) != 0) ctx = nullptr;
    addr_ctx[dev] = ctx;
  }
  *rc = IGA_OK;
  return addr[dev];
}

iga_status iga_combine(int dtype, int cplx, int64_t n, int m_in, const void* A, int64_t lda,
                       int kout, const double* coef, double alpha, double beta, void* out,
                       int64_t ldo, iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(A && coef && out && m_in >= 0 && kout >= 1, "bad argument");
  IGA_CHECK_ARG(!cplx || dtype == IGA_F64, "complex combine needs FP64");
  const int C = cplx ? 2 : 1;
  const size_t smem = (size_t)m_in * kout * C * sizeof(double);
  IGA_CHECK_ARG(smem <= 96 * 1024, "coefficient block %d x %d too large", m_in, kout);
  cudaStream_t st = as_stream(stream);
  if (n == 0) return IGA_OK;
  const unsigned g = grid_for(n);
  if (smem > 48 * 1024) {
    if (dtype == IGA_F64 && cplx)
      IGA_CUDA_TRY(cudaFuncSetAttribute(combine_kernel<double, true>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    else if (dtype == IGA_F64)
      IGA_CUDA_TRY(cudaFuncSetAttribute(combine_kernel<double, false>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    else
      IGA_CUDA_TRY(cudaFuncSetAttribute(combine_kernel<float, false>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  }
  if (dtype == IGA_F64) {
    if (cplx)
      combine_kernel<double, true><<<g, 256, smem, st>>>(n, m_in, (const double*)A, lda, kout,
                                                        coef, alpha, beta, (double*)out, ldo);
    else
      combine_kernel<double, false><<<g, 256, smem, st>>>(n, m_in, (const double*)A, lda, kout,
                                                         coef, alpha, beta, (double*)out, ldo);
  } else if (dtype == IGA_F32) {
    combine_kernel<float, false><<<g, 256, smem, st>>>(n, m_in, (const float*)A, lda, kout, coef,
                                                       alpha, beta, (float*)out, ldo);
  } else {
    set_error("dtype %d not supported", dtype);
    return IGA_ERR_UNSUPPORTED;
  }
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

iga_status iga_gram_noalloc(int dtype, int cplx, int64_t n, int m1, const void* A, int64_t lda,
                            int m2, const void* B, int64_t ldb, double* out, iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(A && B && out && n >= 0 && m1 >= 1 && m2 >= 1, "bad argument");
  const int64_t C = cplx ? 2 : 1;
  const int64_t per_block = (int64_t)m1 * m2 * C;
  IGA_CHECK_ARG((int64_t)m1 * m2 <= (int64_t)kGramThreads * kGramMaxPairs,
                "iga_gram_noalloc: m1*m2 = %lld pairs exceeds the %d pairs of one call",
                (long long)m1 * m2, kGramThreads * kGramMaxPairs);
  IGA_CHECK_ARG(per_block <= kNoAllocPartials,
                "iga_gram_noalloc: %d x %d %s products need %lld partials per block; the "
                "built-in scratch holds %lld (use iga_gram with caller scratch)",
                m1, m2, cplx ? "complex" : "real", (long long)per_block,
                (long long)kNoAllocPartials);
  int nblk = 0;
  int64_t elems = 0;
  iga_status rc = iga_gram_workspace(n, m1, m2, cplx, &nblk, &elems);
  if (rc) return rc;
  if ((int64_t)nblk * per_block > kNoAllocPartials) nblk = (int)(kNoAllocPartials / per_block);
  double* partial = noalloc_partials_for_current_device(&rc);
  if (rc) return rc;
  // stage 1 writes every partial that stage 2 reads: nothing to clear
  return iga_gram(dtype, cplx, n, m1, A, lda, m2, B, ldb, out, partial, nblk, stream);
}

iga_status iga_scale_dev(int dtype, int cplx, int64_t n, void* x, const double* s, int invert,
                         iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(x && s && n >= 0, "bad argument");
  if (n == 0) return IGA_OK;
  cudaStream_t st = as_stream(stream);
  const unsigned g = grid_for(cplx ? 2 * n : n);
  if (dtype == IGA_F64)
    scale_dev_kernel<double><<<g, 256, 0, st>>>(n, (double*)x, s, invert, cplx);
  else if (dtype == IGA_F32 && !cplx)
    scale_dev_kernel<float><<<g, 256, 0, st>>>(n, (float*)x, s, invert, 0);
  else {
    set_error("dtype %d not supported", dtype);
    return IGA_ERR_UNSUPPORTED;
  }
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

iga_status iga_mask_zero(int dtype, int64_t nidx, const int64_t* idx, void* x,
                         iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(nidx >= 0 && (nidx == 0 || (idx && x)), "bad argument");
  if (nidx == 0) return IGA_OK;
  cudaStream_t st = as_stream(stream);
  const unsigned g = grid_for(nidx);
  if (dtype == IGA_F64)
    mask_kernel<double><<<g, 256, 0, st>>>(nidx, idx, (double*)x);
  else if (dtype == IGA_F32)
    mask_kernel<float><<<g, 256, 0, st>>>(nidx, idx, (float*)x);
  else {
    set_error("dtype %d not supported", dtype);
    return IGA_ERR_UNSUPPORTED;
  }
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

iga_status iga_convert(int dtype_in, int dtype_out, int64_t n, const void* src, void* dst,
                       iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(src && dst && n >= 0, "bad argument");
  if (n == 0) return IGA_OK;
  cudaStream_t st = as_stream(stream);
  const unsigned g = grid_for(n);
  double* dd = dtype_out == IGA_F64 ? (double*)dst : nullptr;
  float* df = dtype_out == IGA_F32 ? (float*)dst : nullptr;
  IGA_CHECK_ARG(dd || df, "dtype_out %d not supported", dtype_out);
  if (dtype_in == IGA_F64)
    cast_kernel<double><<<g, 256, 0, st>>>(n, (const double*)src, dd, df);
  else if (dtype_in == IGA_F32)
    cast_kernel<float><<<g, 256, 0, st>>>(n, (const float*)src, dd, df);
  else {
    set_error("dtype_in %d not supported", dtype_in);
    return IGA_ERR_UNSUPPORTED;
  }
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

iga_status iga_complex_split(int64_t n, const double* z, double* re, double* im,
                             iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(z && re && im && n >= 0, "bad argument");
  if (n == 0) return IGA_OK;
  cplx_split_kernel<<<grid_for(n), 256, 0, as_stream(stream)>>>(n, z, re, im);
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

iga_status iga_complex_merge(int64_t n, const double* re, const double* im, double* z,
                             iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(z && re && im && n >= 0, "bad argument");
  if (n == 0) return IGA_OK;
  cplx_merge_kernel<<<grid_for(n), 256, 0, as_stream(stream)>>>(n, re, im, z);
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

}  // extern "C"
