// Segmented Krylov primitives for many independent patches solved together.
//
// The vectors of all patches are concatenated into one flat array; patch p
// owns elements [offs[p], offs[p+1]).  Work is split into blocks of at most
// kSegChunk elements that never straddle two patches: patch p owns blocks
// [blk0[p], blk0[p+1]).  Every reduction is two-stage with a fixed order
// (per-block partials, then a per-patch sum over its blocks), so results do
// not depend on scheduling.
//
// These are the per-patch forms of the GMRES vector work of the reference
// (src/igaops/solvers/linear_solver.py:438-525: the two Gram-Schmidt passes,
// the norms and x = Z y) plus the Givens-rotation form of its Hessenberg
// least squares, kept on the device so that a whole Arnoldi cycle of all
// patches runs without host round trips (and can be captured in a CUDA graph).
#include "common.cuh"

namespace iga {

constexpr int kSegChunk = 2048;
constexpr int kSegThreads = 256;
constexpr int kSegMaxM = 32;

__device__ __forceinline__ int find_patch(const int32_t* __restrict__ blk0, int np, int b) {
  int lo = 0, hi = np;  // blk0[lo] <= b < blk0[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(blk0 + mid) <= b) lo = mid;
    else hi = mid;
  }
  return lo;
}

// stage 1: partial[b*m + j] = sum over the block's elements of A_j[i] * x[i].
// MB (4, 8, 16 or 32) >= m bounds the unrolled accumulator set.
template <typename T, int MB>
__global__ void __launch_bounds__(kSegThreads)
    seg_gram_stage1(int np, const int64_t* __restrict__ offs, const int32_t* __restrict__ blk0,
                    int m, const T* __restrict__ A, int64_t lda, const T* __restrict__ x,
                    double* __restrict__ partial) {
  const int b = blockIdx.x;
  const int p = find_patch(blk0, np, b);
  const int64_t i0 = offs[p] + (int64_t)(b - blk0[p]) * kSegChunk;
  const int64_t i1 = min(i0 + kSegChunk, offs[p + 1]);
  double acc[MB];
#pragma unroll
  for (int j = 0; j < MB; ++j) acc[j] = 0.0;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += kSegThreads) {
    const double xv = (double)x[i];
#pragma unroll
    for (int j = 0; j < MB; ++j)
      if (j < m) acc[j] += (double)A[j * lda + i] * xv;
  }
  __shared__ double red[kSegThreads / 32][MB];
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
    for (int w = 0; w < kSegThreads / 32; ++w) v += red[w][threadIdx.x];
    partial[(int64_t)b * m + threadIdx.x] = v;
  }
}

// stage 2: out[p*ldo + j] = sum over the patch's blocks, one CTA per patch.
// G = the largest power of two <= kSegThreads / m row groups; group g sums
// blocks g, g+G, ... of the patch, then a halving tree over the groups; the
// order of every addition is fixed by (m, block count) alone.
__global__ void __launch_bounds__(kSegThreads)
    seg_gram_stage2(int np, const int32_t* __restrict__ blk0, int m,
                    const double* __restrict__ partial, double* __restrict__ out, int64_t ldo) {
  __shared__ double red[kSegThreads];
  const int p = blockIdx.x;
  if (p >= np) return;
  int G = 1;
  while (2 * G * m <= kSegThreads) G *= 2;
  const int t = threadIdx.x, g = t / m, j = t - g * m;
  const int b0 = blk0[p], b1 = blk0[p + 1];
  double v = 0.0;
  if (g < G)
    for (int b = b0 + g; b < b1; b += G) v += partial[(int64_t)b * m + j];
  red[t] = v;
  __syncthreads();
  for (int s = G / 2; s > 0; s >>= 1) {
    if (g < s) red[t] += red[t + s * m];
    __syncthreads();
  }
  if (t < m) out[(int64_t)p * ldo + t] = red[t];
}

// out[i] = beta*out[i] + alpha * sum_j coef[p*ldc + j] * A_j[i]
template <typename T>
__global__ void __launch_bounds__(kSegThreads)
    seg_combine_kernel(int np, const int64_t* __restrict__ offs, const int32_t* __restrict__ blk0,
                       int m, const T* __restrict__ A, int64_t lda, const double* __restrict__ coef,
                       int64_t ldc, double alpha, double beta, T* __restrict__ out) {
  const int b = blockIdx.x;
  const int p = find_patch(blk0, np, b);
  __shared__ double c[kSegMaxM];
  if (threadIdx.x < m) c[threadIdx.x] = alpha * coef[(int64_t)p * ldc + threadIdx.x];
  __syncthreads();
  const int64_t i0 = offs[p] + (int64_t)(b - blk0[p]) * kSegChunk;
  const int64_t i1 = min(i0 + kSegChunk, offs[p + 1]);
  for (int64_t i = i0 + threadIdx.x; i < i1; i += kSegThreads) {
    double v = beta == 0.0 ? 0.0 : beta * (double)out[i];
    for (int j = 0; j < m; ++j) v += c[j] * (double)A[j * lda + i];
    out[i] = (T)v;
  }
}

// x[i] *= f(s[p*lds]); mode 0: f = s, 1: f = 1/s, 2: f = 1/sqrt(s) (0 if s <= 0)
template <typename T>
__global__ void __launch_bounds__(kSegThreads)
    seg_scale_kernel(int np, const int64_t* __restrict__ offs, const int32_t* __restrict__ blk0,
                     T* __restrict__ x, const double* __restrict__ s, int64_t lds, int mode) {
  const int b = blockIdx.x;
  const int p = find_patch(blk0, np, b);
  const double sv = s[(int64_t)p * lds];
  double f;
  if (mode == 2) {
    const double r = sqrt(fmax(sv, 0.0));
    f = r > 0.0 ? 1.0 / r : 0.0;
  } else {
    f = mode ? 1.0 / sv : sv;
  }
  const int64_t i0 = offs[p] + (int64_t)(b - blk0[p]) * kSegChunk;
  const int64_t i1 = min(i0 + kSegChunk, offs[p + 1]);
  for (int64_t i = i0 + threadIdx.x; i < i1; i += kSegThreads) x[i] = (T)((double)x[i] * f);
}

// Hessenberg of patch p: H[p*m*(m+1) + j*(m+1) + i], column j rows 0..j then
// the squared norm of the new basis vector at row j+1.
__global__ void seg_givens_init(int np, const double* __restrict__ beta2, double* __restrict__ g,
                                int m, int32_t* __restrict__ conv, double* __restrict__ resid) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const double b = sqrt(fmax(beta2[p], 0.0));
  for (int i = 0; i <= m; ++i) g[(int64_t)p * (m + 1) + i] = 0.0;
  g[(int64_t)p * (m + 1)] = b;
  conv[p] = -1;
  resid[p] = b;
}

// Column j: add the second Gram-Schmidt pass (h2), take the square root of
// the norm entry, apply the previous rotations, make the new one, update the
// residual |g[j+1]|; record the first step whose residual is below tol*ref
// (resid then keeps that step's residual: the estimate of the solution the
// back substitution returns).
__global__ void seg_givens_step(int np, int m, int j, double* __restrict__ H,
                                const double* __restrict__ h2, int64_t ldh2,
                                double* __restrict__ cs, double* __restrict__ sn,
                                double* __restrict__ g, const double* __restrict__ ref,
                                double tol, int32_t* __restrict__ conv,
                                double* __restrict__ resid) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  double* h = H + (int64_t)p * m * (m + 1) + (int64_t)j * (m + 1);
  double* c = cs + (int64_t)p * m;
  double* s = sn + (int64_t)p * m;
  double* gp = g + (int64_t)p * (m + 1);
  for (int i = 0; i <= j; ++i) h[i] += h2[(int64_t)p * ldh2 + i];
  double hn = sqrt(fmax(h[j + 1], 0.0));
  for (int i = 0; i < j; ++i) {
    const double a = h[i], bb = h[i + 1];
    h[i] = c[i] * a + s[i] * bb;
    h[i + 1] = -s[i] * a + c[i] * bb;
  }
  const double a = h[j];
  const double r = hypot(a, hn);
  double cj = 1.0, sj = 0.0;
  if (r > 0.0) {
    cj = a / r;
    sj = hn / r;
  }
  h[j] = r;
  h[j + 1] = 0.0;
  c[j] = cj;
  s[j] = sj;
  const double gj = gp[j];
  gp[j] = cj * gj;
  gp[j + 1] = -sj * gj;
  const double res = fabs(gp[j + 1]);
  if (conv[p] < 0) {
    resid[p] = res;
    if (res < tol * ref[p] || ref[p] == 0.0) conv[p] = j;
  }
}

// y[p*m + i], i < k_p: back substitution R y = g with k_p = conv[p]+1 (or k
// when the patch has not converged within the cycle); y[p*m + i] = 0 beyond.
__global__ void seg_trisolve(int np, int m, int k, const double* __restrict__ H,
                             const double* __restrict__ g, const int32_t* __restrict__ conv,
                             double* __restrict__ y) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const int kp = conv[p] >= 0 ? min(conv[p] + 1, k) : k;
  const double* Hp = H + (int64_t)p * m * (m + 1);
  const double* gp = g + (int64_t)p * (m + 1);
  double* yp = y + (int64_t)p * m;
  for (int i = kp; i < m; ++i) yp[i] = 0.0;
  for (int i = kp - 1; i >= 0; --i) {
    double v = gp[i];
    for (int l = i + 1; l < kp; ++l) v -= Hp[(int64_t)l * (m + 1) + i] * yp[l];
    const double d = Hp[(int64_t)i * (m + 1) + i];
    yp[i] = d != 0.0 ? v / d : 0.0;
  }
}

}  // namespace iga

using namespace iga;

extern "C" {

int iga_seg_chunk(void) { return kSegChunk; }

iga_status iga_seg_gram(int dtype, int np, const int64_t* offs, const int32_t* blk0, int nblk,
                        int m, const void* A, int64_t lda, const void* x, double* partial,
                        double* out, int64_t ldo, iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(np >= 1 && nblk >= np && m >= 1 && m <= kSegMaxM, "np %d nblk %d m %d", np, nblk,
                m);
  IGA_CHECK_ARG(offs && blk0 && A && x && partial && out, "null argument");
  cudaStream_t st = as_stream(stream);
  if (dtype != IGA_F64 && dtype != IGA_F32) {
    set_error("dtype %d not supported", dtype);
    return IGA_ERR_UNSUPPORTED;
  }
#define IGA_SEG_GRAM1(MB)                                                                     \
  do {                                                                                        \
    if (dtype == IGA_F64)                                                                     \
      seg_gram_stage1<double, MB><<<nblk, kSegThreads, 0, st>>>(                              \
          np, offs, blk0, m, (const double*)A, lda, (const double*)x, partial);               \
    else                                                                                      \
      seg_gram_stage1<float, MB><<<nblk, kSegThreads, 0, st>>>(                               \
          np, offs, blk0, m, (const float*)A, lda, (const float*)x, partial);                 \
  } while (0)
  if (m <= 4)
    IGA_SEG_GRAM1(4);
  else if (m <= 8)
    IGA_SEG_GRAM1(8);
  else if (m <= 16)
    IGA_SEG_GRAM1(16);
  else
    IGA_SEG_GRAM1(32);
#undef IGA_SEG_GRAM1
  IGA_LAUNCH_CHECK();
  seg_gram_stage2<<<np, kSegThreads, 0, st>>>(np, blk0, m, partial, out, ldo);
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

iga_status iga_seg_combine(int dtype, int np, const int64_t* offs, const int32_t* blk0, int nblk,
                           int m, const void* A, int64_t lda, const double* coef, int64_t ldc,
                           double alpha, double beta, void* out, iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(np >= 1 && nblk >= np && m >= 0 && m <= kSegMaxM, "np %d nblk %d m %d", np, nblk,
                m);
  IGA_CHECK_ARG(offs && blk0 && out && (m == 0 || (A && coef)), "null argument");
  cudaStream_t st = as_stream(stream);
  if (dtype == IGA_F64)
    seg_combine_kernel<double><<<nblk, kSegThreads, 0, st>>>(
        np, offs, blk0, m, (const double*)A, lda, coef, ldc, alpha, beta, (double*)out);
  else if (dtype == IGA_F32)
    seg_combine_kernel<float><<<nblk, kSegThreads, 0, st>>>(
        np, offs, blk0, m, (const float*)A, lda, coef, ldc, alpha, beta, (float*)out);
  else {
    set_error("dtype %d not supported", dtype);
    return IGA_ERR_UNSUPPORTED;
  }
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

iga_status iga_seg_scale(int dtype, int np, const int64_t* offs, const int32_t* blk0, int nblk,
                         void* x, const double* s, int64_t lds, int mode, iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(np >= 1 && nblk >= np && mode >= 0 && mode <= 2, "np %d nblk %d mode %d", np,
                nblk, mode);
  IGA_CHECK_ARG(offs && blk0 && x && s, "null argument");
  cudaStream_t st = as_stream(stream);
  if (dtype == IGA_F64)
    seg_scale_kernel<double><<<nblk, kSegThreads, 0, st>>>(np, offs, blk0, (double*)x, s, lds,
                                                           mode);
  else if (dtype == IGA_F32)
    seg_scale_kernel<float><<<nblk, kSegThreads, 0, st>>>(np, offs, blk0, (float*)x, s, lds, mode);
  else {
    set_error("dtype %d not supported", dtype);
    return IGA_ERR_UNSUPPORTED;
  }
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

iga_status iga_seg_givens_init(int np, int m, const double* beta2, double* g, int32_t* conv,
                               double* resid, iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(np >= 1 && m >= 1 && m <= kSegMaxM && beta2 && g && conv && resid,
                "bad argument");
  seg_givens_init<<<(unsigned)ceil_div(np, 128), 128, 0, as_stream(stream)>>>(np, beta2, g, m,
                                                                              conv, resid);
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

iga_status iga_seg_givens_step(int np, int m, int j, double* H, const double* h2, int64_t ldh2,
                               double* cs, double* sn, double* g, const double* ref, double tol,
                               int32_t* conv, double* resid, iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(np >= 1 && m >= 1 && m <= kSegMaxM && j >= 0 && j < m, "np %d m %d j %d", np, m,
                j);
  IGA_CHECK_ARG(H && h2 && cs && sn && g && ref && conv && resid, "null argument");
  seg_givens_step<<<(unsigned)ceil_div(np, 128), 128, 0, as_stream(stream)>>>(
      np, m, j, H, h2, ldh2, cs, sn, g, ref, tol, conv, resid);
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

iga_status iga_seg_trisolve(int np, int m, int k, const double* H, const double* g,
                            const int32_t* conv, double* y, iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(np >= 1 && m >= 1 && m <= kSegMaxM && k >= 1 && k <= m, "np %d m %d k %d", np, m,
                k);
  IGA_CHECK_ARG(H && g && conv && y, "null argument");
  seg_trisolve<<<(unsigned)ceil_div(np, 128), 128, 0, as_stream(stream)>>>(np, m, k, H, g, conv,
                                                                           y);
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

}  // extern "C"
