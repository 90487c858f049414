// Space-time fast-diagonalisation preconditioner (arrowhead form).
//
// SpTimeFD.apply / apply_transpose (src/igaops/fastdiag/utils/time_arrow.py:
// 112-192): on the free nodes (time indices 1..nt-1 times the spatial free
// box; time is the slowest direction)
//   x -> (U_s^T per space direction) -> (conj(Ut)^T in time)
//     -> arrowhead solve with H_ij = adv*Dt_i + Lambda_j
//     -> (Ut in time) -> (U_s per space direction) -> real part,
// where Ut (complex) diagonalises the time pencil except for one border row
// and column (the arrowhead g).  The transpose swaps Ut / conj(Ut) and uses
// -conj(g).  The arrowhead solve (operations.py:5-93) is one thread per
// spatial eigen-index j walking the time index i: block elimination of the
// border with the Schur complement computed on the fly, complex arithmetic
// in FP64, storage in the element type of the call.
#include "common.cuh"

namespace iga {

template <typename T>
__global__ void __launch_bounds__(256)
    arrowhead_kernel(int mt, int64_t ms, const double* __restrict__ dt,
                     const double* __restrict__ b, const double* __restrict__ lam,
                     T* __restrict__ re, T* __restrict__ im) {
  const int k = mt - 1;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < ms;
       j += (int64_t)gridDim.x * blockDim.x) {
    const double l = lam[j];
    double sr = dt[2 * k] + l, si = dt[2 * k + 1];  // H_last, then the Schur complement
    double ar = 0.0, ai = 0.0;                       // sum_i conj(b_i) y_i
    for (int i = 0; i < k; ++i) {
      const double hr = dt[2 * i] + l, hi = dt[2 * i + 1];
      const double den = hr * hr + hi * hi;
      const double br = b[2 * i], bi = b[2 * i + 1];
      const double bb = br * br + bi * bi;
      sr += bb * hr / den;
      si -= bb * hi / den;
      const int64_t o = (int64_t)i * ms + j;
      const double rr = (double)re[o], ri = (double)im[o];
      const double yr = (rr * hr + ri * hi) / den, yi = (ri * hr - rr * hi) / den;
      re[o] = (T)yr;
      im[o] = (T)yi;
      ar += br * yr + bi * yi;
      ai += br * yi - bi * yr;
    }
    const int64_t ol = (int64_t)k * ms + j;
    const double lr = (double)re[ol] + ar, li = (double)im[ol] + ai;
    const double sd = sr * sr + si * si;
    const double xr = (lr * sr + li * si) / sd, xi = (li * sr - lr * si) / sd;
    re[ol] = (T)xr;
    im[ol] = (T)xi;
    for (int i = 0; i < k; ++i) {
      const double hr = dt[2 * i] + l, hi = dt[2 * i + 1];
      const double den = hr * hr + hi * hi;
      const double br = b[2 * i], bi = b[2 * i + 1];
      const double mr = (br * hr + bi * hi) / den, mi = (bi * hr - br * hi) / den;
      const int64_t o = (int64_t)i * ms + j;
      re[o] = (T)((double)re[o] - (mr * xr - mi * xi));
      im[o] = (T)((double)im[o] - (mr * xi + mi * xr));
    }
  }
}

// Triangular solves of the QZ (legacy) space-time FD (src/igaops/fastdiag/
// utils/time_legacy.py:61-170): for every spatial eigen-index j, the time
// vector (re, im)[i * ms + j], i < mt, is replaced by the solution of
//   (adv S + lam_j T) y = rhs        (upper triangular; apply)
//   (adv S + lam_j T)^T y = rhs      (lower triangular; transpose)
// with S, T the complex generalized Schur forms (row-major (re, im) pairs).
// One thread per j, complex arithmetic in FP64.
template <typename T>
__global__ void __launch_bounds__(256)
    qz_tri_kernel(int mt, int64_t ms, const double* __restrict__ S, const double* __restrict__ Tm,
                  double adv, const double* __restrict__ lam, int transpose, T* __restrict__ re,
                  T* __restrict__ im) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < ms;
       j += (int64_t)gridDim.x * blockDim.x) {
    const double l = lam[j];
    for (int s = 0; s < mt; ++s) {
      const int i = transpose ? s : mt - 1 - s;
      double ar = (double)re[(int64_t)i * ms + j], ai = (double)im[(int64_t)i * ms + j];
      const int k0 = transpose ? 0 : i + 1, k1 = transpose ? i : mt;
      for (int k = k0; k < k1; ++k) {
        // M_ik (apply) or M_ki (transpose), M = adv S + lam T
        const int64_t e = transpose ? ((int64_t)k * mt + i) : ((int64_t)i * mt + k);
        const double mr = adv * S[2 * e] + l * Tm[2 * e];
        const double mi = adv * S[2 * e + 1] + l * Tm[2 * e + 1];
        const double yr = (double)re[(int64_t)k * ms + j], yi = (double)im[(int64_t)k * ms + j];
        ar -= mr * yr - mi * yi;
        ai -= mr * yi + mi * yr;
      }
      const int64_t d = (int64_t)i * mt + i;
      const double dr = adv * S[2 * d] + l * Tm[2 * d], di = adv * S[2 * d + 1] + l * Tm[2 * d + 1];
      const double den = dr * dr + di * di;
      re[(int64_t)i * ms + j] = (T)((ar * dr + ai * di) / den);
      im[(int64_t)i * ms + j] = (T)((ai * dr - ar * di) / den);
    }
  }
}

}  // namespace iga

using namespace iga;

extern "C" {

iga_status iga_mode_product(int dtype, const iga_factor* M, int64_t outer, int64_t inner,
                            const void* x, void* y, int accumulate, iga_stream stream);
iga_status iga_axpby(int dtype, int64_t n, double alpha, const void* x, double beta, void* y,
                     iga_stream stream);
iga_status iga_box_copy(int dtype, int ndim, const int32_t* n, const int32_t* lo,
                        const int32_t* m, int64_t ncols, const void* src, void* dst, int scatter,
                        iga_stream stream);

iga_status iga_arrowhead_solve(int dtype, int mt, int64_t ms, const double* dt, const double* b,
                               const double* lam, void* re, void* im, iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(mt >= 1 && ms >= 0 && dt && lam && re && im && (mt == 1 || b), "bad argument");
  if (ms == 0) return IGA_OK;
  int64_t blocks = ceil_div(ms, 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  cudaStream_t st = as_stream(stream);
  if (dtype == IGA_F64)
    arrowhead_kernel<double><<<(unsigned)blocks, 256, 0, st>>>(mt, ms, dt, b, lam, (double*)re,
                                                               (double*)im);
  else if (dtype == IGA_F32)
    arrowhead_kernel<float><<<(unsigned)blocks, 256, 0, st>>>(mt, ms, dt, b, lam, (float*)re,
                                                              (float*)im);
  else {
    set_error("dtype %d not supported", dtype);
    return IGA_ERR_UNSUPPORTED;
  }
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

iga_status iga_fd_sptime_apply(int dtype, int sdim, const int32_t* n, const int32_t* lo,
                               const int32_t* m, const void* const* U, const void* ut_re,
                               const void* ut_im, const double* dt, const double* bfac,
                               const double* lam, int transpose, const void* x, void* y,
                               void* work0, void* work1, void* work2, iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(sdim >= 1 && sdim <= 3, "space dimension %d out of range", sdim);
  IGA_CHECK_ARG(n && lo && m && U && ut_re && ut_im && dt && lam && x && y && work0 && work1 &&
                    work2,
                "null argument");
  IGA_CHECK_ARG(dtype == IGA_F64 || dtype == IGA_F32, "dtype %d not supported", dtype);
  const int nd = sdim + 1;
  int64_t N = 1, M = 1, ms = 1;
  for (int d = 0; d < nd; ++d) {
    IGA_CHECK_ARG(m[d] >= 1 && lo[d] >= 0 && lo[d] + m[d] <= n[d], "box of direction %d", d);
    N *= n[d];
    M *= m[d];
    if (d < sdim) ms *= m[d];
  }
  const int mt = m[sdim];
  IGA_CHECK_ARG(mt == 1 || bfac, "null arrowhead border");
  cudaStream_t st = as_stream(stream);
  const size_t esz = dtype == IGA_F64 ? 8 : 4;
  IGA_CUDA_TRY(cudaMemsetAsync(y, 0, (size_t)N * esz, st));
  iga_status rc = iga_box_copy(dtype, nd, n, lo, m, 1, x, work0, 0, stream);
  if (rc) return rc;
  void* buf[2] = {work0, work1};
  int cur = 0;
  auto dense = [&](const void* A, int rows, bool tr) {
    iga_factor F;
    memset(&F, 0, sizeof(F));
    F.kind = 1;
    F.rows = F.cols = rows;
    F.ld_row = tr ? 1 : rows;
    F.ld_col = tr ? rows : 1;
    F.dense = A;
    return F;
  };
  auto space_pass = [&](bool forward) -> iga_status {
    // tensor (mt, m_sdim-1, ..., m_0): direction d has outer = mt * prod_{d'>d} m,
    // inner = prod_{d'<d} m
    for (int d = sdim - 1; d >= 0; --d) {
      iga_factor F = dense(U[d], m[d], forward);
      int64_t outer = mt, inner = 1;
      for (int e = sdim - 1; e > d; --e) outer *= m[e];
      for (int e = d - 1; e >= 0; --e) inner *= m[e];
      iga_status r = iga_mode_product(dtype, &F, outer, inner, buf[cur], buf[cur ^ 1], 0, stream);
      if (r) return r;
      cur ^= 1;
    }
    return IGA_OK;
  };
  if ((rc = space_pass(true))) return rc;
  // time forward: re = Ut_re^T a, im = -+ Ut_im^T a (conj(Ut)^T for apply, Ut^T for transpose)
  void* a = buf[cur];
  void* re = buf[cur ^ 1];
  void* im = work2;
  {
    iga_factor Fr = dense(ut_re, mt, true), Fi = dense(ut_im, mt, true);
    if ((rc = iga_mode_product(dtype, &Fr, 1, ms, a, re, 0, stream))) return rc;
    if ((rc = iga_mode_product(dtype, &Fi, 1, ms, a, im, 0, stream))) return rc;
    if (!transpose && (rc = iga_axpby(dtype, M, -1.0, im, 0.0, im, stream))) return rc;
  }
  if ((rc = iga_arrowhead_solve(dtype, mt, ms, dt, bfac, lam, re, im, stream))) return rc;
  // time backward: w = Re(Ut z) = Ut_re z_re - Ut_im z_im (apply) or
  // Re(conj(Ut) z) = Ut_re z_re + Ut_im z_im (transpose)
  {
    if (!transpose && (rc = iga_axpby(dtype, M, -1.0, im, 0.0, im, stream))) return rc;
    iga_factor Fr = dense(ut_re, mt, false), Fi = dense(ut_im, mt, false);
    if ((rc = iga_mode_product(dtype, &Fr, 1, ms, re, a, 0, stream))) return rc;
    if ((rc = iga_mode_product(dtype, &Fi, 1, ms, im, a, 1, stream))) return rc;
  }
  if ((rc = space_pass(false))) return rc;
  return iga_box_copy(dtype, nd, n, lo, m, 1, buf[cur], y, 1, stream);
}


iga_status iga_fd_sptime_qz_apply(int dtype, int sdim, const int32_t* n, const int32_t* lo,
                                  const int32_t* m, const void* const* U, const void* q_re,
                                  const void* q_im, const void* z_re, const void* z_im,
                                  const double* S, const double* Tm, double adv,
                                  const double* lam, int transpose, const void* x, void* y,
                                  void* work0, void* work1, void* work2, iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(sdim >= 1 && sdim <= 3, "space dimension %d out of range", sdim);
  IGA_CHECK_ARG(n && lo && m && U && q_re && q_im && z_re && z_im && S && Tm && lam && x && y &&
                    work0 && work1 && work2,
                "null argument");
  IGA_CHECK_ARG(dtype == IGA_F64 || dtype == IGA_F32, "dtype %d not supported", dtype);
  const int nd = sdim + 1;
  int64_t N = 1, M = 1, ms = 1;
  for (int d = 0; d < nd; ++d) {
    IGA_CHECK_ARG(m[d] >= 1 && lo[d] >= 0 && lo[d] + m[d] <= n[d], "box of direction %d", d);
    N *= n[d];
    M *= m[d];
    if (d < sdim) ms *= m[d];
  }
  const int mt = m[sdim];
  cudaStream_t st = as_stream(stream);
  const size_t esz = dtype == IGA_F64 ? 8 : 4;
  IGA_CUDA_TRY(cudaMemsetAsync(y, 0, (size_t)N * esz, st));
  iga_status rc = iga_box_copy(dtype, nd, n, lo, m, 1, x, work0, 0, stream);
  if (rc) return rc;
  void* buf[2] = {work0, work1};
  int cur = 0;
  auto dense = [&](const void* A, int rows, bool tr) {
    iga_factor F;
    memset(&F, 0, sizeof(F));
    F.kind = 1;
    F.rows = F.cols = rows;
    F.ld_row = tr ? 1 : rows;
    F.ld_col = tr ? rows : 1;
    F.dense = A;
    return F;
  };
  auto space_pass = [&](bool forward) -> iga_status {
    for (int d = sdim - 1; d >= 0; --d) {
      iga_factor F = dense(U[d], m[d], forward);
      int64_t outer = mt, inner = 1;
      for (int e = sdim - 1; e > d; --e) outer *= m[e];
      for (int e = d - 1; e >= 0; --e) inner *= m[e];
      iga_status r = iga_mode_product(dtype, &F, outer, inner, buf[cur], buf[cur ^ 1], 0, stream);
      if (r) return r;
      cur ^= 1;
    }
    return IGA_OK;
  };
  if ((rc = space_pass(true))) return rc;
  // time forward: Q^H a (apply: re = Q_re^T a, im = -Q_im^T a) or Z^T a
  // (transpose: re = Z_re^T a, im = Z_im^T a)
  void* a = buf[cur];
  void* re = buf[cur ^ 1];
  void* im = work2;
  {
    iga_factor Fr = dense(transpose ? z_re : q_re, mt, true);
    iga_factor Fi = dense(transpose ? z_im : q_im, mt, true);
    if ((rc = iga_mode_product(dtype, &Fr, 1, ms, a, re, 0, stream))) return rc;
    if ((rc = iga_mode_product(dtype, &Fi, 1, ms, a, im, 0, stream))) return rc;
    if (!transpose && (rc = iga_axpby(dtype, M, -1.0, im, 0.0, im, stream))) return rc;
  }
  {
    int64_t blocks = ceil_div(ms, 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    if (dtype == IGA_F64)
      qz_tri_kernel<double><<<(unsigned)blocks, 256, 0, st>>>(mt, ms, S, Tm, adv, lam, transpose,
                                                              (double*)re, (double*)im);
    else
      qz_tri_kernel<float><<<(unsigned)blocks, 256, 0, st>>>(mt, ms, S, Tm, adv, lam, transpose,
                                                             (float*)re, (float*)im);
    IGA_LAUNCH_CHECK();
  }
  // time backward: Re(Z y) = Z_re y_re - Z_im y_im (apply) or
  // Re(conj(Q) y) = Q_re y_re + Q_im y_im (transpose)
  {
    if (!transpose && (rc = iga_axpby(dtype, M, -1.0, im, 0.0, im, stream))) return rc;
    iga_factor Fr = dense(transpose ? q_re : z_re, mt, false);
    iga_factor Fi = dense(transpose ? q_im : z_im, mt, false);
    if ((rc = iga_mode_product(dtype, &Fr, 1, ms, re, a, 0, stream))) return rc;
    if ((rc = iga_mode_product(dtype, &Fi, 1, ms, im, a, 1, stream))) return rc;
  }
  if ((rc = space_pass(false))) return rc;
  return iga_box_copy(dtype, nd, n, lo, m, 1, buf[cur], y, 1, stream);
}

}  // extern "C"
