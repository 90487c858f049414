// Solve-level C entry point: flexible, right-preconditioned GMRES with its
// Krylov vectors on the device.
//
// The reference's LinearSolver.solve(Afun, b, Pfun) with linear_type "gmres"
// (src/igaops/solvers/linear_solver.py:149-257,438-525) takes the operator and
// the preconditioner as callables; here they are C callbacks that receive
// device pointers and the stream (a C caller builds them from iga_mf_matvec,
// iga_fd_apply, ... or its own kernels).  Unrestarted GMRES storing Z = P V
// (flexible form), two classical Gram-Schmidt passes (iga_gram / iga_combine,
// the same count as the reference's two modified passes), the Dirichlet DOFs
// of `dirichlet` zeroed in b and in every operator / preconditioner input and
// output (the reference's cleandod, linear_solver.py:119-124,213-233).  The
// small Hessenberg problem is solved on the host by Givens rotations (one
// device-to-host read of the projections and the new norm per iteration);
// stopping rules: relative residual < tolerance or absolute residual
// < 1e-14 (convergence_manager defaults of the reference).
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"

using namespace iga;

extern "C" {

iga_status iga_gram(int dtype, int cplx, int64_t n, int m1, const void* A, int64_t lda, int m2,
                    const void* B, int64_t ldb, double* out, double* partial, int nblk,
                    iga_stream stream);
iga_status iga_gram_workspace(int64_t n, int m1, int m2, int cplx, int* nblk, int64_t* elems);
iga_status iga_combine(int dtype, int cplx, int64_t n, int m_in, const void* A, int64_t lda,
                       int kout, const double* coef, double alpha, double beta, void* out,
                       int64_t ldo, iga_stream stream);
iga_status iga_axpby(int dtype, int64_t n, double alpha, const void* x, double beta, void* y,
                     iga_stream stream);
iga_status iga_mask_zero(int dtype, int64_t nidx, const int64_t* idx, void* x,
                         iga_stream stream);

iga_status iga_gmres_workspace(int64_t n, int maxiters, int64_t* elems) {
  clear_error();
  IGA_CHECK_ARG(n >= 1 && maxiters >= 1 && maxiters <= 4000 && elems, "bad argument");
  int nblk = 0;
  int64_t pe = 0;
  iga_status rc = iga_gram_workspace(n, maxiters + 1, 1, 0, &nblk, &pe);
  if (rc) return rc;
  // V (m + 1) n, Z m n, w n, r n, coefficients 2 (m + 1) + 1, gram scratch
  *elems = (int64_t)(2 * maxiters + 3) * n + 2 * (maxiters + 2) + pe;
  return IGA_OK;
}

iga_status iga_gmres_solve(int64_t n, const double* b, double* x, double tolerance,
                           int maxiters, iga_apply_fn A, iga_apply_fn P, void* user,
                           const int64_t* dirichlet, int64_t ndirichlet, double* work,
                           int64_t work_elems, double* residual_history, int* iterations,
                           iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(n >= 1 && b && x && A && work && maxiters >= 1, "bad argument");
  IGA_CHECK_ARG(tolerance > 0.0 && tolerance < 1.0, "tolerance must be in (0, 1), got %g",
                tolerance);
  IGA_CHECK_ARG(ndirichlet == 0 || dirichlet, "null Dirichlet index array");
  int64_t need = 0;
  iga_status rc = iga_gmres_workspace(n, maxiters, &need);
  if (rc) return rc;
  IGA_CHECK_ARG(work_elems >= need, "workspace holds %lld elements, %lld needed",
                (long long)work_elems, (long long)need);
  cudaStream_t st = as_stream(stream);
  const int m = maxiters;
  double* V = work;                         // (m + 1) x n
  double* Z = V + (int64_t)(m + 1) * n;     // m x n
  double* w = Z + (int64_t)m * n;           // n
  double* r = w + n;                        // n
  double* hd = r + n;                       // 2 (m + 1) + 1: projections, norm / coefficients
  double* partial = hd + 2 * (m + 2);
  int nblk = 0;
  int64_t pe = 0;
  if ((rc = iga_gram_workspace(n, m + 1, 1, 0, &nblk, &pe))) return rc;
  auto mask = [&](double* v) -> iga_status {
    return ndirichlet ? iga_mask_zero(IGA_F64, ndirichlet, dirichlet, v, stream) : IGA_OK;
  };
  auto read = [&](const double* src, double* dst, int cnt) -> iga_status {
    IGA_CUDA_TRY(cudaMemcpyAsync(dst, src, sizeof(double) * cnt, cudaMemcpyDeviceToHost, st));
    IGA_CUDA_TRY(cudaStreamSynchronize(st));
    return IGA_OK;
  };
  if (iterations) *iterations = 0;
  IGA_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(double) * n, st));
  IGA_CUDA_TRY(cudaMemcpyAsync(r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  if ((rc = mask(r))) return rc;
  if ((rc = iga_gram(IGA_F64, 0, n, 1, r, n, 1, r, n, hd, partial, nblk, stream))) return rc;
  double beta2 = 0.0;
  if ((rc = read(hd, &beta2, 1))) return rc;
  if (!std::isfinite(beta2)) {
    set_error("iga_gmres_solve: right-hand side holds non-finite values");
    return IGA_ERR_NONFINITE;
  }
  const double beta = std::sqrt(std::max(beta2, 0.0));
  if (residual_history) residual_history[0] = 1.0;
  if (beta < 1e-14) return IGA_OK;  // the reference stops before iterating
  if ((rc = iga_axpby(IGA_F64, n, 1.0 / beta, r, 0.0, V, stream))) return rc;
  // Hessenberg (column-major, (m + 1) x m), rotations, rhs of the least squares
  std::vector<double> H((size_t)(m + 1) * m, 0.0), cs(m, 0.0), sn(m, 0.0), g(m + 1, 0.0);
  std::vector<double> hv(2 * (m + 1) + 1);
  g[0] = beta;
  int k = 0;
  bool converged = false;
  iga_status result = IGA_ERR_NOT_CONVERGED;
  for (int it = 1; it <= m; ++it) {
    double* vj = V + (int64_t)(it - 1) * n;
    double* zj = Z + (int64_t)(it - 1) * n;
    if (P) {
      IGA_CUDA_TRY(cudaMemcpyAsync(w, vj, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
      if ((rc = mask(w))) return rc;
      if ((rc = P(user, w, zj, stream))) return rc;
    } else {
      IGA_CUDA_TRY(cudaMemcpyAsync(zj, vj, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    }
    if ((rc = mask(zj))) return rc;
    if ((rc = A(user, zj, w, stream))) return rc;
    if ((rc = mask(w))) return rc;
    // two classical Gram-Schmidt passes, then the new norm
    for (int pass = 0; pass < 2; ++pass) {
      double* h = hd + pass * (m + 1);
      if ((rc = iga_gram(IGA_F64, 0, n, it, V, n, 1, w, n, h, partial, nblk, stream))) return rc;
      if ((rc = iga_combine(IGA_F64, 0, n, it, V, n, 1, h, -1.0, 1.0, w, n, stream))) return rc;
    }
    double* nrm = hd + 2 * (m + 1);
    if ((rc = iga_gram(IGA_F64, 0, n, 1, w, n, 1, w, n, nrm, partial, nblk, stream))) return rc;
    // one read: both passes and the norm (the passes sit m + 1 apart)
    if ((rc = read(hd, hv.data(), 2 * (m + 1) + 1))) return rc;
    for (int i = 0; i < 2 * (m + 1) + 1; ++i)
      if ((i < it || (i >= m + 1 && i < m + 1 + it) || i == 2 * (m + 1)) && !std::isfinite(hv[i])) {
        set_error("iga_gmres_solve: non-finite value in the Arnoldi step (operator or "
                  "preconditioner output)");
        return IGA_ERR_NONFINITE;
      }
    double* col = H.data() + (size_t)(it - 1) * (m + 1);
    for (int i = 0; i < it; ++i) col[i] = hv[i] + hv[m + 1 + i];
    const double nw = std::sqrt(std::max(hv[2 * (m + 1)], 0.0));
    col[it] = nw;
    if (nw != 0.0) {
      if ((rc = iga_axpby(IGA_F64, n, 1.0 / nw, w, 0.0, V + (int64_t)it * n, stream))) return rc;
    } else {
      IGA_CUDA_TRY(cudaMemsetAsync(V + (int64_t)it * n, 0, sizeof(double) * n, st));
    }
    // previous rotations, then the new one
    for (int i = 0; i < it - 1; ++i) {
      const double a = col[i], c = col[i + 1];
      col[i] = cs[i] * a + sn[i] * c;
      col[i + 1] = -sn[i] * a + cs[i] * c;
    }
    const double a = col[it - 1], c = col[it];
    const double rr = std::hypot(a, c);
    cs[it - 1] = rr > 0.0 ? a / rr : 1.0;
    sn[it - 1] = rr > 0.0 ? c / rr : 0.0;
    col[it - 1] = rr;
    col[it] = 0.0;
    g[it] = -sn[it - 1] * g[it - 1];
    g[it - 1] = cs[it - 1] * g[it - 1];
    const double res = std::fabs(g[it]);
    if (residual_history) residual_history[it] = res / beta;
    k = it;
    if (res / beta < tolerance || res < 1e-14) {
      converged = true;
      break;
    }
    if (nw == 0.0) {
      // the Krylov space is invariant but the residual did not drop
      result = IGA_ERR_BREAKDOWN;
      break;
    }
  }
  if (iterations) *iterations = k;
  // y = R^-1 g (host), x = Z[:k]^T y (device)
  std::vector<double> y(k, 0.0);
  for (int i = k - 1; i >= 0; --i) {
    double v = g[i];
    for (int l = i + 1; l < k; ++l) v -= H[(size_t)l * (m + 1) + i] * y[l];
    const double d = H[(size_t)i * (m + 1) + i];
    y[i] = d != 0.0 ? v / d : 0.0;
  }
  if (k > 0) {
    IGA_CUDA_TRY(cudaMemcpyAsync(hd, y.data(), sizeof(double) * k, cudaMemcpyHostToDevice, st));
    if ((rc = iga_combine(IGA_F64, 0, n, k, Z, n, 1, hd, 1.0, 0.0, x, n, stream))) return rc;
    IGA_CUDA_TRY(cudaStreamSynchronize(st));  // y lives on this frame
  }
  if ((rc = mask(x))) return rc;
  if (converged) return IGA_OK;
  set_error(result == IGA_ERR_BREAKDOWN ? "iga_gmres_solve: Krylov breakdown before convergence"
                                        : "iga_gmres_solve: no convergence within maxiters");
  return result;
}

}  // extern "C"
