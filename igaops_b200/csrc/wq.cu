// Weighted-quadrature weight rows, computed natively on the host.
//
// The weighted-quadrature rules (src/igaops/quadrature/weighted_quad.py:
// 238-363) find, for each test function i, weights on the quadrature points
// of its support that integrate every target basis function exactly:
// w_i = z_i * v_i where v_i solves (A diag(z_i)) v = b_i in the least-squares
// sense, minimum norm (the reference runs LSQR from zero for it,
// src/igaops/quadrature/utils/operations.py:287-323; on these consistent
// systems LSQR converges to the minimum-norm solution).  Each row system is
// small (about 2(p+1) target functions by the 2-3(p+1) points of the test
// support), so it is solved directly: a one-sided Jacobi SVD of the
// restricted matrix (Hestenes' method: plane rotations of column pairs
// until all columns are mutually orthogonal), then v = V S^+ U^T b with
// singular values below rcond * max dropped.  Microseconds per row instead
// of the ~1 ms of an interpreted iterative solver call.
#include <cmath>
#include <cstdint>
#include <vector>

#include "common.cuh"

namespace iga {

namespace {

// Minimum-norm least-squares solution of G v = b, G m x n row-major (copied).
void min_norm_solve(int m, int n, std::vector<double>& G, const double* b, double rcond,
                    double* v) {
  std::vector<double> V((size_t)n * n, 0.0);
  for (int j = 0; j < n; ++j) V[(size_t)j * n + j] = 1.0;
  auto col_dot = [&](int p, int q) {
    double s = 0.0;
    for (int i = 0; i < m; ++i) s += G[(size_t)i * n + p] * G[(size_t)i * n + q];
    return s;
  };
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < n - 1; ++p) {
      for (int q = p + 1; q < n; ++q) {
        const double alpha = col_dot(p, p), beta = col_dot(q, q), gamma = col_dot(p, q);
        if (gamma == 0.0) continue;
        const double rel = std::fabs(gamma) / std::sqrt(alpha * beta);
        if (!(rel > 1e-15)) continue;
        off = std::fmax(off, rel);
        // rotation angle that zeroes the (p, q) inner product
        const double zeta = (beta - alpha) / (2.0 * gamma);
        const double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
        const double c = 1.0 / std::sqrt(1.0 + t * t), s = c * t;
        for (int i = 0; i < m; ++i) {
          double& gp = G[(size_t)i * n + p];
          double& gq = G[(size_t)i * n + q];
          const double a = gp, bq = gq;
          gp = c * a - s * bq;
          gq = s * a + c * bq;
        }
        for (int i = 0; i < n; ++i) {
          double& vp = V[(size_t)i * n + p];
          double& vq = V[(size_t)i * n + q];
          const double a = vp, bq = vq;
          vp = c * a - s * bq;
          vq = s * a + c * bq;
        }
      }
    }
    if (off <= 1e-15) break;
  }
  // columns of G are now U_j sigma_j
  std::vector<double> sig(n);
  double smax = 0.0;
  for (int j = 0; j < n; ++j) {
    sig[j] = std::sqrt(col_dot(j, j));
    smax = std::fmax(smax, sig[j]);
  }
  for (int k = 0; k < n; ++k) v[k] = 0.0;
  for (int j = 0; j < n; ++j) {
    if (!(sig[j] > rcond * smax) || sig[j] == 0.0) continue;
    double gb = 0.0;  // (U_j sigma_j)^T b
    for (int i = 0; i < m; ++i) gb += G[(size_t)i * n + j] * b[i];
    const double f = gb / (sig[j] * sig[j]);
    for (int k = 0; k < n; ++k) v[k] += V[(size_t)k * n + j] * f;
  }
}

}  // namespace

}  // namespace iga

using namespace iga;

extern "C" {

iga_status iga_wq_min_norm_rows(int nrows, int nt, int npts, const double* A, const double* Z,
                                const double* B, double rcond, double* W) {
  clear_error();
  IGA_CHECK_ARG(nrows >= 0 && nt >= 1 && npts >= 1 && A && Z && B && W, "bad argument");
  IGA_CHECK_ARG(rcond >= 0.0 && rcond < 1.0, "rcond %g out of range", rcond);
  std::vector<int> cols, rows;
  std::vector<double> G, bsub, x;
  for (int i = 0; i < nrows; ++i) {
    const double* z = Z + (size_t)i * npts;
    const double* b = B + (size_t)i * nt;
    double* out = W + (size_t)i * npts;
    for (int j = 0; j < npts; ++j) out[j] = 0.0;
    cols.clear();
    for (int j = 0; j < npts; ++j)
      if (z[j] != 0.0) cols.push_back(j);
    // equations that constrain the active points, plus any with a non-zero
    // right-hand side (which then count in the least-squares residual)
    rows.clear();
    for (int r = 0; r < nt; ++r) {
      bool keep = b[r] != 0.0;
      for (size_t c = 0; !keep && c < cols.size(); ++c) keep = A[(size_t)r * npts + cols[c]] != 0.0;
      if (keep) rows.push_back(r);
    }
    if (cols.empty() || rows.empty()) continue;
    const int m = (int)rows.size(), n = (int)cols.size();
    G.assign((size_t)m * n, 0.0);
    bsub.resize(m);
    for (int r = 0; r < m; ++r) {
      bsub[r] = b[rows[r]];
      for (int c = 0; c < n; ++c)
        G[(size_t)r * n + c] = A[(size_t)rows[r] * npts + cols[c]] * z[cols[c]];
    }
    x.assign(n, 0.0);
    min_norm_solve(m, n, G, bsub.data(), rcond, x.data());
    for (int c = 0; c < n; ++c) out[cols[c]] = z[cols[c]] * x[c];
  }
  return IGA_OK;
}

}  // extern "C"
