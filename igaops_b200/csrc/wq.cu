// Weighted-quadrature rules, computed natively on the host.
//
// The weighted-quadrature rules (src/igaops/quadrature/weighted_quad.py:
// 238-363) find, for each test function i, weights on the quadrature points
// of its support that integrate every target basis function exactly:
// w_i = z_i * v_i where v_i is the minimum-norm solution of
// (A diag(z_i)) v = b_i (the reference's optimisation problem "minimise
// ||diag(z_i)^-1 w|| subject to A w = b_i", which it hands to LSQR from zero,
// src/igaops/quadrature/utils/operations.py:107-143).  Each row system is
// small (about 2(p+1) target functions by the 2-3(p+1) points of the test
// support), so it is solved directly by a complete orthogonal decomposition
// (the construction of LAPACK's xGELSY): Householder QR with column
// pivoting G P = Q [R11 R12; 0 R22], rank r from |R_kk| > rcond |R_00|, then
// a QR of [R11 R12]^T whose orthonormal factor spans the row space, so the
// solution is the minimum-norm one.  A few microseconds per row instead of
// the ~1 ms of an interpreted iterative solver call.
//
// iga_wq_point_counts restates the point-count tables of the rules' point
// layout (src/igaops/quadrature/utils/wq_helpers.py:11-82,221-259): per test
// function the (test, target) pairs' shared element intervals, the count of
// pairs inside every element range, the maximum over test functions, and
// the per-element lower bound, checked against every multi-element range.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "common.cuh"

namespace iga {

namespace {

// Householder vector of x[0..n): on return x holds v (v[0] = 1 implied by
// the scaling below), tau and the new leading value beta (x -> beta e_1).
inline double householder(int n, double* x, double* tau) {
  double sig = 0.0;
  for (int i = 1; i < n; ++i) sig += x[i] * x[i];
  const double a = x[0];
  if (sig == 0.0) {
    *tau = 0.0;
    return a;
  }
  const double nrm = std::sqrt(a * a + sig);
  const double beta = a <= 0.0 ? nrm : -nrm;
  const double v0 = a - beta;
  for (int i = 1; i < n; ++i) x[i] /= v0;
  *tau = (beta - a) / beta;
  return beta;
}

// Minimum-norm least-squares solution of G v = b, G m x n row-major.
// Work arrays are the caller's (reused across rows).
struct CodSolver {
  std::vector<double> A, c, tau, nrm, T, tau2, u;
  std::vector<int> piv;

  void solve(int m, int n, const double* G, const double* b, double rcond, double* v) {
    // column-major copy: column j at A[j * m]
    A.assign((size_t)m * n, 0.0);
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < n; ++j) A[(size_t)j * m + i] = G[(size_t)i * n + j];
    c.assign(b, b + m);
    piv.resize(n);
    for (int j = 0; j < n; ++j) piv[j] = j;
    const int kmax = std::min(m, n);
    tau.assign(kmax, 0.0);
    nrm.resize(n);
    int r = 0;
    double r00 = 0.0;
    for (int k = 0; k < kmax; ++k) {
      // pivot: the remaining column of largest norm (recomputed: sizes are small)
      int best = k;
      double bn = -1.0;
      for (int j = k; j < n; ++j) {
        double s = 0.0;
        const double* col = &A[(size_t)j * m];
        for (int i = k; i < m; ++i) s += col[i] * col[i];
        nrm[j] = s;
        if (s > bn) {
          bn = s;
          best = j;
        }
      }
      if (best != k) {
        std::swap_ranges(&A[(size_t)k * m], &A[(size_t)k * m] + m, &A[(size_t)best * m]);
        std::swap(piv[k], piv[best]);
      }
      double* ak = &A[(size_t)k * m];
      const double beta = householder(m - k, ak + k, &tau[k]);
      // apply H = I - tau v v^T (v = [1, ak[k+1..]]) to the remaining columns and c
      if (tau[k] != 0.0) {
        for (int j = k + 1; j < n; ++j) {
          double* aj = &A[(size_t)j * m];
          double d = aj[k];
          for (int i = k + 1; i < m; ++i) d += ak[i] * aj[i];
          d *= tau[k];
          aj[k] -= d;
          for (int i = k + 1; i < m; ++i) aj[i] -= d * ak[i];
        }
        double d = c[k];
        for (int i = k + 1; i < m; ++i) d += ak[i] * c[i];
        d *= tau[k];
        c[k] -= d;
        for (int i = k + 1; i < m; ++i) c[i] -= d * ak[i];
      }
      ak[k] = beta;
      if (k == 0) r00 = std::fabs(beta);
      if (!(std::fabs(beta) > rcond * r00) || beta == 0.0) break;
      r = k + 1;
    }
    for (int j = 0; j < n; ++j) v[j] = 0.0;
    if (r == 0) return;
    // T = [R11 R12]^T, n x r column-major (column k = row k of R, columns k..n-1)
    T.assign((size_t)n * r, 0.0);
    for (int k = 0; k < r; ++k)
      for (int j = k; j < n; ++j) T[(size_t)k * n + j] = A[(size_t)j * m + k];
    // QR of T (no pivoting): T = Q2 S, S r x r upper triangular; R_top = S^T Q2^T
    tau2.assign(r, 0.0);
    for (int k = 0; k < r; ++k) {
      double* tk = &T[(size_t)k * n];
      const double beta = householder(n - k, tk + k, &tau2[k]);
      if (tau2[k] != 0.0)
        for (int j = k + 1; j < r; ++j) {
          double* tj = &T[(size_t)j * n];
          double d = tj[k];
          for (int i = k + 1; i < n; ++i) d += tk[i] * tj[i];
          d *= tau2[k];
          tj[k] -= d;
          for (int i = k + 1; i < n; ++i) tj[i] -= d * tk[i];
        }
      tk[k] = beta;
    }
    // S^T y = c[0..r) (forward substitution; S[i][j] = T[j * n + i], i <= j)
    u.assign(n, 0.0);
    for (int i = 0; i < r; ++i) {
      double s = c[i];
      for (int j = 0; j < i; ++j) s -= T[(size_t)i * n + j] * u[j];
      u[i] = s / T[(size_t)i * n + i];
    }
    // w = Q2 [y; 0] = H_0 ... H_{r-1} [y; 0]
    for (int k = r - 1; k >= 0; --k) {
      if (tau2[k] == 0.0) continue;
      const double* tk = &T[(size_t)k * n];
      double d = u[k];
      for (int i = k + 1; i < n; ++i) d += tk[i] * u[i];
      d *= tau2[k];
      u[k] -= d;
      for (int i = k + 1; i < n; ++i) u[i] -= d * tk[i];
    }
    for (int j = 0; j < n; ++j) v[piv[j]] = u[j];
  }
};

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
  CodSolver cod;
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
    cod.solve(m, n, G.data(), bsub.data(), rcond, x.data());
    for (int c = 0; c < n; ++c) out[cols[c]] = z[cols[c]] * x[c];
  }
  return IGA_OK;
}

// B-spline basis functions and derivatives at points, host code: knot span
// by binary search (the last s in [p, n-1] with U[s] <= x) and the non-zero
// functions of increasing degree with their derivatives from the table of
// knot differences (Piegl & Tiller, The NURBS Book, A2.1 and A2.3), one
// point at a time in the order of operations of the vectorised form.
// ders[(k * (p + 1) + j) * npts + i] is the k-th derivative of
// N_{span[i] - p + j, p} at x[i].
iga_status iga_bspline_basis(int degree, int nknots, const double* U, int64_t npts,
                             const double* x, int nders, int32_t* span, double* ders) {
  clear_error();
  const int p = degree;
  IGA_CHECK_ARG(p >= 0 && p <= 16 && nknots >= 2 * p + 2 && U && x && span && ders &&
                    npts >= 0 && nders >= 0 && nders <= 16,
                "bad argument");
  const int n = nknots - p - 1;
  std::vector<double> ndu((size_t)(p + 1) * (p + 1)), left(p + 1), right(p + 1), a(2 * (p + 1));
  auto NDU = [&](int r, int c) -> double& { return ndu[(size_t)r * (p + 1) + c]; };
  const int kmax = std::min(nders, p);
  for (int64_t i = 0; i < npts; ++i) {
    const double xi = x[i];
    int s = (int)(std::upper_bound(U, U + nknots, xi) - U) - 1;
    s = std::min(std::max(s, p), n - 1);
    span[i] = s;
    std::fill(a.begin(), a.end(), 0.0);
    NDU(0, 0) = 1.0;
    for (int j = 1; j <= p; ++j) {
      left[j] = xi - U[s + 1 - j];
      right[j] = U[s + j] - xi;
      double saved = 0.0;
      for (int r = 0; r < j; ++r) {
        NDU(j, r) = right[r + 1] + left[j - r];
        const double temp = NDU(r, j - 1) / NDU(j, r);
        NDU(r, j) = saved + right[r + 1] * temp;
        saved = left[j - r] * temp;
      }
      NDU(j, j) = saved;
    }
    for (int k = 0; k <= nders; ++k)
      for (int j = 0; j <= p; ++j) ders[((size_t)k * (p + 1) + j) * npts + i] = 0.0;
    for (int j = 0; j <= p; ++j) ders[(size_t)j * npts + i] = NDU(j, p);
    for (int r = 0; r <= p; ++r) {
      int s1 = 0, s2 = 1;
      a[0] = 1.0;
      for (int k = 1; k <= kmax; ++k) {
        double d = 0.0;
        const int rk = r - k, pk = p - k;
        if (r >= k) {
          a[s2 * (p + 1)] = a[s1 * (p + 1)] / NDU(pk + 1, rk);
          d = a[s2 * (p + 1)] * NDU(rk, pk);
        }
        const int j1 = rk >= -1 ? 1 : -rk;
        const int j2 = (r - 1) <= pk ? k - 1 : p - r;
        for (int jj = j1; jj <= j2; ++jj) {
          a[s2 * (p + 1) + jj] =
              (a[s1 * (p + 1) + jj] - a[s1 * (p + 1) + jj - 1]) / NDU(pk + 1, rk + jj);
          d = d + a[s2 * (p + 1) + jj] * NDU(rk + jj, pk);
        }
        if (r <= pk) {
          a[s2 * (p + 1) + k] = -a[s1 * (p + 1) + k - 1] / NDU(pk + 1, r);
          d = d + a[s2 * (p + 1) + k] * NDU(r, pk);
        }
        ders[((size_t)k * (p + 1) + r) * npts + i] = d;
        std::swap(s1, s2);
      }
    }
    double fac = p;
    for (int k = 1; k <= kmax; ++k) {
      for (int j = 0; j <= p; ++j) ders[((size_t)k * (p + 1) + j) * npts + i] *= fac;
      fac *= p - k;
    }
  }
  return IGA_OK;
}

// Point counts per element of a weighted-quadrature rule.  test_range /
// targ_range: (first, last) element covered with positive measure by each
// test / target basis function, 2 * ntest / 2 * ntarg ints.  For test i and
// element range [a, b] inside its support, mubar_i(a, b) counts the (test
// i, target j) pairs whose shared element interval lies inside [a, b];
// counts[e] = max_i mubar_i(e, e) + 1.  A multi-element range [r, s] needs
// max_i mubar_i(r, s) points; since a range clamped to a test's support
// only loses points, it suffices to check the ranges inside every support:
// *feasible = 1 when every one holds, else 0 (the caller then raises the
// counts by the integer program).
iga_status iga_wq_point_counts(int ne, int ntest, const int32_t* test_range, int ntarg,
                               const int32_t* targ_range, int32_t* counts, int32_t* feasible) {
  clear_error();
  IGA_CHECK_ARG(ne >= 1 && ntest >= 1 && ntarg >= 1 && test_range && targ_range && counts &&
                    feasible,
                "bad argument");
  for (int i = 0; i < ntest; ++i)
    IGA_CHECK_ARG(test_range[2 * i] >= 0 && test_range[2 * i] <= test_range[2 * i + 1] &&
                      test_range[2 * i + 1] < ne,
                  "test function %d has element range (%d, %d) outside [0, %d)", i,
                  test_range[2 * i], test_range[2 * i + 1], ne);
  for (int j = 0; j < ntarg; ++j)
    IGA_CHECK_ARG(targ_range[2 * j] >= 0 && targ_range[2 * j] <= targ_range[2 * j + 1] &&
                      targ_range[2 * j + 1] < ne,
                  "target function %d has element range (%d, %d) outside [0, %d)", j,
                  targ_range[2 * j], targ_range[2 * j + 1], ne);
  for (int e = 0; e < ne; ++e) counts[e] = 0;
  std::vector<int64_t> cnt, bar;
  // pass 1: per-element maxima (the diagonal); pass 2: the range checks
  std::vector<int64_t> diag(ne, 0);
  for (int pass = 0; pass < 2; ++pass) {
    std::vector<int64_t> csum;
    if (pass == 1) {
      csum.assign(ne + 1, 0);
      for (int e = 0; e < ne; ++e) {
        counts[e] = (int32_t)(diag[e] + 1);
        csum[e + 1] = csum[e] + counts[e];
      }
      *feasible = 1;
    }
    for (int i = 0; i < ntest; ++i) {
      const int tf = test_range[2 * i], tl = test_range[2 * i + 1], L = tl - tf + 1;
      cnt.assign((size_t)L * L, 0);
      for (int j = 0; j < ntarg; ++j) {
        const int r = std::max(tf, (int)targ_range[2 * j]);
        const int s2 = std::min(tl, (int)targ_range[2 * j + 1]);
        if (r <= s2) ++cnt[(size_t)(r - tf) * L + (s2 - tf)];
      }
      // bar(a, b) = sum over a <= k <= l <= b of cnt(k, l)
      bar.assign((size_t)L * L, 0);
      for (int a = L - 1; a >= 0; --a)
        for (int b = a; b < L; ++b) {
          int64_t v = cnt[(size_t)a * L + b];
          if (a + 1 <= b) v += bar[(size_t)(a + 1) * L + b];
          if (b - 1 >= a) v += bar[(size_t)a * L + (b - 1)];
          if (a + 1 <= b - 1) v -= bar[(size_t)(a + 1) * L + (b - 1)];
          bar[(size_t)a * L + b] = v;
        }
      if (pass == 0) {
        for (int a = 0; a < L; ++a) diag[tf + a] = std::max(diag[tf + a], bar[(size_t)a * L + a]);
      } else {
        for (int a = 0; a < L; ++a)
          for (int b = a + 1; b < L; ++b)
            if (csum[tf + b + 1] - csum[tf + a] < bar[(size_t)a * L + b]) *feasible = 0;
      }
    }
  }
  return IGA_OK;
}

}  // extern "C"
