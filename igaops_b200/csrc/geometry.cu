// Pointwise geometry at quadrature points: metric, determinant, pseudo-
// inverse of the Jacobian and the stiffness coefficient tensor.
//
// Follows Operations.inverse_rectangular_matrix and
// eval_inverse_and_determinant (src/igaops/geometry/mixin/operations.py:
// 73-159): G = J^T J, det J = sqrt(det G), J^+ = G^{-1} J^T, with the
// closed-form 1x1 / 2x2 / 3x3 inverse of G; the coefficient of the stiffness
// operator is C = det J * J^+ J^{+T} (how the reference's tests and examples
// build it from EvaluatedSpline, tests/test_assemble.py:116-123).
#include "common.cuh"

namespace iga {

template <int D>
__device__ __forceinline__ void inv_det(const double (&G)[3][3], double (&inv)[3][3],
                                        double& det) {
  if (D == 1) {
    det = G[0][0];
    inv[0][0] = 1.0;
  } else if (D == 2) {
    det = G[0][0] * G[1][1] - G[0][1] * G[1][0];
    inv[0][0] = G[1][1];
    inv[1][1] = G[0][0];
    inv[0][1] = -G[0][1];
    inv[1][0] = -G[1][0];
  } else {
    det = G[0][1] * G[1][2] * G[2][0] - G[0][2] * G[1][1] * G[2][0] + G[0][2] * G[1][0] * G[2][1] -
          G[0][0] * G[1][2] * G[2][1] + G[0][0] * G[1][1] * G[2][2] - G[0][1] * G[1][0] * G[2][2];
    inv[0][0] = G[1][1] * G[2][2] - G[1][2] * G[2][1];
    inv[0][1] = G[0][2] * G[2][1] - G[0][1] * G[2][2];
    inv[0][2] = G[0][1] * G[1][2] - G[0][2] * G[1][1];
    inv[1][0] = G[1][2] * G[2][0] - G[1][0] * G[2][2];
    inv[1][1] = G[0][0] * G[2][2] - G[0][2] * G[2][0];
    inv[1][2] = G[0][2] * G[1][0] - G[0][0] * G[1][2];
    inv[2][0] = G[1][0] * G[2][1] - G[1][1] * G[2][0];
    inv[2][1] = G[0][1] * G[2][0] - G[0][0] * G[2][1];
    inv[2][2] = G[0][0] * G[1][1] - G[0][1] * G[1][0];
  }
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) inv[i][j] = inv[i][j] / det;
}

// jac: (M, D, Nq) physical coordinate m, parametric direction j.
// Outputs (each optional): det (Nq), invjac (D, M, Nq), coef (D, D, Nq).
template <int D>
__global__ void __launch_bounds__(256) geometry_kernel(int64_t nq, int M,
                                                       const double* __restrict__ jac,
                                                       double* __restrict__ det_out,
                                                       double* __restrict__ invjac_out,
                                                       double* __restrict__ coef_out,
                                                       int32_t* __restrict__ status) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nq;
       q += (int64_t)gridDim.x * blockDim.x) {
    double J[3][3];
    for (int m = 0; m < M; ++m)
#pragma unroll
      for (int j = 0; j < D; ++j) J[m][j] = jac[((int64_t)m * D + j) * nq + q];
    double G[3][3];
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) {
        double s = 0.0;
        for (int l = 0; l < M; ++l) s += J[l][i] * J[l][j];
        G[i][j] = s;
      }
    double inv[3][3], detG;
    inv_det<D>(G, inv, detG);
    // status bits: 1 = |det G| < 1e-14 (singular metric), 2 = det J <= 0 or NaN
    if (!(fabs(detG) >= 1e-14)) atomicOr(status, 1);
    const double dj = sqrt(detG);
    if (!(dj > 0.0)) atomicOr(status, 2);
    double P[3][3];  // J^+ = G^{-1} J^T : (D x M)
#pragma unroll
    for (int i = 0; i < D; ++i)
      for (int m = 0; m < M; ++m) {
        double s = 0.0;
#pragma unroll
        for (int l = 0; l < D; ++l) s += inv[i][l] * J[m][l];
        P[i][m] = s;
      }
    if (det_out) det_out[q] = dj;
    if (invjac_out)
#pragma unroll
      for (int i = 0; i < D; ++i)
        for (int m = 0; m < M; ++m) invjac_out[((int64_t)i * M + m) * nq + q] = P[i][m];
    if (coef_out)
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) {
          double s = 0.0;
          for (int l = 0; l < M; ++l) s += P[i][l] * P[j][l];
          coef_out[((int64_t)i * D + j) * nq + q] = s * dj;
        }
  }
}

}  // namespace iga

using namespace iga;

extern "C" {

iga_status iga_geometry_pointwise(int ndim, int ncoord, int64_t nq, const double* jac,
                                  double* det_out, double* invjac_out, double* coef_out,
                                  int32_t* status, iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(ndim >= 1 && ndim <= 3, "ndim %d out of range", ndim);
  IGA_CHECK_ARG(ncoord >= ndim && ncoord <= 3, "ncoord %d out of range", ncoord);
  IGA_CHECK_ARG(jac && status && nq >= 0, "null argument");
  if (nq == 0) return IGA_OK;
  int64_t blocks = ceil_div(nq, 256);
  if (blocks > 148 * 32) blocks = 148 * 32;
  cudaStream_t st = as_stream(stream);
  switch (ndim) {
    case 1:
      geometry_kernel<1><<<(unsigned)blocks, 256, 0, st>>>(nq, ncoord, jac, det_out, invjac_out,
                                                           coef_out, status);
      break;
    case 2:
      geometry_kernel<2><<<(unsigned)blocks, 256, 0, st>>>(nq, ncoord, jac, det_out, invjac_out,
                                                           coef_out, status);
      break;
    default:
      geometry_kernel<3><<<(unsigned)blocks, 256, 0, st>>>(nq, ncoord, jac, det_out, invjac_out,
                                                           coef_out, status);
  }
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

}  // extern "C"
