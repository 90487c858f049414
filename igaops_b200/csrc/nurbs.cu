// Coefficient streams of the rational (NURBS) matrix-free operators.
//
// NurbsOperations.compute_mf_scalar_* (src/igaops/operators/nurbs_ops.py:
// 320-463) apply the B-spline operators to the weighted input w_c * x and
// scale the result by w_c again, with the per-point coefficients replaced by
// terms built from the interpolated weight W(q) = sum_c N_c(q) w_c and its
// parametric gradient dW(q) (nurbs_ops.py:14-62): with w = 1/W and
// z_k = dW_k * w^2,
//   mass                : c w^2
//   stiffness           : C_ij w^2  (gradu_gradv)
//                         + sum_ij C_ij z_i z_j            (u_v)
//                         - sum_i C_ij z_i w  for each j   (u_gradv)
//                         - sum_j C_ij z_j w  for each i   (gradu_v)
//   gradu_v / u_gradv   : c_i w^2 (same operator) - sum_i c_i z_i w (u_v)
// This kernel computes all streams of one operator in one pass over the
// quadrature points (one thread per point, grid-stride); the operator terms
// then run as fused matrix-free kernels.
#include "common.cuh"

namespace iga {

template <int SP, int OP>
__global__ void __launch_bounds__(256)
    nurbs_coef_kernel(int64_t nq, const double* __restrict__ c, const double* __restrict__ wq,
                      const double* __restrict__ dwq, double* __restrict__ out_main,
                      double* __restrict__ out_uv, double* __restrict__ out_ug,
                      double* __restrict__ out_gu, int32_t* __restrict__ status) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nq;
       q += (int64_t)gridDim.x * blockDim.x) {
    const double W = wq[q];
    if (!(W != 0.0)) atomicOr(status, 1);
    const double w = 1.0 / W;
    const double w2 = w * w;
    if (OP == IGA_OP_MASS) {
      out_main[q] = c[q] * w2;
      continue;
    }
    double z[SP];
#pragma unroll
    for (int k = 0; k < SP; ++k) z[k] = dwq[(int64_t)k * nq + q] * w2;
    if (OP == IGA_OP_STIFF) {
      double s = 0.0, h[SP], g[SP];
#pragma unroll
      for (int k = 0; k < SP; ++k) h[k] = g[k] = 0.0;
#pragma unroll
      for (int i = 0; i < SP; ++i)
#pragma unroll
        for (int j = 0; j < SP; ++j) {
          const double cij = c[(int64_t)(i * SP + j) * nq + q];
          out_main[(int64_t)(i * SP + j) * nq + q] = cij * w2;
          s += cij * z[i] * z[j];
          h[j] += cij * z[i];
          g[i] += cij * z[j];
        }
      out_uv[q] = s;
#pragma unroll
      for (int k = 0; k < SP; ++k) {
        out_ug[(int64_t)k * nq + q] = h[k] * w;
        out_gu[(int64_t)k * nq + q] = g[k] * w;
      }
    } else {
      double s = 0.0;
#pragma unroll
      for (int i = 0; i < SP; ++i) {
        const double ci = c[(int64_t)i * nq + q];
        out_main[(int64_t)i * nq + q] = ci * w2;
        s += ci * z[i];
      }
      out_uv[q] = s * w;
    }
  }
}

template <int SP>
void launch_nurbs(int op, unsigned blocks, cudaStream_t st, int64_t nq, const double* c,
                  const double* wq, const double* dwq, double* m, double* uv, double* ug,
                  double* gu, int32_t* status) {
  switch (op) {
    case IGA_OP_MASS:
      nurbs_coef_kernel<SP, IGA_OP_MASS><<<blocks, 256, 0, st>>>(nq, c, wq, dwq, m, uv, ug, gu,
                                                                  status);
      break;
    case IGA_OP_STIFF:
      nurbs_coef_kernel<SP, IGA_OP_STIFF><<<blocks, 256, 0, st>>>(nq, c, wq, dwq, m, uv, ug, gu,
                                                                   status);
      break;
    default:
      nurbs_coef_kernel<SP, IGA_OP_GRADU_V><<<blocks, 256, 0, st>>>(nq, c, wq, dwq, m, uv, ug,
                                                                     gu, status);
  }
}

}  // namespace iga

using namespace iga;

extern "C" {

iga_status iga_nurbs_coefficients(int op, int sp, int64_t nq, const double* coef,
                                  const double* wq, const double* dwq, double* out_main,
                                  double* out_uv, double* out_ug, double* out_gu,
                                  int32_t* status, iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(op >= IGA_OP_MASS && op <= IGA_OP_U_GRADV, "unknown operator %d", op);
  IGA_CHECK_ARG(sp >= 1 && sp <= 3, "spatial dimension %d out of range", sp);
  IGA_CHECK_ARG(nq >= 0 && coef && wq && out_main && status, "null argument");
  IGA_CHECK_ARG(op == IGA_OP_MASS || (dwq && out_uv), "null weight gradient or output");
  IGA_CHECK_ARG(op != IGA_OP_STIFF || (out_ug && out_gu), "null stiffness output");
  if (nq == 0) return IGA_OK;
  int64_t blocks = ceil_div(nq, 256);
  if (blocks > 148 * 32) blocks = 148 * 32;
  cudaStream_t st = as_stream(stream);
  if (sp == 1)
    launch_nurbs<1>(op, (unsigned)blocks, st, nq, coef, wq, dwq, out_main, out_uv, out_ug,
                    out_gu, status);
  else if (sp == 2)
    launch_nurbs<2>(op, (unsigned)blocks, st, nq, coef, wq, dwq, out_main, out_uv, out_ug,
                    out_gu, status);
  else
    launch_nurbs<3>(op, (unsigned)blocks, st, nq, coef, wq, dwq, out_main, out_uv, out_ug,
                    out_gu, status);
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

}  // extern "C"
