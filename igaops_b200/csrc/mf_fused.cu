// Host entry points of the fused matrix-free operator: layout, packing of the
// reference-layout coefficients, and the matvec launch.
#include <vector>

#include "mf_fused.cuh"

namespace iga {

static int pattern_nstream(int ndim, int op, int st, int sym) {
  const int sp = st ? ndim - 1 : ndim;
  switch (op) {
    case IGA_OP_MASS: return 1;
    case IGA_OP_STIFF: return sym ? sp * (sp + 1) / 2 : sp * sp;
    case IGA_OP_GRADU_V:
    case IGA_OP_U_GRADV: return sp;
    default: return -1;
  }
}

static iga_status check_plan(const iga_mf_plan* p) {
  IGA_CHECK_ARG(p, "null plan");
  IGA_CHECK_ARG(p->ndim == 2 || p->ndim == 3, "fused matvec supports ndim 2 or 3, got %d", p->ndim);
  IGA_CHECK_ARG(p->op >= IGA_OP_MASS && p->op <= IGA_OP_U_GRADV, "bad op %d", p->op);
  IGA_CHECK_ARG(p->spacetime == 0 || p->spacetime == 1, "bad spacetime flag");
  IGA_CHECK_ARG(p->time_test == 0 || p->time_test == 1, "time_test must be 0 or 1");
  IGA_CHECK_ARG(p->time_trial == 0 || p->time_trial == 1, "time_trial must be 0 or 1");
  const int S = pattern_nstream(p->ndim, p->op, p->spacetime, p->sym);
  IGA_CHECK_ARG(S == p->nstream && S >= 1 && S <= 9, "nstream %d does not match op (%d)",
                p->nstream, S);
  IGA_CHECK_ARG(p->nseg >= 1, "nseg must be >= 1");
  for (int d = 0; d < p->ndim; ++d) {
    IGA_CHECK_ARG(p->n[d] >= 1 && p->nq[d] >= 1, "empty direction %d", d);
    IGA_CHECK_ARG(p->trial[d].rows == p->nq[d] && p->trial[d].cols == p->n[d],
                  "trial band %d has shape %dx%d, expected %dx%d", d, p->trial[d].rows,
                  p->trial[d].cols, p->nq[d], p->n[d]);
    IGA_CHECK_ARG(p->testT[d].rows == p->nq[d] && p->testT[d].cols == p->n[d],
                  "testT band %d shape mismatch", d);
    IGA_CHECK_ARG(p->testR[d].rows == p->n[d] && p->testR[d].cols == p->nq[d],
                  "testR band %d shape mismatch", d);
    IGA_CHECK_ARG(p->trial[d].width == p->width && p->testT[d].width == p->width,
                  "band widths of direction %d differ from plan width %d", d, p->width);
    IGA_CHECK_ARG(p->testR[d].width == p->rwidth, "testR width mismatch in direction %d", d);
  }
  const int last = p->ndim - 1;
  IGA_CHECK_ARG(p->nseg <= p->nq[last], "nseg %d exceeds nq of the streamed direction", p->nseg);
  IGA_CHECK_ARG(p->face[0] >= 1 && (p->ndim == 2 || p->face[1] >= 1), "bad face");
  return IGA_OK;
}

static int64_t layout_elems(const iga_mf_plan* p, int dtype, int64_t* tile_off) {
  const int FX = p->face[0];
  const int FY = p->ndim == 3 ? p->face[1] : 1;
  const int tiles1 = (int)ceil_div(p->nq[0], FX);
  const int tiles2 = p->ndim == 3 ? (int)ceil_div(p->nq[1], FY) : 1;
  const int nlast = p->nq[p->ndim - 1];
  int64_t off = 0;
  for (int t2 = 0; t2 < tiles2; ++t2) {
    const int w2 = p->ndim == 3 ? std::min(FY, p->nq[1] - t2 * FY) : 1;
    for (int t1 = 0; t1 < tiles1; ++t1) {
      const int w1 = std::min(FX, p->nq[0] - t1 * FX);
      if (tile_off) tile_off[(int64_t)t2 * tiles1 + t1] = off;
      const int64_t cs = dtype == IGA_F64 ? chunk_stride_elems<double>(p->nstream, w1, w2)
                                          : chunk_stride_elems<float>(p->nstream, w1, w2);
      off += cs * nlast;
    }
  }
  return off;
}

// pack: thread per (stream, q) in reference order
template <typename Tin, typename Tout>
__global__ void __launch_bounds__(256) mf_pack_kernel(int ndim, int nq1, int nq2, int nq3, int FX,
                                                      int FY, int S, int tiles1,
                                                      const int64_t* __restrict__ tile_off,
                                                      SrcRows rows, const Tin* __restrict__ coefs,
                                                      int64_t ld, Tout* __restrict__ packed) {
  const int64_t Nq = (int64_t)nq1 * nq2 * (ndim == 3 ? nq3 : 1);
  const int64_t total = Nq * S;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int s = (int)(idx / Nq);
    const int64_t q = idx - (int64_t)s * Nq;
    const int q1 = (int)(q % nq1);
    const int64_t r = q / nq1;
    const Tout v = (Tout)coefs[(int64_t)rows.r[s] * ld + q];
    const int t1 = q1 / FX, l1 = q1 - t1 * FX;
    const int w1 = min(FX, nq1 - t1 * FX);
    int64_t off;
    if (ndim == 3) {
      const int q2 = (int)(r % nq2);
      const int q3 = (int)(r / nq2);
      const int t2 = q2 / FY, l2 = q2 - t2 * FY;
      const int w2 = min(FY, nq2 - t2 * FY);
      off = tile_off[(int64_t)t2 * tiles1 + t1] + (int64_t)q3 * chunk_stride_elems<Tout>(S, w1, w2) +
            (point_major3(S) ? ((int64_t)l2 * w1 + l1) * S + s
                             : (int64_t)s * w1 * w2 + (int64_t)l2 * w1 + l1);
    } else {
      const int q2 = (int)r;
      off = tile_off[t1] + (int64_t)q2 * chunk_stride_elems<Tout>(S, w1, 1) + (int64_t)s * w1 + l1;
    }
    packed[off] = v;
  }
}

// pack of point-major 3D chunks: one CTA per (face tile, q3) chunk, one
// thread per face point; each thread reads its point's streams (coalesced
// along q1 per stream) and writes them contiguously (the chunk is one
// contiguous run of the packed buffer)
template <typename Tin, typename Tout>
__global__ void __launch_bounds__(256) mf_pack3_pm_kernel(int nq1, int nq2, int FX, int FY, int S,
                                                          int tiles1,
                                                          const int64_t* __restrict__ tile_off,
                                                          SrcRows rows, const Tin* __restrict__ coefs,
                                                          int64_t ld, Tout* __restrict__ packed) {
  const int tile = blockIdx.x, q3 = blockIdx.y;
  const int t1 = tile % tiles1, t2 = tile / tiles1;
  const int w1 = min(FX, nq1 - t1 * FX), w2 = min(FY, nq2 - t2 * FY);
  const int l = threadIdx.x, l1 = l % FX, l2 = l / FX;
  if (l1 >= w1 || l2 >= w2) return;
  const int64_t q = ((int64_t)q3 * nq2 + t2 * FY + l2) * nq1 + t1 * FX + l1;
  Tout* dst = packed + tile_off[tile] + (int64_t)q3 * chunk_stride_elems<Tout>(S, w1, w2) +
              ((int64_t)l2 * w1 + l1) * S;
  for (int s = 0; s < S; ++s) dst[s] = (Tout)coefs[(int64_t)rows.r[s] * ld + q];
}

// step table rows of the last direction: B0, B1, W0T, W1T (W each), starts
template <typename T>
__global__ void mf_table_kernel(int nq, int W, int rlen, const int32_t* __restrict__ ts,
                                const T* __restrict__ b0, const T* __restrict__ b1,
                                const int32_t* __restrict__ ws, const T* __restrict__ w0,
                                const T* __restrict__ w1, T* __restrict__ table) {
  const int64_t total = (int64_t)nq * rlen;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int q = (int)(idx / rlen), j = (int)(idx - (int64_t)q * rlen);
    const int G = step_group<T>(W);
    const int grp = j / G, k = j - grp * G;
    T v = T(0);
    if (grp < 4) {
      if (k < W) {
        const T* src = grp == 0 ? b0 : grp == 1 ? b1 : grp == 2 ? w0 : w1;
        v = src[(int64_t)q * W + k];
      }
    } else if (j == 4 * G) {
      v = step_start_enc(ts[q], T(0));
    } else if (j == 4 * G + 1) {
      v = step_start_enc(ws[q], T(0));
    }
    table[idx] = v;
  }
}

template <typename T>
static void fill_args(FusedArgs<T>& a, const iga_mf_plan* p, const void* packed, const void* x,
                      void* y) {
  for (int d = 0; d < 3; ++d) {
    a.n[d] = d < p->ndim ? p->n[d] : 1;
    a.nq[d] = d < p->ndim ? p->nq[d] : 1;
    a.tstart[d] = d < p->ndim ? p->trial[d].start : nullptr;
    a.tB0[d] = d < p->ndim ? (const T*)p->trial[d].vals : nullptr;
    a.tB1[d] = d < p->ndim ? (const T*)p->trial_d1[d] : nullptr;
    a.wtstart[d] = d < p->ndim ? p->testT[d].start : nullptr;
    a.wT0[d] = d < p->ndim ? (const T*)p->testT[d].vals : nullptr;
    a.wT1[d] = d < p->ndim ? (const T*)p->testT_d1[d] : nullptr;
    a.rstart[d] = d < p->ndim ? p->testR[d].start : nullptr;
    a.wR0[d] = d < p->ndim ? (const T*)p->testR[d].vals : nullptr;
    a.wR1[d] = d < p->ndim ? (const T*)p->testR_d1[d] : nullptr;
  }
  a.W = p->width;
  a.RW = p->rwidth;
  a.tiles1 = (int)ceil_div(p->nq[0], p->face[0]);
  a.tiles2 = p->ndim == 3 ? (int)ceil_div(p->nq[1], p->face[1]) : 1;
  a.nseg = p->nseg;
  a.cmax1 = p->cmax[0];
  a.cmax2 = p->cmax[1];
  a.dmax1 = p->dmax[0];
  a.dmax2 = p->dmax[1];
  int64_t N = 1;
  for (int d = 0; d < p->ndim; ++d) N *= p->n[d];
  a.N = N;
  a.tile_off = p->tile_off;
  a.step_table = (const T*)p->step_table;
  a.rlen = step_row_len<T>(p->width);
  a.packed = (const T*)packed;
  a.x = (const T*)x;
  a.y = (T*)y;
  a.status = p->status;
  a.wait_test = p->wait_test;
}

template <typename T>
static iga_status launch_dispatch(const FusedArgs<T>& a, const LaunchInfo& li);

template <>
iga_status launch_dispatch<double>(const FusedArgs<double>& a, const LaunchInfo& li) {
#define IGA_W_CASES(D)                                  \
  switch (li.W) {                                       \
    case 3: return launch_mf##D##_f64_w3(a, li);        \
    case 4: return launch_mf##D##_f64_w4(a, li);        \
    case 5: return launch_mf##D##_f64_w5(a, li);        \
    case 6: return launch_mf##D##_f64_w6(a, li);        \
    default: break;                                     \
  }
  if (li.ndim == 3) { IGA_W_CASES(3) } else { IGA_W_CASES(2) }
#undef IGA_W_CASES
  set_error("no fused kernel for band width %d", li.W);
  return IGA_ERR_UNSUPPORTED;
}

template <>
iga_status launch_dispatch<float>(const FusedArgs<float>& a, const LaunchInfo& li) {
#define IGA_W_CASES(D)                                  \
  switch (li.W) {                                       \
    case 3: return launch_mf##D##_f32_w3(a, li);        \
    case 4: return launch_mf##D##_f32_w4(a, li);        \
    case 5: return launch_mf##D##_f32_w5(a, li);        \
    case 6: return launch_mf##D##_f32_w6(a, li);        \
    default: break;                                     \
  }
  if (li.ndim == 3) { IGA_W_CASES(3) } else { IGA_W_CASES(2) }
#undef IGA_W_CASES
  set_error("no fused kernel for band width %d", li.W);
  return IGA_ERR_UNSUPPORTED;
}

// shared memory of the multi-patch kernel for one patch of a pattern
template <typename T>
static size_t batch_smem(const iga_mf_plan* p, int rlen) {
  const int W = p->width, RW = p->rwidth;
  auto f = [&](auto pat) {
    using P = decltype(pat);
    return mf3d_smem_bytes<T, P>(kFace3X, kFace3Y, W, RW, rlen, p->cmax[0], p->cmax[1],
                                 p->dmax[0], p->dmax[1]);
  };
  switch (p->op) {
    case IGA_OP_MASS: return f(Pat<3, IGA_OP_MASS, 0, 0, 0, 0>{});
    case IGA_OP_STIFF:
      return p->sym ? f(Pat<3, IGA_OP_STIFF, 0, 0, 0, 1>{}) : f(Pat<3, IGA_OP_STIFF, 0, 0, 0, 0>{});
    case IGA_OP_GRADU_V: return f(Pat<3, IGA_OP_GRADU_V, 0, 0, 0, 0>{});
    default: return f(Pat<3, IGA_OP_U_GRADV, 0, 0, 0, 0>{});
  }
}

static inline int64_t align256(int64_t b) { return (b + 255) / 256 * 256; }

template <typename T>
static int64_t batch_table_bytes(int npatch) {
  return align256((int64_t)npatch * sizeof(FusedArgs<T>)) + align256((int64_t)(npatch + 1) * 4) +
         (int64_t)npatch * 8;
}

template <typename T>
static iga_status batch_prepare(const iga_mf_plan* plans, int npatch, const void* const* packed,
                                const int64_t* offsets, void* table, int32_t* total_ctas,
                                int64_t* smem_bytes) {
  std::vector<FusedArgs<T>> args((size_t)npatch);
  std::vector<int32_t> cta0((size_t)npatch + 1);
  std::vector<int64_t> offs((size_t)npatch);
  int64_t total = 0;
  size_t smem = 0;
  const iga_mf_plan& p0 = plans[0];
  for (int i = 0; i < npatch; ++i) {
    const iga_mf_plan* p = plans + i;
    iga_status rc = check_plan(p);
    if (rc) return rc;
    IGA_CHECK_ARG(p->ndim == 3 && !p->spacetime, "patch %d: multi-patch matvec covers 3D space operators", i);
    IGA_CHECK_ARG(p->op == p0.op && p->sym == p0.sym && p->width == p0.width &&
                      p->face[0] == kFace3X && p->face[1] == kFace3Y,
                  "patch %d: operator, symmetry, band width and face must match patch 0", i);
    IGA_CHECK_ARG(packed[i] && ((uintptr_t)packed[i] & 15) == 0 && p->step_table,
                  "patch %d: packed coefficients (16-byte aligned) and step table required", i);
    fill_args<T>(args[i], p, packed[i], nullptr, nullptr);
    IGA_CHECK_ARG(offsets[i] >= 0, "patch %d: negative offset", i);
    offs[i] = offsets[i];
    cta0[i] = (int32_t)total;
    total += (int64_t)args[i].tiles1 * args[i].tiles2 * args[i].nseg;
    smem = std::max(smem, batch_smem<T>(p, args[i].rlen));
  }
  IGA_CHECK_ARG(total < (1ll << 31), "too many CTAs (%lld)", (long long)total);
  cta0[npatch] = (int32_t)total;
  char* t = (char*)table;
  const int64_t a_bytes = align256((int64_t)npatch * sizeof(FusedArgs<T>));
  const int64_t c_bytes = align256((int64_t)(npatch + 1) * 4);
  IGA_CUDA_TRY(cudaMemcpy(t, args.data(), npatch * sizeof(FusedArgs<T>), cudaMemcpyHostToDevice));
  IGA_CUDA_TRY(cudaMemcpy(t + a_bytes, cta0.data(), (npatch + 1) * 4, cudaMemcpyHostToDevice));
  IGA_CUDA_TRY(cudaMemcpy(t + a_bytes + c_bytes, offs.data(), npatch * 8, cudaMemcpyHostToDevice));
  *total_ctas = (int32_t)total;
  *smem_bytes = (int64_t)smem;
  return IGA_OK;
}

template <typename T>
static iga_status batch_dispatch(const BatchLaunch& b, const T* x, T* y);

template <>
iga_status batch_dispatch<double>(const BatchLaunch& b, const double* x, double* y) {
  switch (b.W) {
    case 3: return launch_mf3_batch_f64_w3(b, x, y);
    case 4: return launch_mf3_batch_f64_w4(b, x, y);
    case 5: return launch_mf3_batch_f64_w5(b, x, y);
    case 6: return launch_mf3_batch_f64_w6(b, x, y);
    default: break;
  }
  set_error("no multi-patch kernel for band width %d", b.W);
  return IGA_ERR_UNSUPPORTED;
}

template <>
iga_status batch_dispatch<float>(const BatchLaunch& b, const float* x, float* y) {
  switch (b.W) {
    case 3: return launch_mf3_batch_f32_w3(b, x, y);
    case 4: return launch_mf3_batch_f32_w4(b, x, y);
    case 5: return launch_mf3_batch_f32_w5(b, x, y);
    case 6: return launch_mf3_batch_f32_w6(b, x, y);
    default: break;
  }
  set_error("no multi-patch kernel for band width %d", b.W);
  return IGA_ERR_UNSUPPORTED;
}

}  // namespace iga

using namespace iga;

extern "C" {

iga_status iga_mf_batch_table_bytes(int dtype, int npatch, int64_t* bytes) {
  clear_error();
  IGA_CHECK_ARG(npatch >= 1 && bytes, "bad argument");
  if (dtype == IGA_F64) *bytes = batch_table_bytes<double>(npatch);
  else if (dtype == IGA_F32) *bytes = batch_table_bytes<float>(npatch);
  else {
    set_error("dtype %d not supported", dtype);
    return IGA_ERR_UNSUPPORTED;
  }
  return IGA_OK;
}

iga_status iga_mf_batch_prepare(const iga_mf_plan* plans, int npatch, int dtype,
                                const void* const* packed, const int64_t* offsets, void* table,
                                int32_t* total_ctas, int64_t* smem_bytes) {
  clear_error();
  IGA_CHECK_ARG(plans && npatch >= 1 && packed && offsets && table && total_ctas && smem_bytes,
                "null argument");
  IGA_CHECK_ARG(((uintptr_t)table & 255) == 0, "table must be 256-byte aligned");
  IGA_CHECK_ARG(plans[0].width >= 3 && plans[0].width <= 6, "band width %d", plans[0].width);
  if (dtype == IGA_F64)
    return batch_prepare<double>(plans, npatch, packed, offsets, table, total_ctas, smem_bytes);
  if (dtype == IGA_F32)
    return batch_prepare<float>(plans, npatch, packed, offsets, table, total_ctas, smem_bytes);
  set_error("dtype %d not supported", dtype);
  return IGA_ERR_UNSUPPORTED;
}

iga_status iga_mf_batch_matvec(const iga_mf_plan* plan0, int dtype, int npatch, const void* table,
                               int32_t total_ctas, int64_t smem_bytes, const void* x, void* y,
                               int64_t ntot, int zero_y, const int32_t* skip,
                               iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(plan0 && table && x && y && npatch >= 1 && total_ctas >= 1 && ntot >= 0,
                "bad argument");
  cudaStream_t st = as_stream(stream);
  const size_t esz = dtype == IGA_F64 ? 8 : 4;
  if (zero_y) IGA_CUDA_TRY(cudaMemsetAsync(y, 0, (size_t)ntot * esz, st));
  BatchLaunch b;
  b.op = plan0->op;
  b.sym = plan0->sym;
  b.W = plan0->width;
  b.npatch = npatch;
  b.total_ctas = total_ctas;
  b.smem = (size_t)smem_bytes;
  const char* t = (const char*)table;
  const int64_t a_bytes =
      align256((int64_t)npatch * (dtype == IGA_F64 ? sizeof(FusedArgs<double>) : sizeof(FusedArgs<float>)));
  const int64_t c_bytes = align256((int64_t)(npatch + 1) * 4);
  b.args = t;
  b.cta0 = (const int32_t*)(t + a_bytes);
  b.offs = (const int64_t*)(t + a_bytes + c_bytes);
  b.skip = skip;
  b.stream = st;
  if (dtype == IGA_F64) return batch_dispatch<double>(b, (const double*)x, (double*)y);
  if (dtype == IGA_F32) return batch_dispatch<float>(b, (const float*)x, (float*)y);
  set_error("dtype %d not supported", dtype);
  return IGA_ERR_UNSUPPORTED;
}

iga_status iga_mf_layout(const iga_mf_plan* plan, int dtype, int64_t* elems,
                         int64_t* tile_off_host) {
  clear_error();
  iga_status rc = check_plan(plan);
  if (rc) return rc;
  IGA_CHECK_ARG(dtype == IGA_F64 || dtype == IGA_F32, "dtype %d not supported", dtype);
  IGA_CHECK_ARG(elems, "null elems");
  *elems = layout_elems(plan, dtype, tile_off_host);
  return IGA_OK;
}

iga_status iga_mf_table(const iga_mf_plan* plan, int dtype, int64_t* elems, void* table,
                        iga_stream stream) {
  clear_error();
  iga_status rc = check_plan(plan);
  if (rc) return rc;
  IGA_CHECK_ARG(elems, "null elems");
  IGA_CHECK_ARG(dtype == IGA_F64 || dtype == IGA_F32, "dtype %d not supported", dtype);
  const int last = plan->ndim - 1;
  const int W = plan->width;
  const int nq = plan->nq[last];
  const int rlen = dtype == IGA_F64 ? step_row_len<double>(W) : step_row_len<float>(W);
  *elems = (int64_t)nq * rlen;
  if (!table) return IGA_OK;
  const iga_band& tb = plan->trial[last];
  const iga_band& wb = plan->testT[last];
  IGA_CHECK_ARG(tb.start && tb.vals && plan->trial_d1[last] && wb.start && wb.vals &&
                    plan->testT_d1[last],
                "band arrays of the last direction missing");
  const unsigned g = (unsigned)std::min<int64_t>(ceil_div(*elems, 256), 148 * 8);
  cudaStream_t st = as_stream(stream);
  if (dtype == IGA_F64)
    mf_table_kernel<double><<<g, 256, 0, st>>>(
        nq, W, rlen, tb.start, (const double*)tb.vals, (const double*)plan->trial_d1[last],
        wb.start, (const double*)wb.vals, (const double*)plan->testT_d1[last], (double*)table);
  else
    mf_table_kernel<float><<<g, 256, 0, st>>>(
        nq, W, rlen, tb.start, (const float*)tb.vals, (const float*)plan->trial_d1[last],
        wb.start, (const float*)wb.vals, (const float*)plan->testT_d1[last], (float*)table);
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

iga_status iga_mf_pack(const iga_mf_plan* plan, int dtype_in, const void* coefs, int64_t ld,
                       int dtype_out, void* packed, iga_stream stream) {
  clear_error();
  iga_status rc = check_plan(plan);
  if (rc) return rc;
  IGA_CHECK_ARG(coefs && packed && plan->tile_off, "null pointer");
  IGA_CHECK_ARG(dtype_in == IGA_F64 || dtype_in == IGA_F32, "dtype_in %d", dtype_in);
  IGA_CHECK_ARG(dtype_out == IGA_F64 || dtype_out == IGA_F32, "dtype_out %d", dtype_out);
  const int S = plan->nstream;
  SrcRows rows;
  for (int s = 0; s < 9; ++s) {
    rows.r[s] = plan->src_row[s];
    if (s < S) IGA_CHECK_ARG(rows.r[s] >= 0, "src_row[%d] negative", s);
  }
  cudaStream_t st = as_stream(stream);
  const int64_t elems = layout_elems(plan, dtype_out, nullptr);
  const size_t esz = dtype_out == IGA_F64 ? 8 : 4;
  IGA_CUDA_TRY(cudaMemsetAsync(packed, 0, (size_t)elems * esz, st));
  int64_t Nq = 1;
  for (int d = 0; d < plan->ndim; ++d) Nq *= plan->nq[d];
  IGA_CHECK_ARG(ld >= Nq, "ld %lld smaller than Nq %lld", (long long)ld, (long long)Nq);
  int64_t blocks = ceil_div(Nq * S, 256);
  if (blocks > 148 * 64) blocks = 148 * 64;
  const int nq3 = plan->ndim == 3 ? plan->nq[2] : 1;
  const int FY = plan->ndim == 3 ? plan->face[1] : 1;
  const int tiles1 = (int)ceil_div(plan->nq[0], plan->face[0]);
  const bool pm3 = plan->ndim == 3 && point_major3(S) && plan->face[0] * FY <= 256;
  const int tiles2 = plan->ndim == 3 ? (int)ceil_div(plan->nq[1], FY) : 1;
  IGA_CHECK_ARG(!pm3 || nq3 <= 65535, "streamed direction of %d points exceeds the grid", nq3);
#define IGA_PACK(TI, TO)                                                                      \
  do {                                                                                        \
    if (pm3)                                                                                  \
      mf_pack3_pm_kernel<TI, TO><<<dim3((unsigned)(tiles1 * tiles2), (unsigned)nq3),         \
                                   (unsigned)(plan->face[0] * FY), 0, st>>>(                  \
          plan->nq[0], plan->nq[1], plan->face[0], FY, S, tiles1, plan->tile_off, rows,       \
          (const TI*)coefs, ld, (TO*)packed);                                                 \
    else                                                                                      \
      mf_pack_kernel<TI, TO><<<(unsigned)blocks, 256, 0, st>>>(                               \
          plan->ndim, plan->nq[0], plan->nq[1], nq3, plan->face[0], FY, S, tiles1,            \
          plan->tile_off, rows, (const TI*)coefs, ld, (TO*)packed);                           \
  } while (0)
  if (dtype_in == IGA_F64 && dtype_out == IGA_F64) IGA_PACK(double, double);
  else if (dtype_in == IGA_F64 && dtype_out == IGA_F32) IGA_PACK(double, float);
  else if (dtype_in == IGA_F32 && dtype_out == IGA_F64) IGA_PACK(float, double);
  else IGA_PACK(float, float);
#undef IGA_PACK
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

iga_status iga_mf_matvec(const iga_mf_plan* plan, int dtype, const void* packed, int64_t ncols,
                         const void* x, void* y, iga_stream stream) {
  clear_error();
  iga_status rc = check_plan(plan);
  if (rc) return rc;
  IGA_CHECK_ARG(packed && x && y && plan->tile_off, "null pointer");
  IGA_CHECK_ARG(ncols >= 1 && ncols <= 65535, "ncols %lld out of range", (long long)ncols);
  IGA_CHECK_ARG(((uintptr_t)packed & 15) == 0, "packed coefficients must be 16-byte aligned");
  IGA_CHECK_ARG(plan->width >= 3 && plan->width <= 6,
                "fused matvec supports band width 3..6 (degree 2..5), got %d", plan->width);
  cudaStream_t st = as_stream(stream);
  int64_t N = 1;
  for (int d = 0; d < plan->ndim; ++d) N *= plan->n[d];
  const size_t esz = dtype == IGA_F64 ? 8 : 4;
  IGA_CUDA_TRY(cudaMemsetAsync(y, 0, (size_t)N * ncols * esz, st));
  LaunchInfo li;
  li.ndim = plan->ndim;
  li.op = plan->op;
  li.st = plan->spacetime;
  li.tt = plan->time_test;
  li.tr = plan->time_trial;
  li.sym = plan->sym;
  li.W = plan->width;
  li.FX = plan->face[0];
  li.FY = plan->ndim == 3 ? plan->face[1] : 1;
  li.NST = kStages;
  li.ncols = ncols;
  li.stream = st;
  if (dtype == IGA_F64) {
    FusedArgs<double> a;
    fill_args<double>(a, plan, packed, x, y);
    return launch_dispatch<double>(a, li);
  }
  if (dtype == IGA_F32) {
    FusedArgs<float> a;
    fill_args<float>(a, plan, packed, x, y);
    return launch_dispatch<float>(a, li);
  }
  set_error("dtype %d not supported by iga_mf_matvec", dtype);
  return IGA_ERR_UNSUPPORTED;
}

}  // extern "C"
