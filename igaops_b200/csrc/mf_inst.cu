// Instantiation unit of the fused matrix-free kernels.  The build compiles
// this file once per (IGA_INST_D, IGA_INST_T, IGA_INST_W) so that the many
// template instances build in parallel.
#include "mf_fused.cuh"

#ifndef IGA_INST_D
#define IGA_INST_D 3
#define IGA_INST_TN f64
#define IGA_INST_T double
#define IGA_INST_W 4
#endif

namespace iga {

template <typename T, int D, int W, class P>
static iga_status launch_pat(const FusedArgs<T>& a, const LaunchInfo& li) {
  const dim3 grid((unsigned)(a.tiles1 * a.tiles2 * a.nseg), (unsigned)li.ncols);
  if constexpr (D == 3) {
    constexpr int FX = kFace3X, FY = kFace3Y;
    if (li.FX != FX || li.FY != FY) {
      set_error("3D fused kernels are compiled for a %dx%d face, plan has %dx%d", FX, FY, li.FX,
                li.FY);
      return IGA_ERR_UNSUPPORTED;
    }
    if (!a.step_table || a.rlen != step_row_len<T>(W)) {
      set_error("3D fused kernel needs the step table of the plan (iga_mf_table)");
      return IGA_ERR_INVALID_ARG;
    }
    const size_t smem =
        mf3d_smem_bytes<T, P>(FX, FY, W, a.RW, a.rlen, a.cmax1, a.cmax2, a.dmax1, a.dmax2);
    if (smem > 227 * 1024) {
      set_error("fused 3D kernel needs %zu bytes of shared memory (tile ranges %d/%d/%d)", smem,
                a.cmax1, a.cmax2, a.dmax2);
      return IGA_ERR_UNSUPPORTED;
    }
    auto kern = mf3d_kernel<T, FX, FY, W, P>;
    static size_t configured = 48 * 1024;
    if (smem > configured) {
      IGA_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem));
      configured = smem;
    }
    kern<<<grid, FX * FY, smem, li.stream>>>(a);
  } else {
    constexpr int FX = kFace2X;
    constexpr int NST = kStages;
    if (li.FX != FX) {
      set_error("2D fused kernels are compiled for a face of %d, plan has %d", FX, li.FX);
      return IGA_ERR_UNSUPPORTED;
    }
    const size_t smem = mf2d_smem_bytes<T>(P::S, FX, NST);
    auto kern = mf2d_kernel<T, FX, W, NST, P>;
    static size_t configured = 48 * 1024;
    if (smem > configured) {
      IGA_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem));
      configured = smem;
    }
    kern<<<grid, FX, smem, li.stream>>>(a);
  }
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

template <typename T, int D, int W>
static iga_status launch_w(const FusedArgs<T>& a, const LaunchInfo& li) {
  if (!li.st) {
    switch (li.op) {
      case IGA_OP_MASS: return launch_pat<T, D, W, Pat<D, IGA_OP_MASS, 0, 0, 0, 0>>(a, li);
      case IGA_OP_STIFF:
        return li.sym ? launch_pat<T, D, W, Pat<D, IGA_OP_STIFF, 0, 0, 0, 1>>(a, li)
                      : launch_pat<T, D, W, Pat<D, IGA_OP_STIFF, 0, 0, 0, 0>>(a, li);
      case IGA_OP_GRADU_V: return launch_pat<T, D, W, Pat<D, IGA_OP_GRADU_V, 0, 0, 0, 0>>(a, li);
      case IGA_OP_U_GRADV: return launch_pat<T, D, W, Pat<D, IGA_OP_U_GRADV, 0, 0, 0, 0>>(a, li);
      default: break;
    }
  } else if constexpr (D == 3) {
    if (li.op == IGA_OP_MASS) {
      switch (li.tt * 2 + li.tr) {
        case 0: return launch_pat<T, D, W, Pat<D, IGA_OP_MASS, 1, 0, 0, 0>>(a, li);
        case 1: return launch_pat<T, D, W, Pat<D, IGA_OP_MASS, 1, 0, 1, 0>>(a, li);
        case 2: return launch_pat<T, D, W, Pat<D, IGA_OP_MASS, 1, 1, 0, 0>>(a, li);
        case 3: return launch_pat<T, D, W, Pat<D, IGA_OP_MASS, 1, 1, 1, 0>>(a, li);
        default: break;
      }
    } else if (li.op == IGA_OP_STIFF && li.tt == 0 && li.tr == 0) {
      return li.sym ? launch_pat<T, D, W, Pat<D, IGA_OP_STIFF, 1, 0, 0, 1>>(a, li)
                    : launch_pat<T, D, W, Pat<D, IGA_OP_STIFF, 1, 0, 0, 0>>(a, li);
    }
  }
  set_error("no fused kernel for op %d (spacetime %d, time ders %d/%d) in %dD", li.op, li.st,
            li.tt, li.tr, D);
  return IGA_ERR_UNSUPPORTED;
}

template <typename T, int W, class P>
static iga_status launch_pat_batch(const BatchLaunch& b, const T* x, T* y) {
  constexpr int FX = kFace3X, FY = kFace3Y;
  if (b.smem > 227 * 1024) {
    set_error("multi-patch fused kernel needs %zu bytes of shared memory", b.smem);
    return IGA_ERR_UNSUPPORTED;
  }
  auto kern = mf3d_batch_kernel<T, FX, FY, W, P>;
  static size_t configured = 48 * 1024;
  if (b.smem > configured) {
    IGA_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)b.smem));
    configured = b.smem;
  }
  kern<<<(unsigned)b.total_ctas, FX * FY, b.smem, b.stream>>>(
      (const FusedArgs<T>*)b.args, b.cta0, b.npatch, b.offs, x, y, b.skip);
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

template <typename T, int W>
static iga_status launch_w_batch(const BatchLaunch& b, const T* x, T* y) {
  switch (b.op) {
    case IGA_OP_MASS: return launch_pat_batch<T, W, Pat<3, IGA_OP_MASS, 0, 0, 0, 0>>(b, x, y);
    case IGA_OP_STIFF:
      return b.sym ? launch_pat_batch<T, W, Pat<3, IGA_OP_STIFF, 0, 0, 0, 1>>(b, x, y)
                   : launch_pat_batch<T, W, Pat<3, IGA_OP_STIFF, 0, 0, 0, 0>>(b, x, y);
    case IGA_OP_GRADU_V:
      return launch_pat_batch<T, W, Pat<3, IGA_OP_GRADU_V, 0, 0, 0, 0>>(b, x, y);
    case IGA_OP_U_GRADV:
      return launch_pat_batch<T, W, Pat<3, IGA_OP_U_GRADV, 0, 0, 0, 0>>(b, x, y);
    default: break;
  }
  set_error("no multi-patch fused kernel for op %d", b.op);
  return IGA_ERR_UNSUPPORTED;
}

#if IGA_INST_D == 3
#define IGA_BCAT_(b, c) launch_mf3_batch_##b##_w##c
#define IGA_BNAME(TN, W) IGA_BCAT_(TN, W)
iga_status IGA_BNAME(IGA_INST_TN, IGA_INST_W)(const BatchLaunch& b, const IGA_INST_T* x,
                                              IGA_INST_T* y) {
  return launch_w_batch<IGA_INST_T, IGA_INST_W>(b, x, y);
}
#endif

#define IGA_CAT_(a, b, c, d) launch_mf##a##_##b##_w##c
#define IGA_NAME(D, TN, W) IGA_CAT_(D, TN, W, 0)
iga_status IGA_NAME(IGA_INST_D, IGA_INST_TN, IGA_INST_W)(const FusedArgs<IGA_INST_T>& a,
                                                          const LaunchInfo& li) {
  return launch_w<IGA_INST_T, IGA_INST_D, IGA_INST_W>(a, li);
}

}  // namespace iga
