// Fast-diagonalisation apply on the 5th-generation tensor cores (tcgen05).
//
// P^{-1} v = (U_3 x U_2 x U_1) Lambda^{-1} (U_3 x U_2 x U_1)^T v on the free
// box (SpaceFD.apply, src/igaops/fastdiag/utils/space_precond.py:273-320) is
// 2*d mode products with dense m x m eigenvector matrices.  Each mode product
// here is one GEMM
//     D[row][a] = sum_k T[row][k] * B[k][a]
// whose data operand T is K-major: every GEMM stores its output with the
// tensor dims rotated (the contracted dim becomes the slowest, the next
// contraction dim the fastest), so after d products the order is natural
// again.  Operands are BF16 in shared memory (no-swizzle canonical UMMA
// layout), the accumulator is FP32 in tensor memory (TMEM); one CTA of 4
// warps owns 128 rows and the whole N (= m <= 256):
//   * warps stage the A tile (128 rows x Kp) with 16-byte vector loads, or
//     gather it from the FP32/FP64 input vector (first product);
//   * thread 0 brings the pre-tiled B image with one TMA bulk copy, issues
//     Kp/16 tcgen05.mma (M=128, N=Np, K=16) and tcgen05.commit;
//   * each warp reads its 32 TMEM lanes (tcgen05.ld 32x32b) and stores the
//     rotated output as BF16 (optionally times 1/Lambda), or scatters the
//     final product into the output vector.
#include <vector>

#include "common.cuh"

#include <cuda_bf16.h>

namespace iga {

namespace tc {

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  // SWIZZLE_NONE canonical layout; version 1 (sm_100) at bit 46
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: BF16 x BF16 -> F32, both K-major
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void mma_bf16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
      : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Programmatic dependent launch: products 2..6 of an apply are launched
// while the previous product still runs.  A CTA signals that the next
// product may be scheduled once it holds its tensor memory (so a CTA that
// can still block in tcgen05.alloc always belongs to the newest grid, and
// the older grids never wait on it), and waits for the previous product's
// completion before it reads any data that product writes.
__device__ __forceinline__ void launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void wait_prerequisites() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

}  // namespace tc

// Threads of a product CTA: 8 warps; warps w and w + 4 share TMEM lanes
// 32 (w mod 4) .. +31 and split the output columns in 16-column chunks.
constexpr int kTcThreads = 256;

// Output columns of a product are split over two CTAs per 128-row tile
// (the halves' widths multiples of 16, as tcgen05.mma with M = 128 needs),
// so that the MMA chain and the epilogue on a product's critical path are
// half as long and the products run on twice the CTAs.
__host__ __device__ __forceinline__ int tc_nsplit(int Np) { return Np >= 32 ? 2 : 1; }
__host__ __device__ __forceinline__ int tc_first_half(int Np) { return (Np / 16 + 1) / 2 * 16; }

// Gathers the CTA's 128 x Kp A tile (rows (i3, i2) of the free box, k = i1)
// from the input vector into the canonical K-major BF16 layout, in which
// the 8 elements (row r, k = 8 kc .. 8 kc + 7) are the 16 bytes at
// kc * 2048 + r * 16.  rowbase[r] is the vector index of (row r, k = 0).
// Thread t owns row t mod 128 and one half of its chunks, so a warp's
// 16-byte stores cover 512 contiguous bytes (no bank conflicts).  A row's
// elements are read as the aligned 16-byte blocks that hold them (VW
// elements each; every block read holds an element of the row, so it lies
// in memory the row's own elements occupy), VW chunks per round from a
// register window of 9 blocks shifted by the row's misalignment.  Padding
// columns k >= m0 and rows r >= nvalid are written as zeros.
template <typename TX>
__device__ __forceinline__ void gather_tile(const TX* __restrict__ xp, const int64_t* rowbase,
                                            int nvalid, int Kp, int m0, __nv_bfloat16* As,
                                            int tid) {
  constexpr int VW = 16 / (int)sizeof(TX);  // elements per 16-byte block: 4 or 2
  constexpr int G = VW;                     // chunks per round: G * 8 / VW = 8 blocks
  constexpr int NW = 9;                     // blocks in the window (+1 for misalignment)
  const int r = tid & 127;
  const int nkc = Kp / 8, halfc = (nkc + 1) / 2;
  const int kc0 = (tid >> 7) ? halfc : 0, kc1 = (tid >> 7) ? nkc : halfc;
  unsigned char* rowp = reinterpret_cast<unsigned char*>(As) + (size_t)r * 16;
  const int64_t b = r < nvalid ? rowbase[r] : -1;
  uintptr_t a16 = 0;
  int lead = 0, qlast = -1;
  if (b >= 0) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(xp + b);
    a16 = a & ~(uintptr_t)15;
    lead = (int)((a & 15) / sizeof(TX));
    qlast = (lead + m0 - 1) / VW;  // last block holding an element of the row
  }
  for (int kg = kc0; kg < kc1; kg += G) {
    // window: blocks q0 .. q0 + NW - 1, element k = 8 kg at position p0
    const int e0 = lead + 8 * kg;
    const int q0 = e0 / VW, p0 = e0 - q0 * VW;
    TX w[NW * VW];
#pragma unroll
    for (int t = 0; t < NW; ++t) {
      uint4 v = make_uint4(0, 0, 0, 0);
      if (b >= 0 && q0 + t <= qlast)
        v = __ldg(reinterpret_cast<const uint4*>(a16 + (uintptr_t)(q0 + t) * 16));
      const TX* pv = reinterpret_cast<const TX*>(&v);
#pragma unroll
      for (int i = 0; i < VW; ++i) w[t * VW + i] = pv[i];
    }
    // w[i] <- w[i + p0] (p0 < VW), one select per bit of p0
#pragma unroll
    for (int sh = VW / 2; sh >= 1; sh /= 2) {
      const bool on = (p0 & sh) != 0;
#pragma unroll
      for (int i = 0; i + sh < NW * VW; ++i) w[i] = on ? w[i + sh] : w[i];
    }
#pragma unroll
    for (int c = 0; c < G; ++c) {
      const int kc = kg + c;
      if (kc >= kc1) break;
      uint32_t pk[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int k = 8 * kc + 2 * j;
        const float lo = (b >= 0 && k < m0) ? (float)w[8 * c + 2 * j] : 0.f;
        const float hi = (b >= 0 && k + 1 < m0) ? (float)w[8 * c + 2 * j + 1] : 0.f;
        const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
        pk[j] = *reinterpret_cast<const uint32_t*>(&h);
      }
      *reinterpret_cast<uint4*>(rowp + (size_t)kc * 2048) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    }
  }
}


// one mode product
struct TcGemm {
  // rows and their split into (r_slow, r_fast): row = r_slow * rfast + r_fast
  int32_t R, rfast;
  int32_t Kp;      // padded contraction length (multiple of 16)
  int32_t N, Np;   // outputs per row (m of this direction) and its padding
  int32_t kpn;     // padded fastest length of the output tensor
  // A source
  const __nv_bfloat16* A;  // [R][Kp] (mode 0)
  // gather (first product): A[row][k] = x[box(row, k)]
  const void* x;
  int32_t x_f64;
  // output
  __nv_bfloat16* out;      // [N][R/rfast][kpn] (modes 0/1)
  const float* inv_lambda; // scaling (mode 1), index a*R + row
  void* y;                 // scatter target (mode 2)
  int32_t y_f64;
  // box of the free nodes (gather / scatter), direction 1 first
  int32_t n[3], lo[3], m[3];
  const __nv_bfloat16* Bimg;  // pre-tiled B (Np x Kp, canonical K-major)
  int32_t* status;
};

// a_mode: 0 = BF16 tensor, 1 = gather from x (rows (i3,i2), k = i1)
// o_mode: 0 = rotated BF16 store, 1 = same times 1/Lambda, 2 = scatter to y
template <int A_MODE, int O_MODE>
__device__ __forceinline__ void fd_tc_body(const TcGemm& g, const int bx) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ uint64_t bars[2];
  __shared__ uint32_t tmem_base;
  __shared__ int s_fail;
  __shared__ int64_t rowbase[128];
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int Kp = g.Kp, Np = g.Np;
  __nv_bfloat16* As = reinterpret_cast<__nv_bfloat16*>(smem_raw);            // 128 x Kp
  __nv_bfloat16* Bs = reinterpret_cast<__nv_bfloat16*>(smem_raw + 128 * Kp * 2);  // Np x Kp
  // CTA bx: rows of tile bx / nsplit, output columns [n_off, n_off + n_cnt)
  const int nsplit = tc_nsplit(Np);
  const int tile = bx / nsplit, half = bx - tile * nsplit;
  const int n1 = tc_first_half(Np);
  const int n_off = half ? n1 : 0, n_cnt = nsplit == 1 ? Np : (half ? Np - n1 : n1);
  const int row0 = tile * 128;
  uint32_t ncols = 32;
  while ((int)ncols < n_cnt) ncols <<= 1;

  if (tid == 0) {
    mbar_init(smem_u32(&bars[0]), 1);
    mbar_init(smem_u32(&bars[1]), 1);
    s_fail = 0;
    fence_mbar_init();
  }
  if (warp == 0) tc::tmem_alloc(smem_u32(&tmem_base), ncols);
  __syncthreads();
  // this CTA holds its tensor memory: the next product may be scheduled
  tc::launch_dependents();
  if (tid == 0) {
    // the B image is constant (eigenvectors), independent of the previous product
    const uint32_t bytes = (uint32_t)(Np * Kp * 2);
    mbar_arrive_expect_tx(smem_u32(&bars[0]), bytes);
    bulk_g2s(smem_u32(Bs), g.Bimg, bytes, smem_u32(&bars[0]));
  }
  // everything below reads the previous product's output (or the input
  // vector, written before the first product, which is launched in order)
  tc::wait_prerequisites();
  // ---- A tile in canonical K-major layout: core (grp, kc) at (kc*16 + grp)*128 B
  // Loads are issued in groups (all of a group before any of its shared
  // stores), so a thread keeps a group of global reads in flight instead of
  // one.
  // Descriptor fields used inside the loops are copied to registers first:
  // the descriptor may sit in shared memory (batch kernel), and every store
  // below could alias it for the compiler, forcing a re-read per element.
  const int kchunks = Kp / 8;
  const int R = g.R;
  if (A_MODE == 0) {
    // thread t owns row t mod 128 and half of its 16-byte chunks: a warp's
    // stores for one chunk index cover 512 contiguous bytes of the
    // canonical layout (chunk (kc, r) at kc * 2048 + r * 16), no conflicts
    constexpr int U = 8;
    const int r = tid & 127;
    const int halfc = (kchunks + 1) / 2;
    const int kc0 = (tid >> 7) ? halfc : 0, kc1 = (tid >> 7) ? kchunks : halfc;
    const bool live = row0 + r < R;
    const uint4* __restrict__ Arow =
        reinterpret_cast<const uint4*>(g.A + (size_t)(live ? row0 + r : 0) * Kp);
    unsigned char* dst = smem_raw + (size_t)r * 16;
    for (int k0 = kc0; k0 < kc1; k0 += U) {
      uint4 v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        v[u] = make_uint4(0, 0, 0, 0);
        if (live && k0 + u < kc1) v[u] = __ldg(Arow + k0 + u);
      }
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (k0 + u < kc1) *reinterpret_cast<uint4*>(dst + (size_t)(k0 + u) * 2048) = v[u];
    }
  } else {
    // rows (i3, i2) of the free box, k = i1: the vector index of each row's
    // first element once per CTA, then one add per element
    if (tid < 128) {
      const int row = row0 + tid;
      int64_t b = -1;
      if (row < R) {
        const int i3 = row / g.m[1], i2 = row - i3 * g.m[1];
        b = ((int64_t)(g.lo[2] + i3) * g.n[1] + g.lo[1] + i2) * g.n[0] + g.lo[0];
      }
      rowbase[tid] = b;
    }
    __syncthreads();
    const int nvalid = R - row0 < 128 ? R - row0 : 128;
    if (g.x_f64)
      gather_tile(reinterpret_cast<const double*>(g.x), rowbase, nvalid, Kp, g.m[0], As, tid);
    else
      gather_tile(reinterpret_cast<const float*>(g.x), rowbase, nvalid, Kp, g.m[0], As, tid);
  }
  tc::fence_proxy_async_smem();
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tbase = tmem_base;
  if (tid == 0) {
    if (!mbar_wait_bounded(smem_u32(&bars[0]), 0)) {
      s_fail = 1;
      if (g.status) atomicExch(g.status, IGA_ERR_TIMEOUT);
    } else {
      const uint32_t idesc = tc::idesc_bf16(128, n_cnt);
      // this CTA's output columns are B rows n_off .. n_off + n_cnt - 1: the
      // core matrices from group n_off / 8 on, same K stride as the full image
      const uint32_t a0 = smem_u32(As), b0 = smem_u32(Bs) + (uint32_t)(n_off / 8) * 128;
      const uint32_t lbo_a = 16 * 128, lbo_b = (uint32_t)(Np / 8) * 128;
      for (int kk = 0; kk < Kp / 16; ++kk) {
        const uint64_t ad = tc::smem_desc(a0 + 2 * kk * lbo_a, lbo_a, 128);
        const uint64_t bd = tc::smem_desc(b0 + 2 * kk * lbo_b, lbo_b, 128);
        tc::mma_bf16(tbase, ad, bd, idesc, kk > 0 ? 1u : 0u);
      }
      tc::mma_commit(smem_u32(&bars[1]));
    }
  }
  __syncthreads();
  // epilogue rows: warp w reads TMEM lanes 32 (w mod 4) .. +31 (= tile rows),
  // column chunks 16 (w div 4), +32, ...
  const int wq = warp & 3;
  const int r = wq * 32 + lane;
  const int row = row0 + r;
  const bool rv = row < R;
  const int Nout = g.N;
  const float* __restrict__ inv_lambda = g.inv_lambda;
  // 1/Lambda factors of a column chunk (scaling product only); the first
  // chunk's are read while the MMA chain runs, the next one's while the
  // current chunk is stored
  float lam[16], lamn[16];
  auto load_lam = [&](int c, float (&d)[16]) {
#pragma unroll
    for (int i = 0; i < 16; ++i)
      d[i] = (rv && c + i < Nout) ? __ldg(inv_lambda + (int64_t)(c + i) * R + row) : 0.f;
  };
  if (O_MODE == 1) load_lam(n_off + 16 * (warp >> 2), lam);
  bool ok = (s_fail == 0);
  if (ok) ok = mbar_wait_bounded(smem_u32(&bars[1]), 0);
  if (!__syncthreads_and(ok)) {
    if (tid == 0 && g.status) atomicExch(g.status, IGA_ERR_TIMEOUT);
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tbase, ncols);
    return;
  }
  tc::tc_fence_after();
  // ---- epilogue
  const int rs = rv ? row / g.rfast : 0, rf = rv ? row - rs * g.rfast : 0;
  const int nslow = R / g.rfast;
  // rotated store (modes 0/1): out[a][rs][rf]; scatter (mode 2): row =
  // (i2, i1) of the box, a = i3
  __nv_bfloat16* const out = g.out;
  const int64_t ostride = (int64_t)nslow * g.kpn, obase = (int64_t)rs * g.kpn + rf;
  const int64_t yplane = (int64_t)g.n[1] * g.n[0];
  int64_t ybase = 0;
  if (O_MODE == 2 && rv) {
    const int i1 = row % g.m[0], i2 = row / g.m[0];
    ybase = ((int64_t)g.lo[2] * g.n[1] + g.lo[1] + i2) * g.n[0] + g.lo[0] + i1;
  }
  const bool yf64 = g.y_f64 != 0;
  void* const yp = g.y;
  for (int c0 = 16 * (warp >> 2); c0 < n_cnt; c0 += 32) {
    if (O_MODE == 1 && c0 + 32 < n_cnt) load_lam(n_off + c0 + 32, lamn);
    float v[16];
    tc::tmem_ld16(tbase + ((uint32_t)(wq * 32) << 16) + (uint32_t)c0, v);
    if (rv) {
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int a = n_off + c0 + i;
        if (a >= Nout) break;
        if (O_MODE == 2) {
          const int64_t idx = ybase + (int64_t)a * yplane;
          if (yf64)
            reinterpret_cast<double*>(yp)[idx] = (double)v[i];
          else
            reinterpret_cast<float*>(yp)[idx] = v[i];
        } else {
          float val = v[i];
          if (O_MODE == 1) val *= lam[i];
          out[obase + (int64_t)a * ostride] = __float2bfloat16(val);
        }
      }
    }
    if (O_MODE == 1) {
#pragma unroll
      for (int i = 0; i < 16; ++i) lam[i] = lamn[i];
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tbase, ncols);
}

template <int A_MODE, int O_MODE>
__global__ void __launch_bounds__(kTcThreads) fd_tc_kernel(const __grid_constant__ TcGemm g) {
  fd_tc_body<A_MODE, O_MODE>(g, blockIdx.x);
}

// Many patches in one launch: patch p owns CTAs [cta0[p], cta0[p+1]); its
// product descriptor gs[p] goes to shared memory, with the gather source /
// scatter target moved to element offset offs[p] of the flat x / y.
template <int A_MODE, int O_MODE>
__global__ void __launch_bounds__(kTcThreads)
    fd_tc_batch_kernel(const TcGemm* __restrict__ gs, const int32_t* __restrict__ cta0, int np,
                       const int64_t* __restrict__ offs, const void* xb, void* yb,
                       const int32_t* __restrict__ skip) {
  __shared__ TcGemm sg;
  __shared__ int sp;
  if (threadIdx.x == 0) {
    int lo = 0, hi = np;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (__ldg(cta0 + mid) <= (int)blockIdx.x) lo = mid;
      else hi = mid;
    }
    sp = lo;
  }
  __syncthreads();
  const int p = sp;
  // one round of independent reads: the skip flag, one word of the product
  // descriptor per thread, the patch's vector offset and its first CTA
  constexpr int kWords = (int)(sizeof(TcGemm) / sizeof(int));
  static_assert(kWords <= kTcThreads, "descriptor copy: one word per thread");
  const int sk = skip ? __ldg(skip + p) : -1;
  const int word = threadIdx.x < kWords
                       ? __ldg(reinterpret_cast<const int*>(gs + p) + threadIdx.x) : 0;
  const int64_t off = (A_MODE == 1 || O_MODE == 2) ? __ldg(offs + p) : 0;
  const int first = __ldg(cta0 + p);
  if (sk >= 0) return;  // patch done: its output stays zero (same p for the whole CTA)
  if (threadIdx.x < kWords) reinterpret_cast<int*>(&sg)[threadIdx.x] = word;
  __syncthreads();
  if (threadIdx.x == 0) {
    if (A_MODE == 1) sg.x = (const char*)xb + off * (sg.x_f64 ? 8 : 4);
    if (O_MODE == 2) sg.y = (char*)yb + off * (sg.y_f64 ? 8 : 4);
  }
  __syncthreads();
  fd_tc_body<A_MODE, O_MODE>(sg, (int)blockIdx.x - first);
}

template <int A_MODE, int O_MODE>
static iga_status set_smem_tc(size_t smem) {
  IGA_CUDA_TRY(cudaFuncSetAttribute(fd_tc_batch_kernel<A_MODE, O_MODE>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  return IGA_OK;
}

// Launch configuration of one product: products after the first of an
// apply overlap their launch and prologue with the previous product
// (programmatic stream serialization; the kernels wait for it in-kernel).
struct TcLaunch {
  cudaLaunchConfig_t cfg;
  cudaLaunchAttribute attr[1];
  TcLaunch(unsigned grid, size_t smem, cudaStream_t st, bool overlap) {
    memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kTcThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = overlap ? 1 : 0;
  }
};

template <int A_MODE, int O_MODE>
static iga_status launch_tc_batch(const TcGemm* gs, const int32_t* cta0, int np,
                                  const int64_t* offs, int grid, size_t smem, const void* x,
                                  void* y, const int32_t* skip, cudaStream_t st, bool overlap) {
  static size_t configured = 48 * 1024;
  if (smem > configured) {
    iga_status rc = set_smem_tc<A_MODE, O_MODE>(smem);
    if (rc) return rc;
    configured = smem;
  }
  TcLaunch L((unsigned)grid, smem, st, overlap);
  IGA_CUDA_TRY(cudaLaunchKernelEx(&L.cfg, fd_tc_batch_kernel<A_MODE, O_MODE>, gs, cta0, np, offs,
                                  x, y, skip));
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

// The six rotated products of one patch (see iga_fd_apply_tc).
static void tc_stages(TcGemm g[6], const int32_t* n, const int32_t* lo, const int32_t* m,
                      const void* const* Bfwd, const void* const* Bbwd, const float* inv_lambda,
                      const void* x, void* y, int io_f64, void* work0, void* work1,
                      int32_t* status) {
  int kp[3];
  for (int d = 0; d < 3; ++d) kp[d] = (int)ceil_div(m[d], 16) * 16;
  const int m1 = m[0], m2 = m[1], m3 = m[2];
  __nv_bfloat16* w0 = (__nv_bfloat16*)work0;
  __nv_bfloat16* w1 = (__nv_bfloat16*)work1;
  TcGemm b;
  memset(&b, 0, sizeof(b));
  for (int d = 0; d < 3; ++d) {
    b.n[d] = n[d];
    b.lo[d] = lo[d];
    b.m[d] = m[d];
  }
  b.status = status;
  b.x = x;
  b.x_f64 = io_f64;
  b.y = y;
  b.y_f64 = io_f64;
  b.inv_lambda = inv_lambda;
  const __nv_bfloat16* F[3] = {(const __nv_bfloat16*)Bfwd[0], (const __nv_bfloat16*)Bfwd[1],
                               (const __nv_bfloat16*)Bfwd[2]};
  const __nv_bfloat16* Bk[3] = {(const __nv_bfloat16*)Bbwd[0], (const __nv_bfloat16*)Bbwd[1],
                                (const __nv_bfloat16*)Bbwd[2]};
  // (R, rfast, K dir, out fastest dir, A, B, out)
  auto set = [&](TcGemm& g, int R, int rfast, int kd, int od, const __nv_bfloat16* A,
                 const __nv_bfloat16* B, __nv_bfloat16* out) {
    g = b;
    g.R = R;
    g.rfast = rfast;
    g.Kp = kp[kd];
    g.N = m[kd];
    g.Np = kp[kd];
    g.kpn = kp[od];
    g.A = A;
    g.Bimg = B;
    g.out = out;
  };
  set(g[0], m3 * m2, m2, 0, 1, nullptr, F[0], w0);  // gather -> [a1][i3][Kp2]
  set(g[1], m1 * m3, m3, 1, 2, w0, F[1], w1);       // -> [a2][a1][Kp3]
  set(g[2], m2 * m1, m1, 2, 0, w1, F[2], w0);       // -> [a3][a2][Kp1] / Lambda
  set(g[3], m3 * m2, m2, 0, 1, w0, Bk[0], w1);      // -> [i1][a3][Kp2]
  set(g[4], m1 * m3, m3, 1, 2, w1, Bk[1], w0);      // -> [i2][i1][Kp3]
  set(g[5], m2 * m1, m1, 2, 0, w0, Bk[2], nullptr); // -> scatter y
}

template <int A_MODE, int O_MODE>
static iga_status launch_tc(const TcGemm& g, cudaStream_t st, bool overlap) {
  const size_t smem = (size_t)(128 + g.Np) * g.Kp * 2;
  auto kern = fd_tc_kernel<A_MODE, O_MODE>;
  static size_t configured = 48 * 1024;
  if (smem > configured) {
    IGA_CUDA_TRY(
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    configured = smem;
  }
  TcLaunch L((unsigned)(ceil_div(g.R, 128) * tc_nsplit(g.Np)), smem, st, overlap);
  IGA_CUDA_TRY(cudaLaunchKernelEx(&L.cfg, kern, g));
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

}  // namespace iga

using namespace iga;

extern "C" {

iga_status iga_fd_tc_workspace(const int32_t* m, int64_t* elems) {
  clear_error();
  IGA_CHECK_ARG(m && elems, "null argument");
  int64_t kp[3];
  for (int d = 0; d < 3; ++d) kp[d] = ceil_div(m[d], 16) * 16;
  // rotated intermediates: [a1][m3][Kp2], [a2][m1][Kp3], [a3][m2][Kp1] and
  // the backward ones; the largest bounds all
  int64_t big = 0;
  big = std::max<int64_t>(big, (int64_t)m[0] * m[2] * kp[1]);
  big = std::max<int64_t>(big, (int64_t)m[1] * m[0] * kp[2]);
  big = std::max<int64_t>(big, (int64_t)m[2] * m[1] * kp[0]);
  *elems = big;
  return IGA_OK;
}

// 3D FD apply with BF16 tensor-core mode products.  Bfwd[d] / Bbwd[d]: the
// pre-tiled images of U_d^T / U_d (Np_d x Kp_d BF16, canonical K-major, see
// igaops_b200/fastdiag.py); inv_lambda: FP32, prod(m) entries (direction 1
// fastest); x, y: FP32 or FP64 (io_dtype), full control-point vectors; y is
// zeroed outside the box.  work0 / work1: BF16, iga_fd_tc_workspace elements
// each, zero-initialised once by the caller (their padding is never written).
iga_status iga_fd_apply_tc(int io_dtype, const int32_t* n, const int32_t* lo, const int32_t* m,
                           const void* const* Bfwd, const void* const* Bbwd,
                           const float* inv_lambda, const void* x, void* y, void* work0,
                           void* work1, int32_t* status, iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(n && lo && m && Bfwd && Bbwd && inv_lambda && x && y && work0 && work1,
                "null argument");
  IGA_CHECK_ARG(io_dtype == IGA_F64 || io_dtype == IGA_F32, "io dtype %d", io_dtype);
  for (int d = 0; d < 3; ++d) {
    IGA_CHECK_ARG(m[d] >= 1 && m[d] <= 256, "free extent %d of direction %d not in 1..256", m[d],
                  d);
    IGA_CHECK_ARG(lo[d] >= 0 && lo[d] + m[d] <= n[d], "free box out of range in direction %d", d);
    IGA_CHECK_ARG(Bfwd[d] && Bbwd[d] && ((uintptr_t)Bfwd[d] & 15) == 0 &&
                      ((uintptr_t)Bbwd[d] & 15) == 0,
                  "B images must be 16-byte aligned");
  }
  IGA_CHECK_ARG(((uintptr_t)work0 & 15) == 0 && ((uintptr_t)work1 & 15) == 0,
                "work buffers must be 16-byte aligned");
  cudaStream_t st = as_stream(stream);
  int64_t N = (int64_t)n[0] * n[1] * n[2];
  IGA_CUDA_TRY(cudaMemsetAsync(y, 0, (size_t)N * (io_dtype == IGA_F64 ? 8 : 4), st));
  TcGemm g[6];
  tc_stages(g, n, lo, m, Bfwd, Bbwd, inv_lambda, x, y, io_dtype == IGA_F64, work0, work1, status);
  iga_status rc;
  if ((rc = launch_tc<1, 0>(g[0], st, false))) return rc;
  if ((rc = launch_tc<0, 0>(g[1], st, true))) return rc;
  if ((rc = launch_tc<0, 1>(g[2], st, true))) return rc;
  if ((rc = launch_tc<0, 0>(g[3], st, true))) return rc;
  if ((rc = launch_tc<0, 0>(g[4], st, true))) return rc;
  if ((rc = launch_tc<0, 2>(g[5], st, true))) return rc;
  return IGA_OK;
}


static inline int64_t tc_align(int64_t b) { return (b + 255) / 256 * 256; }

iga_status iga_fd_tc_batch_table_bytes(int npatch, int64_t* bytes) {
  clear_error();
  IGA_CHECK_ARG(npatch >= 1 && bytes, "bad argument");
  *bytes = 6 * tc_align((int64_t)npatch * sizeof(TcGemm)) + 6 * tc_align((int64_t)(npatch + 1) * 4) +
           (int64_t)npatch * 8;
  return IGA_OK;
}

// Multi-patch FD apply: per patch p the arrays hold n/lo/m at [3p..3p+2],
// Bfwd/Bbwd images at [3p..3p+2], inv_lambda[p], work0[p], work1[p] and the
// element offset of its vectors in the flat x / y.  Fills the device table
// (synchronous copies) and returns the grid of each of the six products and
// the dynamic shared memory of the largest patch.
iga_status iga_fd_tc_batch_prepare(int npatch, const int32_t* n, const int32_t* lo,
                                   const int32_t* m, const void* const* Bfwd,
                                   const void* const* Bbwd, const float* const* inv_lambda,
                                   void* const* work0, void* const* work1,
                                   const int64_t* offsets, int io_dtype, int32_t* status,
                                   void* table, int32_t* grid, int64_t* smem) {
  clear_error();
  IGA_CHECK_ARG(npatch >= 1 && n && lo && m && Bfwd && Bbwd && inv_lambda && work0 && work1 &&
                    offsets && table && grid && smem,
                "null argument");
  IGA_CHECK_ARG(io_dtype == IGA_F64 || io_dtype == IGA_F32, "io dtype %d", io_dtype);
  IGA_CHECK_ARG(((uintptr_t)table & 255) == 0, "table must be 256-byte aligned");
  std::vector<TcGemm> st((size_t)6 * npatch);
  std::vector<int32_t> cta((size_t)6 * (npatch + 1));
  std::vector<int64_t> offs((size_t)npatch);
  int64_t tot[6] = {0, 0, 0, 0, 0, 0};
  size_t sm = 0;
  for (int p = 0; p < npatch; ++p) {
    for (int d = 0; d < 3; ++d) {
      const int mm = m[3 * p + d];
      IGA_CHECK_ARG(mm >= 1 && mm <= 256, "patch %d: free extent %d not in 1..256", p, mm);
      IGA_CHECK_ARG(lo[3 * p + d] >= 0 && lo[3 * p + d] + mm <= n[3 * p + d],
                    "patch %d: free box out of range", p);
      IGA_CHECK_ARG(Bfwd[3 * p + d] && Bbwd[3 * p + d] && ((uintptr_t)Bfwd[3 * p + d] & 15) == 0 &&
                        ((uintptr_t)Bbwd[3 * p + d] & 15) == 0,
                    "patch %d: B images must be 16-byte aligned", p);
      const size_t kp = (size_t)ceil_div(mm, 16) * 16;
      sm = std::max(sm, (128 + kp) * kp * 2);
    }
    IGA_CHECK_ARG(inv_lambda[p] && work0[p] && work1[p] && ((uintptr_t)work0[p] & 15) == 0 &&
                      ((uintptr_t)work1[p] & 15) == 0 && offsets[p] >= 0,
                  "patch %d: bad Lambda / work / offset", p);
    TcGemm g[6];
    tc_stages(g, n + 3 * p, lo + 3 * p, m + 3 * p, Bfwd + 3 * p, Bbwd + 3 * p, inv_lambda[p],
              nullptr, nullptr, io_dtype == IGA_F64, work0[p], work1[p], status);
    for (int s = 0; s < 6; ++s) {
      st[(size_t)s * npatch + p] = g[s];
      cta[(size_t)s * (npatch + 1) + p] = (int32_t)tot[s];
      tot[s] += ceil_div(g[s].R, 128) * tc_nsplit(g[s].Np);
    }
    offs[p] = offsets[p];
  }
  for (int s = 0; s < 6; ++s) {
    IGA_CHECK_ARG(tot[s] < (1ll << 31), "too many CTAs");
    cta[(size_t)s * (npatch + 1) + npatch] = (int32_t)tot[s];
    grid[s] = (int32_t)tot[s];
  }
  char* t = (char*)table;
  const int64_t gb = tc_align((int64_t)npatch * sizeof(TcGemm));
  const int64_t cb = tc_align((int64_t)(npatch + 1) * 4);
  for (int s = 0; s < 6; ++s) {
    IGA_CUDA_TRY(cudaMemcpy(t + s * gb, st.data() + (size_t)s * npatch, npatch * sizeof(TcGemm),
                            cudaMemcpyHostToDevice));
    IGA_CUDA_TRY(cudaMemcpy(t + 6 * gb + s * cb, cta.data() + (size_t)s * (npatch + 1),
                            (npatch + 1) * 4, cudaMemcpyHostToDevice));
  }
  IGA_CUDA_TRY(cudaMemcpy(t + 6 * gb + 6 * cb, offs.data(), npatch * 8, cudaMemcpyHostToDevice));
  *smem = (int64_t)sm;
  return IGA_OK;
}

iga_status iga_fd_tc_batch_apply(int io_dtype, int npatch, const void* table, const int32_t* grid,
                                 int64_t smem, const void* x, void* y, int64_t ntot,
                                 const int32_t* skip, iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(npatch >= 1 && table && grid && x && y && ntot >= 0 && smem > 0 &&
                    smem <= 227 * 1024,
                "bad argument");
  IGA_CHECK_ARG(io_dtype == IGA_F64 || io_dtype == IGA_F32, "io dtype %d", io_dtype);
  cudaStream_t st = as_stream(stream);
  IGA_CUDA_TRY(cudaMemsetAsync(y, 0, (size_t)ntot * (io_dtype == IGA_F64 ? 8 : 4), st));
  const char* t = (const char*)table;
  const int64_t gb = tc_align((int64_t)npatch * sizeof(TcGemm));
  const int64_t cb = tc_align((int64_t)(npatch + 1) * 4);
  const int64_t* offs = (const int64_t*)(t + 6 * gb + 6 * cb);
  auto G = [&](int s) { return (const TcGemm*)(t + s * gb); };
  auto C = [&](int s) { return (const int32_t*)(t + 6 * gb + s * cb); };
  iga_status rc;
  if ((rc = launch_tc_batch<1, 0>(G(0), C(0), npatch, offs, grid[0], smem, x, y, skip, st,
                                     false)))
    return rc;
  if ((rc = launch_tc_batch<0, 0>(G(1), C(1), npatch, offs, grid[1], smem, x, y, skip, st,
                                     true)))
    return rc;
  if ((rc = launch_tc_batch<0, 1>(G(2), C(2), npatch, offs, grid[2], smem, x, y, skip, st,
                                     true)))
    return rc;
  if ((rc = launch_tc_batch<0, 0>(G(3), C(3), npatch, offs, grid[3], smem, x, y, skip, st,
                                     true)))
    return rc;
  if ((rc = launch_tc_batch<0, 0>(G(4), C(4), npatch, offs, grid[4], smem, x, y, skip, st,
                                     true)))
    return rc;
  if ((rc = launch_tc_batch<0, 2>(G(5), C(5), npatch, offs, grid[5], smem, x, y, skip, st,
                                     true)))
    return rc;
  return IGA_OK;
}

}  // extern "C"
