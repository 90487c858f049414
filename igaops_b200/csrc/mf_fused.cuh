// Fused matrix-free weighted-quadrature operator kernels (2D and 3D).
//
// One kernel computes, for one patch,
//     y = sum_i W^{(alpha_i)} [ sum_j C_ij  (B^{(beta_j)} x) ]
// which is the arithmetic of BsplineOperations.compute_mf_scalar_u_v /
// gradu_gradv / gradu_v / u_gradv (src/igaops/operators/bsplines_ops.py:
// 290-429): the trial factors B (basis values/derivatives at quadrature
// points) interpolate x, the per-point coefficients C mix the components,
// the test factors W (weighted-quadrature weights) project back.  The
// reference runs this as separate sparse mode products over full Nq-sized
// intermediates (src/igaops/operators/utils/matrix_free.py:77-119); here all
// intermediates live in registers / shared memory and only C is streamed.
//
// Work decomposition (3D): a CTA owns a face tile of FX x FY quadrature points
// in directions 1,2 and a segment of direction 3.  Thread (lx, ly) owns the
// pencil (q1, q2, :) and marches along q3:
//   * trial window: the values A_{b1 b2}(q1,q2,c3) of W consecutive control
//     planes c3 (W = band width = p+1) sit in registers; a new plane is made
//     cooperatively from the x plane slice (dir-1 then dir-2 contractions in
//     shared memory) when the band start of row q3 advances;
//   * the coefficient chunk C(:, q1, q2, q3) of the tile arrives by a 1D TMA
//     bulk copy into a ring of NST shared-memory slots (mbarrier completion);
//   * test accumulators G_i(q1,q2,c3') for W control planes sit in registers;
//     when the band start of W^T row q3 passes plane c3', that plane is final:
//     the CTA contracts it over q2 and q1 in shared memory and adds it to y
//     with atomics (control planes near tile/segment edges are shared).
// 2D is the same with a 1D face (FX threads) marching along q2.
//
// This requires the test weights to depend on the test derivative only
// (W00 == W01 and W10 == W11), true for weighted quadrature of type "2" and
// for Gauss rules; other rules use the unfused path.
#pragma once

#include <algorithm>
#include <cstring>

#include "common.cuh"

namespace iga {

struct SrcRows {
  int32_t r[9];
};

// ----------------------------------------------------------- op patterns
// D: parametric dimension; OP: IGA_OP_*; ST: last direction is time with
// test/trial time-derivative orders TT/TR; SYM: symmetric stiffness packing.
template <int D, int OP, int ST, int TT, int TR, int SYM>
struct Pat {
  static constexpr int SP = ST ? D - 1 : D;  // spatial directions
  static constexpr bool trial_grad = (OP == IGA_OP_STIFF || OP == IGA_OP_U_GRADV);
  static constexpr bool test_grad = (OP == IGA_OP_STIFF || OP == IGA_OP_GRADU_V);
  static constexpr int J = trial_grad ? SP : 1;
  static constexpr int I = test_grad ? SP : 1;
  static constexpr int S =
      OP == IGA_OP_STIFF ? (SYM ? SP * (SP + 1) / 2 : SP * SP) : (OP == IGA_OP_MASS ? 1 : SP);
  // derivative order of trial component j in direction k
  __host__ __device__ static constexpr int beta(int j, int k) {
    return (ST && k == D - 1) ? TR : (trial_grad ? (k == j ? 1 : 0) : 0);
  }
  // derivative order of test component i in direction k
  __host__ __device__ static constexpr int alpha(int i, int k) {
    return (ST && k == D - 1) ? TT : (test_grad ? (k == i ? 1 : 0) : 0);
  }
  __host__ __device__ static constexpr int tri(int a, int b) {  // a < b
    return SP == 2 ? 0 : (a == 0 ? b - 1 : 2);
  }
  // coefficient stream feeding (test i, trial j)
  __host__ __device__ static constexpr int cidx(int i, int j) {
    return OP == IGA_OP_MASS      ? 0
           : OP == IGA_OP_GRADU_V ? i
           : OP == IGA_OP_U_GRADV ? j
           : SYM ? (i == j ? i : SP + (i < j ? tri(i, j) : tri(j, i)))
                 : i * SP + j;
  }
  // forward combo (b1 + 2*b2) of trial component j (3D) / b1 (2D)
  __host__ __device__ static constexpr int combo(int j) {
    return D == 3 ? beta(j, 0) + 2 * beta(j, 1) : beta(j, 0);
  }
  __host__ __device__ static constexpr bool combo_needed(int c) {
    for (int j = 0; j < J; ++j)
      if (combo(j) == c) return true;
    return false;
  }
  __host__ __device__ static constexpr bool b1_needed(int b) {
    for (int j = 0; j < J; ++j)
      if (beta(j, 0) == b) return true;
    return false;
  }
  __host__ __device__ static constexpr bool last_trial_needed(int b) {
    for (int j = 0; j < J; ++j)
      if (beta(j, D - 1) == b) return true;
    return false;
  }
  __host__ __device__ static constexpr bool last_test_needed(int a) {
    for (int i = 0; i < I; ++i)
      if (alpha(i, D - 1) == a) return true;
    return false;
  }
  // (3D) test pair index a1 + 2*a2 of component i; 2D: a1
  __host__ __device__ static constexpr int tpair(int i) {
    return D == 3 ? alpha(i, 0) + 2 * alpha(i, 1) : alpha(i, 0);
  }
  __host__ __device__ static constexpr bool tpair_needed(int pr) {
    for (int i = 0; i < I; ++i)
      if (tpair(i) == pr) return true;
    return false;
  }
  __host__ __device__ static constexpr bool a1_needed(int g) {
    for (int i = 0; i < I; ++i)
      if (alpha(i, 0) == g) return true;
    return false;
  }
};

// ----------------------------------------------------------- arguments
template <typename T>
struct FusedArgs {
  int32_t n[3], nq[3];
  int32_t W, RW;
  int32_t tiles1, tiles2, nseg;
  int32_t cmax1, cmax2, dmax1, dmax2;
  int64_t N;  // number of control points (column stride of x, y)
  const int64_t* tile_off;
  const int32_t* tstart[3];
  const T* tB0[3];
  const T* tB1[3];
  const int32_t* wtstart[3];
  const T* wT0[3];
  const T* wT1[3];
  const int32_t* rstart[3];
  const T* wR0[3];
  const T* wR1[3];
  const T* packed;
  const T* step_table;  // [nq_last][rlen]: B0, B1, W0T, W1T (W each), tstart, wtstart
  int32_t rlen;
  const T* x;
  T* y;
  int32_t* status;
  int32_t wait_test;  // test hook: withhold point 0's copies (see iga_mf_plan)
};

// Band starts in the step table are stored as integer bit patterns in an
// element of the table's type (no conversion on the per-point path).
__host__ __device__ inline double step_start_enc(int v, double) {
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)v);
#else
  long long b = v;
  double d;
  memcpy(&d, &b, 8);
  return d;
#endif
}
__host__ __device__ inline float step_start_enc(int v, float) {
#ifdef __CUDA_ARCH__
  return __int_as_float(v);
#else
  float f;
  memcpy(&f, &v, 4);
  return f;
#endif
}
__device__ __forceinline__ int step_start(double v) { return (int)__double_as_longlong(v); }
__device__ __forceinline__ int step_start(float v) { return __float_as_int(v); }

// Step-table row of one point of the streamed direction: the groups B0, B1,
// W0^T, W1^T (W values each) at stride step_group(W) -- W rounded up to a
// whole number of 16-byte vectors, so each group loads as 16-byte vectors --
// then the two band starts; the row is padded to 16 bytes.
template <typename T>
__host__ __device__ constexpr int step_group(int W) {
  return (W + 16 / (int)sizeof(T) - 1) / (16 / (int)sizeof(T)) * (16 / (int)sizeof(T));
}
template <typename T>
__host__ __device__ constexpr int step_row_len(int W) {
  return (4 * step_group<T>(W) + 2 + 16 / (int)sizeof(T) - 1) / (16 / (int)sizeof(T)) *
         (16 / (int)sizeof(T));
}

// A group of the step-table row as 16-byte vector loads (G a multiple of
// 16 / sizeof(T)).
template <typename T, int G>
__device__ __forceinline__ void load_group(const T* src, T (&dst)[G]) {
  if constexpr (sizeof(T) == 8) {
#pragma unroll
    for (int k = 0; k < G / 2; ++k) {
      const double2 v = reinterpret_cast<const double2*>(src)[k];
      dst[2 * k] = v.x;
      dst[2 * k + 1] = v.y;
    }
  } else {
#pragma unroll
    for (int k = 0; k < G / 4; ++k) {
      const float4 v = reinterpret_cast<const float4*>(src)[k];
      dst[4 * k] = v.x;
      dst[4 * k + 1] = v.y;
      dst[4 * k + 2] = v.z;
      dst[4 * k + 3] = v.w;
    }
  }
}

// 3D coefficient chunks with an even stream count are stored point-major,
// [l2][l1][stream], so that a thread reads its point's streams as pairs
// (vector loads); odd stream counts stay stream-major, [stream][l2][l1].
__host__ __device__ constexpr bool point_major3(int S) { return S % 2 == 0; }

template <typename T>
__host__ __device__ inline int64_t chunk_stride_elems(int S, int w1, int w2) {
  const int64_t e = 16 / (int64_t)sizeof(T);
  return ((int64_t)S * w1 * w2 + e - 1) / e * e;
}

template <typename T>
inline size_t mf2d_smem_bytes(int S, int FX, int NST) {
  return 128 + ((size_t)NST * S * FX + 2 * (size_t)FX) * sizeof(T);
}

template <class P>
__host__ __device__ constexpr int npair3() {
  int n = 0;
  for (int pr = 0; pr < 4; ++pr)
    if (P::tpair_needed(pr)) ++n;
  return n;
}
template <class P>
__host__ __device__ constexpr int pair_slot(int pr) {
  int n = 0;
  for (int q = 0; q < pr; ++q)
    if (P::tpair_needed(q)) ++n;
  return n;
}

__device__ __forceinline__ void report_status(int32_t* status, int32_t code) {
  if (status) atomicExch(status, code);
}

// ===================================================================== 3D
// Number of (b1, b2) trial combos a pattern needs, and the slot of each.
template <class P>
__host__ __device__ constexpr int ncombo3() {
  int n = 0;
  for (int c = 0; c < 4; ++c)
    if (P::combo_needed(c)) ++n;
  return n;
}
template <class P>
__host__ __device__ constexpr int combo_slot(int c) {
  int n = 0;
  for (int q = 0; q < c; ++q)
    if (P::combo_needed(q)) ++n;
  return n;
}
template <class P>
__host__ __device__ constexpr int combo_of_slot(int cs) {
  for (int c = 0; c < 4; ++c)
    if (P::combo_needed(c) && combo_slot<P>(c) == cs) return c;
  return 0;
}
template <class P>
__host__ __device__ constexpr int nb1() {
  return (P::b1_needed(0) ? 1 : 0) + (P::b1_needed(1) ? 1 : 0);
}
template <class P>
__host__ __device__ constexpr int b1_slot(int b) {
  return (b == 1 && P::b1_needed(0)) ? 1 : 0;
}
template <class P>
__host__ __device__ constexpr int ng() {
  return (P::a1_needed(0) ? 1 : 0) + (P::a1_needed(1) ? 1 : 0);
}
template <class P>
__host__ __device__ constexpr int g_slot(int g) {
  return (g == 1 && P::a1_needed(0)) ? 1 : 0;
}

// Pipeline depths and resident CTAs per SM of the 3D kernel (overridable at
// build time for tuning): QC points per chunk, NST coefficient slots in the
// TMA ring (it runs NST / QC whole chunks ahead), MINB the resident CTAs the
// register budget is set for. FP64
// patterns with >= 3 coefficient streams ("S") keep three CTAs in shared
// memory; the light patterns and FP32 run more, smaller CTAs (FP32 "S" with
// band width <= 4: the "SN" depths).
#ifndef IGA_QC64
#define IGA_QC64 6
#endif
#ifndef IGA_NST64
#define IGA_NST64 6
#endif
#ifndef IGA_MINB64
#define IGA_MINB64 5
#endif
#ifndef IGA_QC64S
#define IGA_QC64S 4
#endif
#ifndef IGA_NST64S
#define IGA_NST64S 4
#endif
#ifndef IGA_MINB64S
#define IGA_MINB64S 3
#endif
#ifndef IGA_ALIAS64S
#define IGA_ALIAS64S 1
#endif
#ifndef IGA_MINB64SA
#define IGA_MINB64SA 4
#endif
#ifndef IGA_QC32
#define IGA_QC32 8
#endif
#ifndef IGA_NST32
#define IGA_NST32 8
#endif
#ifndef IGA_MINB32
#define IGA_MINB32 6
#endif
#ifndef IGA_QC32S
#define IGA_QC32S 6
#endif
#ifndef IGA_NST32S
#define IGA_NST32S 6
#endif
#ifndef IGA_MINB32S
#define IGA_MINB32S 4
#endif
#ifndef IGA_QC32SN
#define IGA_QC32SN 4
#endif
#ifndef IGA_NST32SN
#define IGA_NST32SN 4
#endif
#ifndef IGA_MINB32SN
#define IGA_MINB32SN 6
#endif
// The FP64 q1 contraction of the test planes (the last flush stage) runs on
// the FP64 tensor cores (DMMA, one mma.sync.m8n8k4 per 8 x 8 x 4 block: 256
// FMAs per warp instruction), and for the light patterns the q2 flush stage
// too; everything else, and all of FP32, stays on the FMA pipes (the trial
// contractions are banded, so their dense tensor-core form does more work
// than it saves in issue slots).
template <typename T>
__host__ __device__ constexpr bool use_dmma() {
  return sizeof(T) == 8;
}

template <typename T, class P>
struct Depth3 {
  static constexpr bool heavy = P::S >= 3;
  __host__ __device__ static constexpr bool narrow(int W) { return W <= 4; }
  __host__ __device__ static constexpr int qc0(int W) {
    return sizeof(T) == 8 ? (heavy ? IGA_QC64S : IGA_QC64)
                          : (heavy ? (narrow(W) ? IGA_QC32SN : IGA_QC32S) : IGA_QC32);
  }
  __host__ __device__ static constexpr int nst0(int W) {
    return sizeof(T) == 8 ? (heavy ? IGA_NST64S : IGA_NST64)
                          : (heavy ? (narrow(W) ? IGA_NST32SN : IGA_NST32S) : IGA_NST32);
  }
  // resident CTAs per SM (register budget of a thread)
  __host__ __device__ static constexpr int minb(int W) {
    return sizeof(T) == 8 ? (heavy ? (alias(W) ? IGA_MINB64SA : IGA_MINB64S) : IGA_MINB64)
                          : (heavy ? (narrow(W) ? IGA_MINB32SN : IGA_MINB32S) : IGA_MINB32);
  }
  // buffers with disjoint lifetimes share memory (FP64 stiffness of band
  // width 3: four CTAs per SM instead of three; at width 4 the register
  // budget of four CTAs costs more than the fourth CTA gains)
  __host__ __device__ static constexpr bool alias(int W) {
    return sizeof(T) == 8 && heavy && W <= 3 && IGA_ALIAS64S;
  }
  // the q2 flush on the FP64 tensor cores pays off for the light patterns
  // only (one test pair; the stiffness's three pairs keep the FMA pipes)
  __host__ __device__ static constexpr bool q2_dmma() { return use_dmma<T>() && !heavy; }
  // a chunk holds at least a full band of W planes; the ring at least a
  // whole chunk
  __host__ __device__ static constexpr int qc(int W) { return qc0(W) > W ? qc0(W) : W; }
  __host__ __device__ static constexpr int nst(int W) { return nst0(W) > qc(W) ? nst0(W) : qc(W); }
};


// Column swizzle of the 16-wide shared-memory tiles read as DMMA fragments
// (rows of 16 doubles span all 32 banks, so the four rows of a fragment
// would collide): column c of row r is stored at c ^ 4 (r mod 4). Identity
// for FP32.
template <typename T>
__device__ __forceinline__ int swz(int c, int r) {
  if constexpr (use_dmma<T>()) return c ^ ((r & 3) << 2);
  else return c;
}

// Shared-memory layout of the 3D kernel: element offsets of its regions
// after the 128-byte barrier area, each region starting on a 16-byte
// boundary (vector loads of pairs and groups).
template <typename T, class P>
struct Smem3 {
  static constexpr int A = 16 / (int)sizeof(T);
  int ks_row, w1_row, w2_row;  // row strides (elements)
  int ring, stage, done, ks, xs, a1s, b1tab, b2tab, w1d, w2d, total;
  __host__ __device__ static int up(long v) { return (int)((v + A - 1) / A * A); }
  __host__ __device__ Smem3(int FX, int FY, int W, int rlen, int cmax1, int cmax2, int dmax1,
                            int dmax2) {
    const int QC = Depth3<T, P>::qc(W), NST = Depth3<T, P>::nst(W);
    const int nt = FX * FY;
    // FP32: rows padded by two (conflict-free pair loads); FP64: swizzled
    ks_row = FX + (use_dmma<T>() ? 0 : 2);
    w1_row = 2 * FX + (use_dmma<T>() ? 0 : 2);
    // w2d: [r2][l2][b] rows of 2 FY (FP64: + 2, so that the two halves of a
    // warp read different banks); with the tensor-core q2 flush [b][r2][l2]
    // rows of FY + 4 (conflict-free A fragments)
    w2_row = Depth3<T, P>::q2_dmma() ? FY + 4 : 2 * FY + (sizeof(T) == 8 ? 2 : 0);
    ring = 0;
    stage = ring + up((long)NST * (P::S * nt + rlen));
    const int n_stage = up((long)QC * ncombo3<P>() * nt), n_done = up((long)QC * npair3<P>() * nt);
    const int n_ks = up((long)QC * ng<P>() * dmax2 * ks_row), n_xs = up((long)QC * cmax1 * cmax2);
    const int n_a1s = up((long)QC * nb1<P>() * cmax2 * FX);
    if (Depth3<T, P>::alias(W)) {
      // the q2 flush buffer and the x slab live inside the trial staging
      // ring, the q1 production buffer inside the test ring (the kernel
      // separates their lifetimes with barriers)
      ks = stage;
      xs = ks + n_ks;
      done = stage + (n_stage > n_ks + n_xs ? n_stage : n_ks + n_xs);
      a1s = done;
      b1tab = done + (n_done > n_a1s ? n_done : n_a1s);
    } else {
      done = stage + n_stage;
      ks = done + n_done;
      xs = ks + n_ks;
      a1s = xs + n_xs;
      b1tab = a1s + n_a1s;
    }
    b2tab = b1tab + up((long)FX * 2 * W);
    w1d = b2tab + up((long)FY * 2 * W);
    w2d = w1d + up((long)dmax1 * w1_row);
    total = w2d + up((long)(Depth3<T, P>::q2_dmma() ? 2 : 1) * dmax2 * w2_row);
  }
};

// D += A B on one 8 x 8 x 4 FP64 block (mma.sync.m8n8k4, row.col): lane l
// holds A[l / 4][l % 4], B[l % 4][l / 4] and D[l / 4][2 (l % 4) + {0, 1}].
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Shared-memory size of the 3D kernel (bytes).
template <typename T, class P>
inline size_t mf3d_smem_bytes(int FX, int FY, int W, int RW, int rlen, int cmax1, int cmax2,
                              int dmax1, int dmax2) {
  (void)RW;
  const Smem3<T, P> L(FX, FY, W, rlen, cmax1, cmax2, dmax1, dmax2);
  return 128 + (size_t)L.total * sizeof(T) + 16;
}

// Two adjacent elements as one vector load (address aligned to 2 elements).
template <typename T>
__device__ __forceinline__ void ld2(const T* p, T& a, T& b) {
  if constexpr (sizeof(T) == 8) {
    const double2 v = *reinterpret_cast<const double2*>(p);
    a = v.x;
    b = v.y;
  } else {
    const float2 v = *reinterpret_cast<const float2*>(p);
    a = v.x;
    b = v.y;
  }
}

// Every thread owns one pencil (q1,q2,:) of the face tile; thread 0 also
// streams the coefficient chunks and step-table rows through an NST-deep
// ring of TMA bulk copies completing on full[] mbarriers.  Threads
// synchronise (named barrier 1) only at chunk boundaries, every QC points.
template <typename T, int FX, int FY, int W, class P>
__device__ __forceinline__ void mf3d_body(const FusedArgs<T>& a, const int unit, const int col) {
  constexpr int NT = FX * FY;
  constexpr int S = P::S;
  constexpr int I = P::I;
  constexpr int J = P::J;
  constexpr int QC = Depth3<T, P>::qc(W);
  constexpr int NST = Depth3<T, P>::nst(W);
  constexpr int NPAIR = npair3<P>();
  constexpr int NCOMBO = ncombo3<P>();
  constexpr int NB1 = nb1<P>();
  constexpr int NG = ng<P>();
  static_assert(NT % 32 == 0, "face must be a whole number of warps");
  static_assert(FX % 2 == 0 && FY % 2 == 0, "pair loads over the face");
  static_assert(!use_dmma<T>() || (FX == 16 && FY == 8), "DMMA tiling of the 16 x 8 face");
  static_assert(QC >= W, "a chunk must hold a full band of planes");
  static_assert(NST >= QC, "the ring must hold a whole chunk");
  static_assert(NST * sizeof(uint64_t) <= 128, "barrier area");
  static_assert(NST % QC == 0, "a chunk's points share one lap of the ring");

  const int RW = a.RW;
  // Light patterns (a chunk unrolled, registers to spare) address a point's
  // ring slot as a fixed offset from its chunk's slot base -- the step-table
  // row length follows from the band width (the host sets a.rlen from the
  // same formula) -- and advance the windows' ring positions with the
  // windows; heavy patterns, at their register budget, recompute both per
  // point (one register fewer per value, measured faster there).
  constexpr bool kRunSlots = !Depth3<T, P>::heavy;
  const int rlen = kRunSlots ? step_row_len<T>(W) : a.rlen;
  const int slot_elems = S * NT + rlen;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw);
  const Smem3<T, P> lay(FX, FY, W, rlen, a.cmax1, a.cmax2, a.dmax1, a.dmax2);
  const int KS = lay.ks_row;   // ks[(pl, g, r2)][l1], row stride KS
  const int W1S = lay.w1_row;  // w1d[r1][b][l1], row stride W1S
  T* base = reinterpret_cast<T*>(smem_raw + 128);
  T* cring = base + lay.ring;
  T* stage = base + lay.stage;
  T* done = base + lay.done;
  T* ks = base + lay.ks;
  T* xs = base + lay.xs;
  T* a1s = base + lay.a1s;
  T* b1tab = base + lay.b1tab;  // [2][W][FX] (lanes of a warp read consecutive lx)
  T* b2tab = base + lay.b2tab;  // [FY][2][W]
  // test weights of the tile as dense blocks (zero outside the band):
  // w1d[r1][b][l1] = W_b(d1lo + r1, q1lo + l1), w2d[r2][l2][b] likewise
  T* w1d = base + lay.w1d;  // [dmax1][2][FX] (swizzled / padded rows)
  T* w2d = base + lay.w2d;  // [dmax2][FY][2] (rows of W2S)
  const int W2S = lay.w2_row;
  __shared__ int s_abort;

  const int tid = threadIdx.x;
  const int n1 = a.n[0], n2 = a.n[1], n3 = a.n[2];
  const int nq1 = a.nq[0], nq2 = a.nq[1], nq3 = a.nq[2];
  const int seg = unit % a.nseg;
  const int tt = unit / a.nseg;
  const int t1 = tt % a.tiles1;
  const int t2 = tt / a.tiles1;
  const int q1lo = t1 * FX, w1 = min(FX, nq1 - q1lo);
  const int q2lo = t2 * FY, w2 = min(FY, nq2 - q2lo);
  const int qa = (int)((int64_t)nq3 * seg / a.nseg);
  const int qb = (int)((int64_t)nq3 * (seg + 1) / a.nseg);
  const int L = qb - qa;
  const int64_t cstride = chunk_stride_elems<T>(S, w1, w2);
  const uint32_t cbytes = (uint32_t)(cstride * sizeof(T));
  const uint32_t rbytes = (uint32_t)(rlen * sizeof(T));
  const T* cbase = a.packed + __ldg(a.tile_off + (int64_t)t2 * a.tiles1 + t1);

  // Thread 0 streams, per point q3 of the segment, the coefficient chunk of
  // the tile plus the step-table row of q3 into ring slot q3 % NST (1D TMA
  // bulk copies, completion on full[slot]). The ring runs RA points (whole
  // chunks) ahead: when every thread has consumed a chunk's points (after
  // the chunk barrier) the copies of the points up to RA past its end are
  // issued into the freed slots, so they land during the flush / produce
  // phases and the per-point steps of the chunks before them.
  // Lane 0 of warp w issues points w, w + NT/32, ...: the issue cost is
  // spread over the warps instead of holding one warp back.
  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < NST; ++s) mbar_init(smem_u32(&full[s]), 1);
    s_abort = 0;
    fence_mbar_init();
  }
  __syncthreads();
  int issued_hi = 0;  // points whose copies are issued
  auto issue = [&](int t_lo, int t_hi) {
    if ((tid & 31) == 0) {
      for (int t = t_lo + tid / 32; t < t_hi; t += NT / 32) {
        if (a.wait_test && t == 0) continue;  // the withheld copy: its wait runs out
        const int slot = t % NST;
        const uint32_t bar = smem_u32(&full[slot]);
        T* dst = cring + slot * slot_elems;
        mbar_arrive_expect_tx(bar, cbytes + rbytes);
        bulk_g2s(smem_u32(dst), cbase + (int64_t)(qa + t) * cstride, cbytes, bar);
        bulk_g2s(smem_u32(dst + S * NT), a.step_table + (int64_t)(qa + t) * rlen, rbytes, bar);
      }
    }
    issued_hi = t_hi;
  };
  constexpr int RA = NST / QC * QC;  // points in flight at a chunk's start
  issue(0, min(RA, L));

  // ----------------------------------------------------- consumer warps
  const int lx = tid % FX, ly = tid / FX;
  const int warp = tid >> 5, gq = (tid & 31) >> 2, tq = tid & 3;  // DMMA fragment coordinates
  const bool valid = (lx < w1) && (ly < w2);
  const int q1 = q1lo + min(lx, w1 - 1);
  const int q2 = q2lo + min(ly, w2 - 1);
  const T* __restrict__ x = a.x + (int64_t)col * a.N;
  T* __restrict__ y = a.y + (int64_t)col * a.N;

  const int c1lo = __ldg(a.tstart[0] + q1lo);
  const int C1r = __ldg(a.tstart[0] + q1lo + w1 - 1) - c1lo + W;
  const int c2lo = __ldg(a.tstart[1] + q2lo);
  const int C2r = __ldg(a.tstart[1] + q2lo + w2 - 1) - c2lo + W;
  const int d1lo = __ldg(a.wtstart[0] + q1lo);
  const int D1r = min(__ldg(a.wtstart[0] + q1lo + w1 - 1) + W - 1, n1 - 1) - d1lo + 1;
  const int d2lo = __ldg(a.wtstart[1] + q2lo);
  const int D2r = min(__ldg(a.wtstart[1] + q2lo + w2 - 1) + W - 1, n2 - 1) - d2lo + 1;
  const int s1rel = __ldg(a.tstart[0] + q1) - c1lo;
  const int s2rel = __ldg(a.tstart[1] + q2) - c2lo;
  // tile-local index decompositions (divisors fixed for the CTA)
  const int perx = C2r * C1r, perf = D2r * D1r;
  const FastDiv dv_perx(perx), dv_c1(C1r), dv_c2(C2r), dv_perf(perf), dv_d1(D1r), dv_d2(D2r);
  // tensor-core flush task decomposition (8-row / 8-column blocks)
  const FastDiv dv_mt((D2r + 7) >> 3), dv_nt1((D1r + 7) >> 3);

  // per-tile coefficient tables
  for (int e = tid; e < FX * 2 * W; e += NT) {
    const int l = e / (2 * W), r = e - l * 2 * W, b = r / W, k = r - b * W;
    const int qq = q1lo + min(l, w1 - 1);
    b1tab[(b * W + k) * FX + l] = __ldg((b ? a.tB1[0] : a.tB0[0]) + (int64_t)qq * W + k);
  }
  for (int e = tid; e < FY * 2 * W; e += NT) {
    const int l = e / (2 * W), r = e - l * 2 * W, b = r / W, k = r - b * W;
    const int qq = q2lo + min(l, w2 - 1);
    b2tab[e] = __ldg((b ? a.tB1[1] : a.tB0[1]) + (int64_t)qq * W + k);
  }
  for (int e = tid; e < a.dmax1 * 2 * FX; e += NT) {
    const int r = e / (2 * FX), rem = e - r * 2 * FX;
    const int b = rem / FX, l1 = rem - b * FX;
    T v = T(0);
    if (r < D1r && l1 < w1) {
      const int k = q1lo + l1 - __ldg(a.rstart[0] + d1lo + r);
      if (k >= 0 && k < RW) v = __ldg((b ? a.wR1[0] : a.wR0[0]) + (int64_t)(d1lo + r) * RW + k);
    }
    w1d[r * W1S + b * FX + swz<T>(l1, r)] = v;
  }
  for (int e = tid; e < a.dmax2 * FY * 2; e += NT) {
    const int r = e / (FY * 2), rem = e - r * FY * 2, l2 = rem >> 1, b = rem & 1;
    T v = T(0);
    if (r < D2r && l2 < w2) {
      const int k = q2lo + l2 - __ldg(a.rstart[1] + d2lo + r);
      if (k >= 0 && k < RW) v = __ldg((b ? a.wR1[1] : a.wR0[1]) + (int64_t)(d2lo + r) * RW + k);
    }
    if constexpr (Depth3<T, P>::q2_dmma()) w2d[(b * a.dmax2 + r) * W2S + l2] = v;
    else w2d[r * W2S + rem] = v;
  }
  named_sync(1, NT);

  // x slab of planes p0 .. p0+np-1: the first XPF*NT elements are fetched
  // into registers ahead of time (prefetch), the rest when stored
  constexpr int XPF = (sizeof(T) == 8 && Depth3<T, P>::heavy) ? 2 : 4;
  T xpf[XPF];
  // the first XPF*NT slab elements of this thread: shared-memory index and
  // global offset relative to plane p0 (fixed for the CTA)
  int xsi[XPF], xpl[XPF];
  int64_t xgo[XPF];
  bool xin[XPF];
#pragma unroll
  for (int i = 0; i < XPF; ++i) {
    const int e = tid + i * NT;
    const int pl = dv_perx.div(e), rem = e - pl * perx;
    const int r = dv_c1.div(rem), c = rem - r * C1r;
    const int g1 = c1lo + c, g2 = c2lo + r;
    xsi[i] = pl * a.cmax1 * a.cmax2 + rem;
    xpl[i] = pl;
    xgo[i] = ((int64_t)pl * n2 + g2) * n1 + g1;
    xin[i] = g1 < n1 && g2 < n2;
  }
  auto slab_fetch = [&](int p0, int np) {
    const int64_t pbase = (int64_t)p0 * n2 * n1;
#pragma unroll
    for (int i = 0; i < XPF; ++i) {
      const int e = tid + i * NT;
      T v = T(0);
      if (e < np * perx) {
        const int c3 = p0 + xpl[i];
        if (c3 < n3 && xin[i]) v = __ldg(x + pbase + xgo[i]);
      }
      xpf[i] = v;
    }
  };
  auto slab_store = [&](int p0, int np) {
    const int per = perx;
#pragma unroll
    for (int i = 0; i < XPF; ++i) {
      const int e = tid + i * NT;
      if (e < np * per) xs[xsi[i]] = xpf[i];
    }
    for (int e = tid + XPF * NT; e < np * per; e += NT) {
      const int pl = dv_perx.div(e), rem = e - pl * per;
      const int r = dv_c1.div(rem), c = rem - r * C1r;
      const int c3 = p0 + pl, g1 = c1lo + c, g2 = c2lo + r;
      T v = T(0);
      if (c3 < n3 && g1 < n1 && g2 < n2) v = __ldg(x + ((int64_t)c3 * n2 + g2) * n1 + g1);
      xs[pl * a.cmax1 * a.cmax2 + rem] = v;
    }
  };
  // produce trial planes p0 .. p0+np-1 (np <= QC) into the staging ring from
  // the slab in xs; each thread ends with its own (q1, q2) entries of every
  // needed combo
  // stage 1: dir-1 contraction of the slab (xs -> a1s)
  auto produce_st1 = [&](int np) {
    // this lx's band values, read once for all rows
    T bv[2 * W];
#pragma unroll
    for (int m = 0; m < 2 * W; ++m) bv[m] = b1tab[m * FX + lx];
#pragma unroll 2
    for (int rr = ly; rr < np * C2r; rr += FY) {
      const int pl = dv_c2.div(rr), r = rr - pl * C2r;
      const T* xr = xs + pl * a.cmax1 * a.cmax2 + r * C1r + s1rel;
      T v0 = T(0), v1 = T(0);
#pragma unroll
      for (int k = 0; k < W; ++k) {
        const T xv = xr[k];
        if (P::b1_needed(0)) v0 += bv[k] * xv;
        if (P::b1_needed(1)) v1 += bv[W + k] * xv;
      }
      T* dst = a1s + ((size_t)pl * NB1 * a.cmax2 + r) * FX + lx;
      if (P::b1_needed(0)) dst[b1_slot<P>(0) * a.cmax2 * FX] = v0;
      if (P::b1_needed(1)) dst[b1_slot<P>(1) * a.cmax2 * FX] = v1;
    }
  };
  // stage 2: dir-2 contraction (a1s -> this thread's stage entries)
  auto produce_st2 = [&](int p0, int np) {
    const T* b2v = b2tab + ly * 2 * W;
    for (int pl = 0; pl < np; ++pl) {
      const int slot = (p0 + pl) % QC;
      // each dir-1 result column is loaded once and used by every combo
      // that shares it
#pragma unroll
      for (int b1 = 0; b1 < 2; ++b1) {
        if (!P::b1_needed(b1)) continue;
        const T* src = a1s + ((size_t)(pl * NB1 + b1_slot<P>(b1)) * a.cmax2 + s2rel) * FX + lx;
        T xw[W];
#pragma unroll
        for (int k = 0; k < W; ++k) xw[k] = src[k * FX];
#pragma unroll
        for (int b2 = 0; b2 < 2; ++b2) {
          const int c = b1 | (b2 << 1);
          if (!P::combo_needed(c)) continue;
          T v = T(0);
#pragma unroll
          for (int k = 0; k < W; ++k) v += b2v[b2 * W + k] * xw[k];
          stage[(slot * NCOMBO + combo_slot<P>(c)) * NT + tid] = v;
        }
      }
    }
  };

  // contract final test planes lo .. lo+np-1 (np <= QC) over q2 (stage 1,
  // done -> ks) and q1 (stage 2, ks -> y)
  auto flush_st1 = [&](int lo, int np) {
    if constexpr (Depth3<T, P>::q2_dmma()) {
      // per (plane, g, 8-row block of r2, 8-wide half of the face):
      // ks[g][r2][lx] = sum over the pairs (b, g) of
      //                 sum_l2 w2d[b][r2][l2] done[pair][l2][lx]
      const int MT = (D2r + 7) >> 3;
      for (int task = warp; task < np * NG * MT * 2; task += NT / 32) {
        const int nt = task & 1;
        const int rest0 = task >> 1;
        const int rest = dv_mt.div(rest0), mt = rest0 - rest * MT;
        const int gs = rest % NG, pl = rest / NG;
        const int g = (NG == 2) ? gs : (P::a1_needed(0) ? 0 : 1);
        const T* dn = done + (size_t)((lo + pl) % QC) * NPAIR * NT;
        const int r2 = mt * 8 + gq, r2c = min(r2, a.dmax2 - 1);
        const int n = nt * 8 + gq;
        double cc[4][2];
#pragma unroll
        for (int pr = 0; pr < 4; ++pr) cc[pr][0] = cc[pr][1] = 0.0;
#pragma unroll
        for (int pr = 0; pr < 4; ++pr) {
          if (!P::tpair_needed(pr)) continue;
          if ((pr & 1) != g) continue;
          const T* wa = w2d + ((pr >> 1) * a.dmax2 + r2c) * W2S;
          const T* db = dn + pair_slot<P>(pr) * NT;
#pragma unroll
          for (int kt = 0; kt < FY / 4; ++kt) {
            const int l2 = kt * 4 + tq;
            dmma_8x8x4(cc[pr][0], cc[pr][1], wa[l2], db[l2 * FX + swz<T>(n, l2)]);
          }
        }
        if (r2 < D2r) {
          double c0 = 0.0, c1 = 0.0;
#pragma unroll
          for (int pr = 0; pr < 4; ++pr) {
            c0 += cc[pr][0];
            c1 += cc[pr][1];
          }
          T* kd = ks + ((size_t)(pl * NG + gs) * a.dmax2 + r2) * KS;
          *reinterpret_cast<double2*>(kd + swz<T>(nt * 8 + 2 * tq, r2)) = make_double2(c0, c1);
        }
      }
    } else {
      for (int it = ly; it < np * D2r; it += FY) {
        const int pl = dv_d2.div(it), r = it - pl * D2r;
        const T* dn = done + (size_t)((lo + pl) % QC) * NPAIR * NT + lx;
        const T* wr = w2d + r * W2S;
        // dense over the tile's q2 points, one accumulator per (pair, parity)
        T kp[4][2];
  #pragma unroll
        for (int pr = 0; pr < 4; ++pr) kp[pr][0] = kp[pr][1] = T(0);
  #pragma unroll
        for (int l2 = 0; l2 < FY; ++l2) {
          T wa0, wa1;
          ld2(wr + 2 * l2, wa0, wa1);
  #pragma unroll
          for (int pr = 0; pr < 4; ++pr) {
            if (!P::tpair_needed(pr)) continue;
            kp[pr][l2 & 1] += ((pr >> 1) ? wa1 : wa0) * dn[pair_slot<P>(pr) * NT + l2 * FX];
          }
        }
        T kv0 = T(0), kv1 = T(0);
  #pragma unroll
        for (int pr = 0; pr < 4; ++pr) {
          if (!P::tpair_needed(pr)) continue;
          if (pr & 1)
            kv1 += kp[pr][0] + kp[pr][1];
          else
            kv0 += kp[pr][0] + kp[pr][1];
        }
        T* kd = ks + ((size_t)pl * NG * a.dmax2 + r) * KS + swz<T>(lx, r);
        if (P::a1_needed(0)) kd[g_slot<P>(0) * a.dmax2 * KS] = kv0;
        if (P::a1_needed(1)) kd[g_slot<P>(1) * a.dmax2 * KS] = kv1;
      }
    }
  };
  auto flush_st2 = [&](int lo, int np) {
    if constexpr (use_dmma<T>()) {
      // per (plane, 8-row block of r2, 8-column block of r1):
      // y[r2][r1] += sum_g sum_l1 ks[g][r2][l1] w1d[r1][g][l1]
      const int MT = (D2r + 7) >> 3, NT1 = (D1r + 7) >> 3;
      for (int task = warp; task < np * MT * NT1; task += NT / 32) {
        const int rest = dv_nt1.div(task), nt = task - rest * NT1;
        const int pl = dv_mt.div(rest), mt = rest - pl * MT;
        const int r2 = mt * 8 + gq, r2c = min(r2, a.dmax2 - 1);
        const int r1b = nt * 8 + gq, r1c = min(r1b, a.dmax1 - 1);
        double c0 = 0.0, c1 = 0.0;
#pragma unroll
        for (int gs = 0; gs < NG; ++gs) {
          const int g = (NG == 2) ? gs : (P::a1_needed(0) ? 0 : 1);
          const T* ka = ks + ((size_t)(pl * NG + gs) * a.dmax2 + r2c) * KS;
          const T* wb = w1d + r1c * W1S + g * FX;
#pragma unroll
          for (int kt = 0; kt < FX / 4; ++kt) {
            const int l1 = kt * 4 + tq;
            dmma_8x8x4(c0, c1, ka[swz<T>(l1, r2c)], wb[swz<T>(l1, r1c)]);
          }
        }
        if (r2 < D2r) {
          T* yr = y + ((int64_t)(lo + pl) * n2 + d2lo + r2) * n1 + d1lo;
          const int r1 = nt * 8 + 2 * tq;
          if (r1 < D1r && c0 != 0.0) atomicAdd(yr + r1, c0);
          if (r1 + 1 < D1r && c1 != 0.0) atomicAdd(yr + r1 + 1, c1);
        }
      }
    } else {
      const int per = perf;
      for (int e = tid; e < np * per; e += NT) {
        const int pl = dv_perf.div(e), rem = e - pl * per;
        const int r2 = dv_d1.div(rem), r1 = rem - r2 * D1r;
        const int c1p = d1lo + r1;
        const T* kr = ks + ((size_t)pl * NG * a.dmax2 + r2) * KS;
        const T* wc = w1d + r1 * W1S;
        // dense over the tile's q1 points
        T va[2] = {T(0), T(0)}, vb[2] = {T(0), T(0)};
#pragma unroll
        for (int l1 = 0; l1 < FX; ++l1) {
          if (P::a1_needed(0)) va[l1 & 1] += wc[l1] * kr[g_slot<P>(0) * a.dmax2 * KS + l1];
          if (P::a1_needed(1)) vb[l1 & 1] += wc[FX + l1] * kr[g_slot<P>(1) * a.dmax2 * KS + l1];
        }
        const T v = (va[0] + va[1]) + (vb[0] + vb[1]);
        if (v != T(0)) atomicAdd(y + ((int64_t)(lo + pl) * n2 + d2lo + r2) * n1 + c1p, v);
      }
    }
  };

  // retire the oldest test plane of the window into the done ring (own entries)
  T acc[I][W];
#pragma unroll
  for (int i = 0; i < I; ++i)
#pragma unroll
    for (int k = 0; k < W; ++k) acc[i][k] = T(0);
  auto retire = [&](int dslot) {  // dslot = the plane's index mod QC
    T* dn = done + (size_t)dslot * NPAIR * NT +
            (Depth3<T, P>::q2_dmma() ? ly * FX + swz<T>(lx, ly) : tid);
#pragma unroll
    for (int pr = 0; pr < 4; ++pr) {
      if (!P::tpair_needed(pr)) continue;
      T v = T(0);
#pragma unroll
      for (int i = 0; i < I; ++i)
        if (P::tpair(i) == pr) v += acc[i][0];
      dn[pair_slot<P>(pr) * NT] = valid ? v : T(0);
    }
#pragma unroll
    for (int i = 0; i < I; ++i) {
#pragma unroll
      for (int k = 0; k < W - 1; ++k) acc[i][k] = acc[i][k + 1];
      acc[i][W - 1] = T(0);
    }
  };

  // trial window: F[combo][k] = A_combo(q1, q2, fbase + k)
  T F[NCOMBO][W];
  int fbase = __ldg(a.tstart[2] + qa);
  slab_fetch(fbase, W);
  slab_store(fbase, W);
  named_sync(1, NT);
  produce_st1(W);
  named_sync(1, NT);
  produce_st2(fbase, W);
  int produced_hi = fbase + W;
#pragma unroll
  for (int k = 0; k < W; ++k) {
    const int slot = (fbase + k) % QC;
#pragma unroll
    for (int c = 0; c < NCOMBO; ++c) F[c][k] = stage[(slot * NCOMBO + c) * NT + tid];
  }
  // aliased buffers: the first chunk's slab overwrites the staging ring
  if constexpr (Depth3<T, P>::alias(W)) named_sync(1, NT);
  int abase = __ldg(a.wtstart[2] + qa);
  // ring positions (mod QC) of the oldest test plane and of the next trial
  // plane (light patterns: advanced with the windows)
  int aslot = abase % QC;
  int fslot = (fbase + W) % QC;
  int flush_lo = abase;
  bool aborted = false;

  const int nchunk = (L + QC - 1) / QC;
  int pf_lo = produced_hi, pf_n = 0;  // slab prefetched for the coming chunk
  {
    const int need0 = __ldg(a.tstart[2] + qa + min(QC, L) - 1) + W;
    if (need0 > produced_hi) {
      pf_n = need0 - produced_hi;
      slab_fetch(pf_lo, pf_n);
    }
  }
  // trial planes needed by the chunk after next, loaded one chunk ahead
  int need_nx = __ldg(a.tstart[2] + qa + min(2 * QC, L) - 1) + W;
  int fl_lo = 0, fl_n = 0;  // planes of the previous chunk waiting for their flush
  for (int ch = 0; ch < nchunk; ++ch) {
    const int tb = ch * QC, te = min(tb + QC, L);
    // the previous chunk's flush and this chunk's plane production share
    // two barrier intervals (they touch disjoint buffers)
    if (fl_n > 0) flush_st1(fl_lo, fl_n);
    if (pf_n > 0) slab_store(pf_lo, pf_n);
    named_sync(1, NT);
    if (fl_n > 0) flush_st2(fl_lo, fl_n);
    if (pf_n > 0) produce_st1(pf_n);
    named_sync(1, NT);
    if (pf_n > 0) {
      produce_st2(pf_lo, pf_n);
      produced_hi = pf_lo + pf_n;
    }
    // prefetch the slab of the next chunk while this one computes
    pf_lo = produced_hi;
    pf_n = 0;
    if (ch + 1 < nchunk) {
      const int need_next = need_nx;
      if (ch + 2 < nchunk) need_nx = __ldg(a.tstart[2] + qa + min(te + 2 * QC, L) - 1) + W;
      if (need_next > produced_hi) {
        pf_n = need_next - produced_hi;
        slab_fetch(pf_lo, pf_n);
      }
    }
    // aliased buffers: the points' retirements overwrite the q1 production
    // buffer that the q2 production above still reads in other warps
    if constexpr (Depth3<T, P>::alias(W)) named_sync(1, NT);
    if (!aborted) {
      const uint64_t limit = a.wait_test ? kWaitTestLimitNs : kWaitLimitNs;
      for (int t = tb; t < te; ++t) {
        if (!mbar_wait_bounded_ns(smem_u32(&full[t % NST]), (uint32_t)((t / NST) & 1), limit)) {
          aborted = true;
          atomicExch(&s_abort, 1);
          break;
        }
      }
    }
    const T* cchunk = cring + (tb % NST) * slot_elems;
    auto step = [&](const int t) {
      const T* cs = kRunSlots ? cchunk + (t - tb) * slot_elems : cring + (t % NST) * slot_elems;
      const T* row = cs + S * NT;  // step table row of q3 = qa + t
      constexpr int G = (W + 16 / sizeof(T) - 1) / (16 / sizeof(T)) * (16 / sizeof(T));
      T tsv, wsv;
      ld2(row + 4 * G, tsv, wsv);  // band starts, one 16-byte load
      const int ts = step_start(tsv);
      const int ws = step_start(wsv);
      // this point's coefficients, loaded ahead of the window moves
      T cv[S];
      if constexpr (point_major3(S)) {
        const T* cp = cs + (ly * w1 + lx) * S;
#pragma unroll
        for (int s = 0; s < S; s += 2) ld2(cp + s, cv[s], cv[s + 1]);
      } else {
        const int fsz = w1 * w2;
        const T* cp = cs + ly * w1 + lx;
#pragma unroll
        for (int s = 0; s < S; ++s) cv[s] = cp[s * fsz];
      }
      // the test window first (its oldest plane may be final), then the
      // trial window; band starts advance by at most one plane per point
      // (the plan checks this), so each window moves at most once
      if (abase < ws) {
        retire(kRunSlots ? aslot : abase % QC);
        ++abase;
        if constexpr (kRunSlots) aslot = (aslot + 1 == QC) ? 0 : aslot + 1;
      }
      if (fbase < ts) {
        const int ps = kRunSlots ? fslot : (fbase + W) % QC;
#pragma unroll
        for (int c = 0; c < NCOMBO; ++c) {
#pragma unroll
          for (int m = 0; m < W - 1; ++m) F[c][m] = F[c][m + 1];
          F[c][W - 1] = stage[(ps * NCOMBO + c) * NT + tid];
        }
        ++fbase;
        if constexpr (kRunSlots) fslot = (fslot + 1 == QC) ? 0 : fslot + 1;
      }
      // band values and coefficients are read from the ring slot where they
      // are used (broadcast / coalesced shared loads), so that few values
      // stay live in registers; the slot is released after the last read
      T u[J];
#pragma unroll
      for (int j = 0; j < J; ++j) {
        T bq[G];
        load_group<T, G>(row + P::beta(j, 2) * G, bq);
        const T* f = F[combo_slot<P>(P::combo(j))];
        T v0 = bq[0] * f[0], v1 = bq[1] * f[1];
#pragma unroll
        for (int k = 2; k < W; ++k) {
          if (k & 1)
            v1 += bq[k] * f[k];
          else
            v0 += bq[k] * f[k];
        }
        u[j] = v0 + v1;
      }
#pragma unroll
      for (int i = 0; i < I; ++i) {
        T g = T(0);
#pragma unroll
        for (int j = 0; j < J; ++j) g += cv[P::cidx(i, j)] * u[j];
        if (!valid) g = T(0);
        T wq[G];
        load_group<T, G>(row + (2 + P::alpha(i, 2)) * G, wq);
#pragma unroll
        for (int k = 0; k < W; ++k) acc[i][k] += wq[k] * g;
      }
        };
    // light patterns: a full chunk is unrolled (the next point's loads are
    // scheduled across the window moves); heavy ones keep the loop (registers)
    if (!Depth3<T, P>::heavy && te - tb == QC) {
#pragma unroll
      for (int k = 0; k < QC; ++k) step(tb + k);
    } else {
      for (int t = tb; t < te; ++t) step(t);
    }
    named_sync(1, NT);
    if (*(volatile int*)&s_abort) aborted = true;
    if (aborted) break;  // uniform: every thread read s_abort after the barrier
    // every thread is done with this chunk's slots: stream the points up to
    // RA past it into them
    if (issued_hi < min(te + RA, L)) issue(issued_hi, min(te + RA, L));
    fl_lo = flush_lo;
    fl_n = abase - flush_lo;
    flush_lo = abase;
  }
  if (aborted) {
    if (tid == 0) {
      // the copies still in flight land before the CTA exits (the withheld
      // copy of the wait test hook was never issued)
      for (int t = max(0, issued_hi - NST); t < issued_hi; ++t)
        if (!(a.wait_test && t == 0))
          (void)mbar_wait_bounded(smem_u32(&full[t % NST]), (uint32_t)((t / NST) & 1));
      report_status(a.status, IGA_ERR_TIMEOUT);
    }
    return;
  }
  if (fl_n > 0) {
    flush_st1(fl_lo, fl_n);
    named_sync(1, NT);
    flush_st2(fl_lo, fl_n);
  }
  // the planes still in the window are final
  named_sync(1, NT);
  int nfin = 0;
#pragma unroll
  for (int k = 0; k < W; ++k) {
    if (abase + k < n3) ++nfin;
  }
#pragma unroll
  for (int k = 0; k < W; ++k) retire((abase + k) % QC);
  named_sync(1, NT);
  if (nfin > 0) {
    flush_st1(abase, nfin);
    named_sync(1, NT);
    flush_st2(abase, nfin);
  }
}

// One patch: CTA blockIdx.x is work unit (tile, segment), blockIdx.y the column.
template <typename T, int FX, int FY, int W, class P>
__global__ void __launch_bounds__(FX* FY, Depth3<T, P>::minb(W))
    mf3d_kernel(const __grid_constant__ FusedArgs<T> a) {
  mf3d_body<T, FX, FY, W, P>(a, blockIdx.x, blockIdx.y);
}

// Many patches of one pattern and band width in one launch: patch p owns CTAs
// [cta0[p], cta0[p+1]); its arguments args[p] are copied to shared memory and
// its vectors sit at element offset offs[p] of the flat x / y.
template <typename T, int FX, int FY, int W, class P>
__global__ void __launch_bounds__(FX* FY, Depth3<T, P>::minb(W))
    mf3d_batch_kernel(const FusedArgs<T>* __restrict__ args, const int32_t* __restrict__ cta0,
                      int npatch, const int64_t* __restrict__ offs, const T* xb, T* yb,
                      const int32_t* __restrict__ skip) {
  __shared__ FusedArgs<T> sa;
  __shared__ int sp;
  if (threadIdx.x == 0) {
    int lo = 0, hi = npatch;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (__ldg(cta0 + mid) <= (int)blockIdx.x) lo = mid;
      else hi = mid;
    }
    sp = lo;
  }
  __syncthreads();
  const int p = sp;
  if (skip && __ldg(skip + p) >= 0) return;  // patch done: its output stays zero
  {
    const int* src = reinterpret_cast<const int*>(args + p);
    int* dst = reinterpret_cast<int*>(&sa);
    for (int i = threadIdx.x; i < (int)(sizeof(FusedArgs<T>) / sizeof(int)); i += blockDim.x)
      dst[i] = src[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    sa.x = xb + offs[p];
    sa.y = yb + offs[p];
  }
  __syncthreads();
  mf3d_body<T, FX, FY, W, P>(sa, (int)blockIdx.x - __ldg(cta0 + p), 0);
}

// ===================================================================== 2D
template <typename T, int FX, int W, int NST, class P>
__global__ void __launch_bounds__(FX) mf2d_kernel(const __grid_constant__ FusedArgs<T> a) {
  constexpr int S = P::S;
  constexpr int I = P::I;
  constexpr int J = P::J;

  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);
  T* cring = reinterpret_cast<T*>(smem_raw + 128);
  T* hs = cring + NST * S * FX;  // [2][FX]

  const int tid = threadIdx.x;
  const int n1 = a.n[0], n2 = a.n[1];
  const int nq1 = a.nq[0], nq2 = a.nq[1];
  const int unit = blockIdx.x;
  const int seg = unit % a.nseg;
  const int t1 = unit / a.nseg;
  const T* __restrict__ x = a.x + (int64_t)blockIdx.y * a.N;
  T* __restrict__ y = a.y + (int64_t)blockIdx.y * a.N;

  const int q1lo = t1 * FX, w1 = min(FX, nq1 - q1lo);
  const bool valid = tid < w1;
  const int q1 = q1lo + min(tid, w1 - 1);
  const int qa = (int)((int64_t)nq2 * seg / a.nseg);
  const int qb = (int)((int64_t)nq2 * (seg + 1) / a.nseg);
  const int L = qb - qa;
  const int d1lo = __ldg(a.wtstart[0] + q1lo);
  const int D1r = min(__ldg(a.wtstart[0] + q1lo + w1 - 1) + W - 1, n1 - 1) - d1lo + 1;

  T b1c[2][W];
  const int s1 = __ldg(a.tstart[0] + q1);
#pragma unroll
  for (int k = 0; k < W; ++k) {
    b1c[0][k] = __ldg(a.tB0[0] + (int64_t)q1 * W + k);
    b1c[1][k] = P::b1_needed(1) ? __ldg(a.tB1[0] + (int64_t)q1 * W + k) : T(0);
  }

  const int64_t cstride = chunk_stride_elems<T>(S, w1, 1);
  const uint32_t cbytes = (uint32_t)(cstride * sizeof(T));
  const T* cbase = a.packed + __ldg(a.tile_off + t1);

  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < NST; ++s) mbar_init(smem_u32(&bars[s]), 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (tid == 0) {
    for (int s = 0; s < NST && s < L; ++s) {
      const uint32_t bar = smem_u32(&bars[s]);
      mbar_arrive_expect_tx(bar, cbytes);
      bulk_g2s(smem_u32(cring + s * S * FX), cbase + (int64_t)(qa + s) * cstride, cbytes, bar);
    }
  }

  auto produce = [&](int c2, T out[2]) {
#pragma unroll
    for (int b = 0; b < 2; ++b) out[b] = T(0);
    if (c2 >= n2) return;
#pragma unroll
    for (int k = 0; k < W; ++k) {
      const int c1 = s1 + k;
      const T xv = (c1 < n1) ? __ldg(x + (int64_t)c2 * n1 + c1) : T(0);
      out[0] += b1c[0][k] * xv;
      if (P::b1_needed(1)) out[1] += b1c[1][k] * xv;
    }
  };

  auto flush = [&](int cp, const T (&g0)[I]) {
#pragma unroll
    for (int g = 0; g < 2; ++g) {
      if (!P::a1_needed(g)) continue;
      T v = T(0);
#pragma unroll
      for (int i = 0; i < I; ++i)
        if (P::alpha(i, 0) == g) v += g0[i];
      hs[g * FX + tid] = valid ? v : T(0);
    }
    __syncthreads();
    for (int e = tid; e < D1r; e += FX) {
      const int c1p = d1lo + e;
      const int rs = __ldg(a.rstart[0] + c1p);
      T v = T(0);
      for (int k = 0; k < a.RW; ++k) {
        const int l1 = rs + k - q1lo;
        if (l1 < 0 || l1 >= w1) continue;
        if (P::a1_needed(0)) v += __ldg(a.wR0[0] + (int64_t)c1p * a.RW + k) * hs[l1];
        if (P::a1_needed(1)) v += __ldg(a.wR1[0] + (int64_t)c1p * a.RW + k) * hs[FX + l1];
      }
      if (v != T(0)) atomicAdd(y + (int64_t)cp * n1 + c1p, v);
    }
    __syncthreads();
  };

  T F[2][W];
  int fbase = __ldg(a.tstart[1] + qa);
#pragma unroll
  for (int k = 0; k < W; ++k) {
    T out[2];
    produce(fbase + k, out);
    F[0][k] = out[0];
    F[1][k] = out[1];
  }
  T acc[I][W];
#pragma unroll
  for (int i = 0; i < I; ++i)
#pragma unroll
    for (int k = 0; k < W; ++k) acc[i][k] = T(0);
  int abase = __ldg(a.wtstart[1] + qa);

  for (int t = 0; t < L; ++t) {
    const int q2 = qa + t;
    const int ws = __ldg(a.wtstart[1] + q2);
    while (abase < ws) {
      if (abase < n2) {
        T g0[I];
#pragma unroll
        for (int i = 0; i < I; ++i) g0[i] = acc[i][0];
        flush(abase, g0);
      }
#pragma unroll
      for (int i = 0; i < I; ++i) {
#pragma unroll
        for (int k = 0; k < W - 1; ++k) acc[i][k] = acc[i][k + 1];
        acc[i][W - 1] = T(0);
      }
      ++abase;
    }
    const int ts = __ldg(a.tstart[1] + q2);
    while (fbase < ts) {
      T out[2];
      produce(fbase + W, out);
#pragma unroll
      for (int b = 0; b < 2; ++b) {
#pragma unroll
        for (int k = 0; k < W - 1; ++k) F[b][k] = F[b][k + 1];
        F[b][W - 1] = out[b];
      }
      ++fbase;
    }
    const int slot = t % NST;
    const bool ok = mbar_wait_bounded(smem_u32(&bars[slot]), (uint32_t)((t / NST) & 1));
    const T* cs = cring + slot * S * FX;
    T u[J];
#pragma unroll
    for (int j = 0; j < J; ++j) {
      const T* bp = (P::beta(j, 1) ? a.tB1[1] : a.tB0[1]) + (int64_t)q2 * W;
      T v = T(0);
#pragma unroll
      for (int k = 0; k < W; ++k) v += __ldg(bp + k) * F[P::beta(j, 0)][k];
      u[j] = v;
    }
    T cv[S];
#pragma unroll
    for (int s = 0; s < S; ++s) cv[s] = valid ? cs[s * w1 + tid] : T(0);
#pragma unroll
    for (int i = 0; i < I; ++i) {
      T g = T(0);
#pragma unroll
      for (int j = 0; j < J; ++j) g += cv[P::cidx(i, j)] * u[j];
      const T* wp = (P::alpha(i, 1) ? a.wT1[1] : a.wT0[1]) + (int64_t)q2 * W;
#pragma unroll
      for (int k = 0; k < W; ++k) acc[i][k] += __ldg(wp + k) * g;
    }
    const bool all_ok = __syncthreads_and(ok);
    if (!all_ok) {
      if (tid == 0) {
        report_status(a.status, IGA_ERR_TIMEOUT);
        for (int s = 1; s < NST && t + s < L; ++s)
          (void)mbar_wait_bounded(smem_u32(&bars[(t + s) % NST]), (uint32_t)(((t + s) / NST) & 1));
      }
      __syncthreads();
      return;
    }
    if (tid == 0 && t + NST < L) {
      const uint32_t bar = smem_u32(&bars[slot]);
      mbar_arrive_expect_tx(bar, cbytes);
      bulk_g2s(smem_u32(cring + slot * S * FX), cbase + (int64_t)(q2 + NST) * cstride, cbytes, bar);
    }
  }
#pragma unroll
  for (int k = 0; k < W; ++k) {
    if (abase + k < n2) {
      T g0[I];
#pragma unroll
      for (int i = 0; i < I; ++i) g0[i] = acc[i][k];
      flush(abase + k, g0);
    }
  }
}

// ----------------------------------------------------------- launching
struct LaunchInfo {
  int ndim, op, st, tt, tr, sym, W;
  int FX, FY, NST;
  int64_t ncols;
  cudaStream_t stream;
};

// One object file per (dimension, element type, band width); see mf_inst.cu.
#define IGA_DECL_LAUNCH(D, TN, T, W) \
  iga_status launch_mf##D##_##TN##_w##W(const FusedArgs<T>& a, const LaunchInfo& li);
#define IGA_DECL_ALL_W(D, TN, T) \
  IGA_DECL_LAUNCH(D, TN, T, 3)   \
  IGA_DECL_LAUNCH(D, TN, T, 4)   \
  IGA_DECL_LAUNCH(D, TN, T, 5)   \
  IGA_DECL_LAUNCH(D, TN, T, 6)
// Multi-patch 3D launch (all patches share op, symmetry and band width).
struct BatchLaunch {
  int op, sym, W;
  int npatch, total_ctas;
  size_t smem;
  const void* args;     // device FusedArgs<T>[npatch]
  const int32_t* cta0;  // device [npatch + 1]
  const int64_t* offs;  // device [npatch]
  const int32_t* skip;  // device [npatch] or null: patches with skip[p] >= 0 are not computed
  cudaStream_t stream;
};
#define IGA_DECL_BATCH(TN, T, W) \
  iga_status launch_mf3_batch_##TN##_w##W(const BatchLaunch& b, const T* x, T* y);
#define IGA_DECL_BATCH_W(TN, T) \
  IGA_DECL_BATCH(TN, T, 3)      \
  IGA_DECL_BATCH(TN, T, 4)      \
  IGA_DECL_BATCH(TN, T, 5)      \
  IGA_DECL_BATCH(TN, T, 6)
IGA_DECL_BATCH_W(f64, double)
IGA_DECL_BATCH_W(f32, float)
#undef IGA_DECL_BATCH_W
#undef IGA_DECL_BATCH

IGA_DECL_ALL_W(2, f64, double)
IGA_DECL_ALL_W(3, f64, double)
IGA_DECL_ALL_W(2, f32, float)
IGA_DECL_ALL_W(3, f32, float)
#undef IGA_DECL_ALL_W
#undef IGA_DECL_LAUNCH

// Face tile and pipeline depth of the compiled kernels.
constexpr int kFace3X = 16, kFace3Y = 8, kFace2X = 128, kStages = 4;

}  // namespace iga
