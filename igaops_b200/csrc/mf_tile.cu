// Tensor-core 3D matrix-free operator (FP64): stiffness with symmetric
// coefficients and mass, one persistent CTA per SM.
//
// Computes y = sum_i W^{(alpha_i)} [ sum_j C_ij (B^{(beta_j)} x) ], the
// arithmetic of BsplineOperations.compute_mf_scalar_gradu_gradv /
// compute_mf_scalar_u_v (src/igaops/operators/bsplines_ops.py:290-355), as
// sum factorisation over 3D tiles of 16 x 8 x 16 quadrature points.  Along
// each direction a tile's points form groups of 8 whose trial and test bands
// lie in windows of 8 control points (the host checks this,
// igaops_b200/tile3d.py), so every 1D contraction of a tile is a set of
// 8 x 8 x (2 x 4) FP64 tensor-core products (mma.sync.m8n8k4.f64; the A
// operand from shared memory, the B operand -- the 1D factor window -- from a
// fragment table in register order):
//
//   stage 1  T1_b  [d3][d2][q1] = B_b^(1)  X            b = 0, 1
//   stage 2  T2_c  [d3][q2][q1] = B^(2)    T1           c = 00, 10, 01
//   stage 3  per (q1, q2) row block: U_j = B^(3) T2 (products), V_i =
//            sum_j C_ij U_j (coefficients from a TMA ring), Y3_i = W^(3) V_i
//            with V_i passed register to register: the product's output
//            layout is the next product's input layout once the test
//            contraction takes the group's even / odd points as its k-steps
//   stage 4  Y2 = W^(2) Y3      stage 5  Y1 = W^(1) Y2
//   stage 6  y += Y1 (FP64 atomics: neighbouring tiles share control points)
//
// Shared-memory buffers of the stages are laid out (with XOR swizzles of
// the 16-wide q1 rows) so that every fragment load and store runs at the
// minimum number of wavefronts.  The coefficients stream once from HBM: per
// warp a ring of NSLOT units (8 rows x 8 q3 points x S streams, in the order
// the mixing step reads them), each one 1D bulk copy (cp.async.bulk, no
// multicast) completing on an mbarrier; every wait is bounded.
#include "common.cuh"

namespace iga {
namespace mft {

constexpr int NCWARP = 8;  // compute warps
constexpr int NTHR = NCWARP * 32;
constexpr int GEOM = 16;
enum { G_QA = 0, G_Q, G_XA, G_YA, G_DX, G_DY, G_TW0, G_TW1, G_SW0, G_SW1, G_NG, G_CUM, G_WT };
// allocated control-point extents of a tile (directions 1, 2, 3)
constexpr int XP1 = 12, XP2 = 8, XP3 = 12;
constexpr int XS = XP3 * XP2 * XP1;        // X / Y1 box (doubles)
constexpr int FR = 5 * 256;                // fragment slots of a tile
constexpr int T1S = 2 * XP3 * XP2 * 16;    // T1 / Y2
constexpr int T2S = 3 * XP3 * 8 * 16;      // T2 / Y3

template <int OP>
struct Cfg {
  static constexpr bool kMass = OP == IGA_OP_MASS;
  static constexpr int S = kMass ? 1 : 6;
  static constexpr int UE = 2 * S * 32;         // doubles per coefficient unit
  static constexpr int NSLOT = kMass ? 12 : 4;  // ring depth per warp
};

struct Args {
  int32_t n[3], nq[3], ntile[3], wsum[3];
  int32_t src_row[6];
  const int32_t* geom;
  const double* frag;
  const double* packed;
  const double* x;
  double* y;
  int32_t* status;
};

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// q1 column of the [plane][q2][16] buffers (T2 / Y3): half-row swap keyed
// by plane and q2 so that 4 consecutive planes, or the 4 even / odd q2 of a
// fragment, land in both halves of the 32 banks
__device__ __forceinline__ int swz2(int q1, int p, int q2) {
  return q1 ^ (((p ^ (p >> 1) ^ (q2 >> 1)) & 1) << 3);
}

// (direction k, tile t) record in shared memory
__device__ __forceinline__ const int32_t* rec(const int32_t* g, const Args& a, int k, int t) {
  const int off = k == 0 ? 0 : (k == 1 ? a.ntile[0] : a.ntile[0] + a.ntile[1]);
  return g + (off + t) * GEOM;
}

__device__ __forceinline__ void tile_coords(const Args& a, int t, int& t1, int& t2, int& t3) {
  t1 = t % a.ntile[0];
  const int r = t / a.ntile[0];
  t2 = r % a.ntile[1];
  t3 = r / a.ntile[1];
}

// element offset of the first coefficient unit of tile (t1, t2, t3); units of
// a tile are ordered [m-tile][q3 group]; m-tile = q2 * H + h
__device__ __forceinline__ int64_t tile_units(const int32_t* g, const Args& a, int t1, int t2,
                                              int t3) {
  const int32_t* r1 = rec(g, a, 0, t1);
  const int32_t* r2 = rec(g, a, 1, t2);
  const int32_t* r3 = rec(g, a, 2, t3);
  const int64_t SH = a.wsum[0], SQ2 = a.wsum[1];
  return (int64_t)r3[G_CUM] * SQ2 * SH +
         (int64_t)r3[G_WT] * ((int64_t)r2[G_CUM] * SH + (int64_t)r2[G_WT] * r1[G_CUM]);
}

// Walks one consumer warp's coefficient units in the order stage 3 consumes
// them (this CTA's tiles, the warp's m-tiles, q3 groups); the tile decode
// (divisions) runs once per tile, not per unit.
struct UnitWalk {
  int t, mt, nt, NT, nmt;
  int64_t base;  // element offset of the tile's first unit
  bool valid;
  __device__ void seek(const int32_t* g, const Args& a, int warp, int ntiles, int UE) {
    // first tile from t on in which the warp owns an m-tile
    while (t < ntiles) {
      int t1, t2, t3;
      tile_coords(a, t, t1, t2, t3);
      nmt = rec(g, a, 1, t2)[G_WT] * rec(g, a, 0, t1)[G_WT];
      if (warp < nmt) {
        NT = rec(g, a, 2, t3)[G_WT];
        base = tile_units(g, a, t1, t2, t3) * UE;
        mt = warp;
        nt = 0;
        valid = true;
        return;
      }
      t += gridDim.x;
    }
    valid = false;
  }
  __device__ __forceinline__ void advance(const int32_t* g, const Args& a, int warp, int ntiles,
                                          int UE) {
    if (++nt < NT) return;
    nt = 0;
    mt += NCWARP;
    if (mt < nmt) return;
    t += gridDim.x;
    seek(g, a, warp, ntiles, UE);
  }
  __device__ __forceinline__ int64_t offset(int UE) const {
    return base + (int64_t)(mt * NT + nt) * UE;
  }
};

__device__ __forceinline__ void cp_async_mbar_arrive_noinc(uint32_t bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(bar) : "memory");
}

// Barrier among the consumer warps (named barrier 1).
__device__ __forceinline__ void consumers_sync() { named_sync(1, NCWARP * 32); }

// Warp-uniform bounded wait.
__device__ __forceinline__ bool warp_wait(uint32_t bar, uint32_t parity) {
  const bool ok = mbar_wait_bounded(bar, parity);
  return __all_sync(0xffffffffu, ok);
}

// Kernel layout: 8 warps, one CTA per SM, persistent over tiles.  Warp 0
// also fills the X box and fragment tables of the CTA's next tile (cp.async,
// completion tracked on an mbarrier; three 1D bulk copies); every warp
// refills its own coefficient ring slots as soon as it has read them.
template <int OP>
__global__ void __launch_bounds__(NTHR, 1) mf3d_tile_kernel(const Args a) {
  using C = Cfg<OP>;
  constexpr int UE = C::UE, NSLOT = C::NSLOT;
  constexpr bool kMass = C::kMass;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ int s_abort;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r = lane >> 2, c = lane & 3;
  const int ntiles = a.ntile[0] * a.ntile[1] * a.ntile[2];
  const int ngeom = a.ntile[0] + a.ntile[1] + a.ntile[2];

  // barriers: full per compute warp and ring slot, xfull per X / fragment buffer
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* xfull = full + NCWARP * NSLOT;
  int32_t* geo = reinterpret_cast<int32_t*>(smem + 2048);
  const int geo_bytes = (ngeom * GEOM * 4 + 127) / 128 * 128;
  double* xs = reinterpret_cast<double*>(smem + 2048 + geo_bytes);  // [2][XS]
  double* fr = xs + 2 * XS;                                         // [2][FR]
  double* t1s = fr + 2 * FR;
  double* t2s = t1s + T1S;
  double* ring = t2s + T2S;  // [NCWARP][NSLOT][UE]

  // ---- set-up: geometry table, finite contents everywhere, barriers
  for (int i = tid; i < ngeom * GEOM; i += NTHR) geo[i] = a.geom[i];
  for (int i = tid; i < 2 * XS + 2 * FR + T1S + T2S; i += NTHR) xs[i] = 0.0;
  if (tid == 0) {
    s_abort = 0;
    for (int i = 0; i < NCWARP * NSLOT; ++i) mbar_init(smem_u32(&full[i]), 1);
    for (int b = 0; b < 2; ++b)
      mbar_init(smem_u32(&xfull[b]), 33);  // 32 cp.async lanes + the bulk copies' arrive
    fence_mbar_init();
  }
  __syncthreads();

  // X box and fragment tables of tile t into buffer b, issued by warp 0:
  // cp.async (X, 8 bytes per element; completion tracked on xfull[b]) and
  // three 1D bulk copies (fragment tables)
  int fills[2] = {0, 0};  // prefetches issued into each buffer (warp 0)
  auto prefetch = [&](int t, int b) {
    ++fills[b];
    int t1, t2, t3;
    tile_coords(a, t, t1, t2, t3);
    const int32_t* r1 = rec(geo, a, 0, t1);
    const int32_t* r2 = rec(geo, a, 1, t2);
    const int32_t* r3 = rec(geo, a, 2, t3);
    const int dx1 = r1[G_DX], dx2 = r2[G_DX], dx3 = r3[G_DX];
    double* xb = xs + b * XS;
    const int d1 = lane & 15;
    if (d1 < dx1) {
      const int64_t plane = (int64_t)a.n[1] * a.n[0];
      const double* src = a.x + ((int64_t)r3[G_XA] * a.n[1] + r2[G_XA]) * a.n[0] + r1[G_XA] + d1;
      for (int d2 = 0; d2 < dx2; ++d2)
        for (int d3 = lane >> 4; d3 < dx3; d3 += 2)
          cp_async8(smem_u32(xb + (d3 * XP2 + d2) * XP1 + d1), src + d3 * plane + (int64_t)d2 * a.n[0]);
    }
    const uint32_t xb_bar = smem_u32(&xfull[b]);
    cp_async_mbar_arrive_noinc(xb_bar);
    if (lane == 0) {
      double* fb = fr + b * FR;
      mbar_arrive_expect_tx(xb_bar, FR * 8);
      bulk_g2s(smem_u32(fb), a.frag + (int64_t)t1 * 512, 512 * 8, xb_bar);
      bulk_g2s(smem_u32(fb + 512), a.frag + (int64_t)(a.ntile[0] + t2) * 512, 256 * 8, xb_bar);
      bulk_g2s(smem_u32(fb + 768), a.frag + (int64_t)(a.ntile[0] + a.ntile[1] + t3) * 512,
               512 * 8, xb_bar);
    }
  };
  if (warp == 0 && (int)blockIdx.x < ntiles) prefetch(blockIdx.x, 0);

  // ================================================================== consumers
  // coefficient ring of this warp: lane 0 refills a slot as soon as the warp
  // has read it (the values are in registers by then)
  UnitWalk wk;
  wk.t = blockIdx.x;
  wk.seek(geo, a, warp, ntiles, UE);
  int issued = 0;
  auto issue = [&]() {
    if (wk.valid) {
      const int slot = issued % NSLOT;
      if (lane == 0) {
        const uint32_t bar = smem_u32(&full[warp * NSLOT + slot]);
        mbar_arrive_expect_tx(bar, UE * 8);
        bulk_g2s(smem_u32(ring + (warp * NSLOT + slot) * UE), a.packed + wk.offset(UE), UE * 8,
                 bar);
      }
      ++issued;
      wk.advance(geo, a, warp, ntiles, UE);
    }
  };
  for (int k = 0; k < NSLOT; ++k) issue();
  bool aborted = false;
  int consumed = 0;
  int it = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
    const int cur = it & 1;
    if (!warp_wait(smem_u32(&xfull[cur]), (uint32_t)((it >> 1) & 1))) {
      aborted = true;
      if (lane == 0) atomicExch(&s_abort, 1);
    }
    consumers_sync();
    if (*(volatile int*)&s_abort) {
      aborted = true;
      break;  // uniform among the consumers: read after the barrier
    }
    // the other buffer finished its tile (stage 5 ended with a barrier)
    if (warp == 0 && t + (int)gridDim.x < ntiles) prefetch(t + gridDim.x, cur ^ 1);
    int t1, t2, t3;
    tile_coords(a, t, t1, t2, t3);
    const int32_t* R1 = rec(geo, a, 0, t1);
    const int32_t* R2 = rec(geo, a, 1, t2);
    const int32_t* R3 = rec(geo, a, 2, t3);
    const int Q2 = R2[G_Q];
    const int H1 = R1[G_WT];   // q1 groups (1 or 2)
    const int NG1 = R1[G_NG];  // = H1
    const int NT3 = R3[G_WT];  // q3 groups (1 or 2)
    const int DX3 = R3[G_DX], DY3 = R3[G_DY];
    const double* X = xs + cur * XS;
    const double* F = fr + cur * FR;

    // ---------------- stage 1: T1_b = B_b^(1) X, rows (d3, d2), cols q1
    for (int it = warp; it < DX3 * NG1; it += NCWARP) {
      const int d3 = NG1 == 2 ? it >> 1 : it;
      const int g = it - d3 * NG1;
      const double* Fg = F + g * 256;
      const int tw = R1[G_TW0 + g];
      const double* xr = X + (d3 * XP2 + r) * XP1 + tw + c;
      const double a0 = xr[0], a1 = xr[4];
      const int col = ((8 * g) ^ ((r & 1) << 3)) + 2 * c;
      {
        double p0 = 0.0, p1 = 0.0;
        dmma(p0, p1, a0, Fg[0 * 32 + lane]);
        dmma(p0, p1, a1, Fg[1 * 32 + lane]);
        *reinterpret_cast<double2*>(t1s + ((0 * XP3 + d3) * XP2 + r) * 16 + col) =
            make_double2(p0, p1);
      }
      if constexpr (!kMass) {
        double p0 = 0.0, p1 = 0.0;
        dmma(p0, p1, a0, Fg[2 * 32 + lane]);
        dmma(p0, p1, a1, Fg[3 * 32 + lane]);
        *reinterpret_cast<double2*>(t1s + ((1 * XP3 + d3) * XP2 + r) * 16 + col) =
            make_double2(p0, p1);
      }
    }
    consumers_sync();

    // ---------------- stage 2: T2 = B^(2) T1, rows (d3, q1), cols q2
    {
      const double* Fg = F + 2 * 256;
      const double b00 = Fg[0 * 32 + lane], b01 = Fg[1 * 32 + lane];
      double b10 = 0.0, b11 = 0.0;
      if constexpr (!kMass) {
        b10 = Fg[2 * 32 + lane];
        b11 = Fg[3 * 32 + lane];
      }
      for (int it = warp; it < DX3 * H1; it += NCWARP) {
        const int d3 = H1 == 2 ? it >> 1 : it;
        const int h = it - d3 * H1;
        const int q1p = (8 * h + r) ^ ((c & 1) << 3);
        const double* p0 = t1s + ((0 * XP3 + d3) * XP2 + c) * 16 + q1p;
        const double a00 = p0[0], a01 = p0[4 * 16];
        double s0 = 0.0, s1 = 0.0;
        dmma(s0, s1, a00, b00);
        dmma(s0, s1, a01, b01);
        const int q1 = 8 * h + r;
        double* o0 = t2s + (0 * XP3 + d3) * 8 * 16;
        o0[(2 * c) * 16 + swz2(q1, d3, 2 * c)] = s0;
        o0[(2 * c + 1) * 16 + swz2(q1, d3, 2 * c + 1)] = s1;
        if constexpr (!kMass) {
          const double* p1 = t1s + ((1 * XP3 + d3) * XP2 + c) * 16 + q1p;
          const double a10 = p1[0], a11 = p1[4 * 16];
          double u0 = 0.0, u1 = 0.0, v0 = 0.0, v1 = 0.0;
          dmma(u0, u1, a10, b00);  // T2_10 = B0 T1_1
          dmma(u0, u1, a11, b01);
          dmma(v0, v1, a00, b10);  // T2_01 = B1 T1_0
          dmma(v0, v1, a01, b11);
          double* o1 = t2s + (1 * XP3 + d3) * 8 * 16;
          double* o2 = t2s + (2 * XP3 + d3) * 8 * 16;
          o1[(2 * c) * 16 + swz2(q1, d3, 2 * c)] = u0;
          o1[(2 * c + 1) * 16 + swz2(q1, d3, 2 * c + 1)] = u1;
          o2[(2 * c) * 16 + swz2(q1, d3, 2 * c)] = v0;
          o2[(2 * c + 1) * 16 + swz2(q1, d3, 2 * c + 1)] = v1;
        }
      }
    }
    consumers_sync();

    // ---------------- stage 3: per (q2, q1-half) row block: trial products
    // along q3, coefficient mix, test products along q3 (into Y3 in place)
    {
      const int nmt = Q2 * H1;
      // direction-3 fragments of both q3 groups
      double bt0[2][2], bt1[2][2], wt0[2][2], wt1[2][2];
#pragma unroll
      for (int g = 0; g < 2; ++g)
#pragma unroll
        for (int s = 0; s < 2; ++s) {
          const double* Fg = F + (3 + g) * 256;
          bt0[g][s] = Fg[(0 * 2 + s) * 32 + lane];
          bt1[g][s] = kMass ? 0.0 : Fg[(1 * 2 + s) * 32 + lane];
          wt0[g][s] = Fg[(2 * 2 + s) * 32 + lane];
          wt1[g][s] = kMass ? 0.0 : Fg[(3 * 2 + s) * 32 + lane];
        }
      const int tw0 = R3[G_TW0], tw1 = R3[G_TW1], sw1 = R3[G_SW1];
      for (int mt = warp; mt < nmt && !aborted; mt += NCWARP) {
        const int q2 = H1 == 2 ? mt >> 1 : mt;
        const int h = mt - q2 * H1;
        const int q1 = 8 * h + r;
        constexpr int NC = kMass ? 1 : 3;
        double af[2][NC][2];
#pragma unroll
        for (int g = 0; g < 2; ++g) {
          const int tw = g == 0 ? tw0 : tw1;
#pragma unroll
          for (int cb = 0; cb < NC; ++cb)
#pragma unroll
            for (int s = 0; s < 2; ++s) {
              const int p = tw + 4 * s + c;
              af[g][cb][s] = (g < NT3) ? t2s[((cb * XP3 + p) * 8 + q2) * 16 + swz2(q1, p, q2)] : 0.0;
            }
        }
        double yo[2][NC][2];
        double u[2][NC][2];
#pragma unroll
        for (int g = 0; g < 2; ++g)
#pragma unroll
          for (int i = 0; i < NC; ++i) yo[g][i][0] = yo[g][i][1] = u[g][i][0] = u[g][i][1] = 0.0;
        // trial products of both q3 groups: U_j at (row, q3 = 8g + 2c + e)
#pragma unroll
        for (int g = 0; g < 2; ++g) {
          if (g >= NT3) break;
          if constexpr (kMass) {
            dmma(u[g][0][0], u[g][0][1], af[g][0][0], bt0[g][0]);
            dmma(u[g][0][0], u[g][0][1], af[g][0][1], bt0[g][1]);
          } else {
            // d/dxi1: B0^(3) T2_10; d/dxi2: B0^(3) T2_01; d/dxi3: B1^(3) T2_00
            dmma(u[g][0][0], u[g][0][1], af[g][1][0], bt0[g][0]);
            dmma(u[g][1][0], u[g][1][1], af[g][2][0], bt0[g][0]);
            dmma(u[g][2][0], u[g][2][1], af[g][0][0], bt1[g][0]);
            dmma(u[g][0][0], u[g][0][1], af[g][1][1], bt0[g][1]);
            dmma(u[g][1][0], u[g][1][1], af[g][2][1], bt0[g][1]);
            dmma(u[g][2][0], u[g][2][1], af[g][0][1], bt1[g][1]);
          }
        }
        // coefficients of the block's units
        double v[2][NC][2];
#pragma unroll
        for (int g = 0; g < 2; ++g) {
          if (g >= NT3) break;
          const int slot = (consumed + g) % NSLOT;
          if (!warp_wait(smem_u32(&full[warp * NSLOT + slot]),
                         (uint32_t)(((consumed + g) / NSLOT) & 1))) {
            aborted = true;
            if (lane == 0) atomicExch(&s_abort, 1);
            break;
          }
          const double* cs = ring + (warp * NSLOT + slot) * UE;
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            if constexpr (kMass) {
              v[g][0][e] = cs[e * 32 + lane] * u[g][0][e];
            } else {
              const double c00 = cs[(e * 6 + 0) * 32 + lane], c01 = cs[(e * 6 + 1) * 32 + lane];
              const double c02 = cs[(e * 6 + 2) * 32 + lane], c11 = cs[(e * 6 + 3) * 32 + lane];
              const double c12 = cs[(e * 6 + 4) * 32 + lane], c22 = cs[(e * 6 + 5) * 32 + lane];
              v[g][0][e] = c00 * u[g][0][e] + c01 * u[g][1][e] + c02 * u[g][2][e];
              v[g][1][e] = c01 * u[g][0][e] + c11 * u[g][1][e] + c12 * u[g][2][e];
              v[g][2][e] = c02 * u[g][0][e] + c12 * u[g][1][e] + c22 * u[g][2][e];
            }
          }
        }
        if (aborted) break;
        // the units are consumed: refill their slots with the warp's next units
        __syncwarp();
        consumed += NT3;
        issue();
        if (NT3 == 2) issue();
        // test products: the even / odd points of a group are the k-steps,
        // so V's output fragment is the A operand as it stands
#pragma unroll
        for (int g = 0; g < 2; ++g) {
          if (g >= NT3) break;
          if constexpr (kMass) {
            dmma(yo[g][0][0], yo[g][0][1], v[g][0][0], wt0[g][0]);
            dmma(yo[g][0][0], yo[g][0][1], v[g][0][1], wt0[g][1]);
          } else {
            // test derivative 1 and 2 keep W0 in direction 3, derivative 3 takes W1
            dmma(yo[g][0][0], yo[g][0][1], v[g][0][0], wt0[g][0]);
            dmma(yo[g][1][0], yo[g][1][1], v[g][1][0], wt0[g][0]);
            dmma(yo[g][2][0], yo[g][2][1], v[g][2][0], wt1[g][0]);
            dmma(yo[g][0][0], yo[g][0][1], v[g][0][1], wt0[g][1]);
            dmma(yo[g][1][0], yo[g][1][1], v[g][1][1], wt0[g][1]);
            dmma(yo[g][2][0], yo[g][2][1], v[g][2][1], wt1[g][1]);
          }
        }
        if (aborted) break;
        // Y3_i [d3'][q2][q1] in place of this block's T2 rows: group 0 covers
        // planes 0..7, group 1 planes sw1..sw1+7 (added where they overlap)
        __syncwarp();
#pragma unroll
        for (int i = 0; i < NC; ++i)
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int p = 2 * c + e;
            t2s[((i * XP3 + p) * 8 + q2) * 16 + swz2(q1, p, q2)] = yo[0][i][e];
          }
        if (NT3 == 2) {
          __syncwarp();
#pragma unroll
          for (int i = 0; i < NC; ++i)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int p = sw1 + 2 * c + e;
              double* dst = t2s + ((i * XP3 + p) * 8 + q2) * 16 + swz2(q1, p, q2);
              const double prev = p < 8 ? *dst : 0.0;
              *dst = prev + yo[1][i][e];
            }
        }
      }
    }
    consumers_sync();
    if (*(volatile int*)&s_abort) {
      aborted = true;
      break;  // uniform: read after the barrier
    }

    // ---------------- stage 4: Y2 = W^(2) Y3, rows (d3', q1), cols d2'
    {
      const double* Fg = F + 2 * 256;
      const double w00 = Fg[4 * 32 + lane], w01 = Fg[5 * 32 + lane];
      double w10 = 0.0, w11 = 0.0;
      if constexpr (!kMass) {
        w10 = Fg[6 * 32 + lane];
        w11 = Fg[7 * 32 + lane];
      }
      for (int it = warp; it < DY3 * H1; it += NCWARP) {
        const int p = H1 == 2 ? it >> 1 : it;
        const int h = it - p * H1;
        const int q1 = 8 * h + r;
        const int qa2 = c, qb2 = 4 + c;
        const int ia = swz2(q1, p, qa2), ib = swz2(q1, p, qb2);
        double s0 = 0.0, s1 = 0.0;
        {
          const double* y0 = t2s + (0 * XP3 + p) * 8 * 16;
          dmma(s0, s1, y0[qa2 * 16 + ia], w00);
          dmma(s0, s1, y0[qb2 * 16 + ib], w01);
        }
        double t0 = 0.0, tt1 = 0.0;
        if constexpr (!kMass) {
          const double* y1 = t2s + (1 * XP3 + p) * 8 * 16;
          const double* y2 = t2s + (2 * XP3 + p) * 8 * 16;
          dmma(t0, tt1, y1[qa2 * 16 + ia], w10);  // W1 in dir 2 on Y3_1
          dmma(t0, tt1, y1[qb2 * 16 + ib], w11);
          dmma(t0, tt1, y2[qa2 * 16 + ia], w00);  // W0 in dir 2 on Y3_2
          dmma(t0, tt1, y2[qb2 * 16 + ib], w01);
        }
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int d2 = 2 * c + e;
          const int col = q1 ^ ((d2 & 3) << 2);
          t1s[((0 * XP3 + p) * XP2 + d2) * 16 + col] = e ? s1 : s0;
          if constexpr (!kMass) t1s[((1 * XP3 + p) * XP2 + d2) * 16 + col] = e ? tt1 : t0;
        }
      }
    }
    consumers_sync();

    // ---------------- stage 5: y += W^(1) Y2, rows (d3', d2'), cols d1',
    // added into y straight from the fragments (neighbouring tiles and the
    // two q1 groups share control points)
    {
      const int dy1 = R1[G_DY], dy2 = R2[G_DY];
      const int64_t plane = (int64_t)a.n[1] * a.n[0];
      double* ybase = a.y + ((int64_t)R3[G_YA] * a.n[1] + R2[G_YA] + r) * a.n[0] + R1[G_YA];
      for (int p = warp; p < DY3; p += NCWARP) {
#pragma unroll
        for (int g = 0; g < 2; ++g) {
          if (g >= NG1) break;
          const double* Fg = F + g * 256;
          const double w00 = Fg[4 * 32 + lane], w01 = Fg[5 * 32 + lane];
          double s0 = 0.0, s1 = 0.0;
          const double* ya = t1s + ((0 * XP3 + p) * XP2 + r) * 16;
          const int ca = (8 * g + c) ^ ((r & 3) << 2), cb = (8 * g + 4 + c) ^ ((r & 3) << 2);
          if constexpr (kMass) {
            dmma(s0, s1, ya[ca], w00);
            dmma(s0, s1, ya[cb], w01);
          } else {
            const double w10 = Fg[6 * 32 + lane], w11 = Fg[7 * 32 + lane];
            const double* yb = t1s + ((1 * XP3 + p) * XP2 + r) * 16;
            dmma(s0, s1, ya[ca], w10);  // W1 in dir 1 on Y2_a
            dmma(s0, s1, ya[cb], w11);
            dmma(s0, s1, yb[ca], w00);  // W0 in dir 1 on Y2_bc
            dmma(s0, s1, yb[cb], w01);
          }
          const int j0 = R1[G_SW0 + g] + 2 * c;
          if (r < dy2) {
            double* dst = ybase + p * plane + j0;
            if (j0 < dy1) atomicAdd(dst, s0);
            if (j0 + 1 < dy1) atomicAdd(dst + 1, s1);
          }
        }
      }
    }
    consumers_sync();
  }
  // the warp's copies still in flight (after an abort) land before the CTA exits
  if (lane == 0)
    for (int u = consumed; u < issued; ++u)
      (void)mbar_wait_bounded(smem_u32(&full[warp * NSLOT + (u % NSLOT)]),
                              (uint32_t)((u / NSLOT) & 1));
  // cp.async and bulk copies of a prefetch in flight land before the CTA exits
  cp_async_wait_all();
  if (warp == 0 && lane == 0 && aborted)
    for (int b = 0; b < 2; ++b)
      if (fills[b] > 0) (void)mbar_wait_bounded(smem_u32(&xfull[b]), (uint32_t)((fills[b] - 1) & 1));
  if (aborted && tid == 0) atomicExch(a.status, IGA_ERR_TIMEOUT);
}

// Coefficient packing: one CTA per tile writes the tile's units,
// element (m-tile, q3 group, e, s, lane = 4 r + c) = stream s at
// (q1 = qa1 + 8 h + r, q2 = qa2 + m-tile / H, q3 = qa3 + 8 group + 2 c + e),
// zero where the tile has no such point.
template <typename Tin>
__global__ void mft_pack_kernel(Args a, int S, const Tin* __restrict__ coefs, int64_t ld,
                                double* __restrict__ packed) {
  const int t = blockIdx.x;
  int t1, t2, t3;
  t1 = t % a.ntile[0];
  const int rr = t / a.ntile[0];
  t2 = rr % a.ntile[1];
  t3 = rr / a.ntile[1];
  const int32_t* r1 = a.geom + t1 * GEOM;
  const int32_t* r2 = a.geom + (a.ntile[0] + t2) * GEOM;
  const int32_t* r3 = a.geom + (a.ntile[0] + a.ntile[1] + t3) * GEOM;
  const int64_t SH = a.wsum[0], SQ2 = a.wsum[1];
  const int64_t ubase = (int64_t)r3[G_CUM] * SQ2 * SH +
                        (int64_t)r3[G_WT] * ((int64_t)r2[G_CUM] * SH + (int64_t)r2[G_WT] * r1[G_CUM]);
  const int H = r1[G_WT], NT = r3[G_WT];
  const int nmt = r2[G_WT] * H;
  const int UE = 2 * S * 32;
  const int64_t count = (int64_t)nmt * NT * UE;
  double* out = packed + ubase * UE;
  for (int64_t i = threadIdx.x; i < count; i += blockDim.x) {
    const int w = (int)(i % UE);
    const int64_t u = i / UE;
    const int nt = (int)(u % NT), mt = (int)(u / NT);
    const int lane = w % 32, s = (w / 32) % S, e = w / (32 * S);
    const int r = lane >> 2, c = lane & 3;
    const int q2l = mt / H, h = mt % H;
    const int q1l = 8 * h + r, q3l = 8 * nt + 2 * c + e;
    double v = 0.0;
    if (q1l < r1[G_Q] && q3l < r3[G_Q]) {
      const int64_t q = ((int64_t)(r3[G_QA] + q3l) * a.nq[1] + r2[G_QA] + q2l) * a.nq[0] +
                        r1[G_QA] + q1l;
      v = (double)coefs[(int64_t)a.src_row[s] * ld + q];
    }
    out[i] = v;
  }
}

inline size_t smem_bytes(int op, const iga_mft_plan* p) {
  const int ngeom = p->ntile[0] + p->ntile[1] + p->ntile[2];
  const size_t geo = (size_t)(ngeom * GEOM * 4 + 127) / 128 * 128;
  const int UE = op == IGA_OP_MASS ? Cfg<IGA_OP_MASS>::UE : Cfg<IGA_OP_STIFF>::UE;
  const int NS = op == IGA_OP_MASS ? Cfg<IGA_OP_MASS>::NSLOT : Cfg<IGA_OP_STIFF>::NSLOT;
  return 2048 + geo + (size_t)(2 * XS + 2 * FR + T1S + T2S) * 8 + (size_t)NCWARP * NS * UE * 8;
}

inline Args make_args(const iga_mft_plan* p) {
  Args a;
  for (int k = 0; k < 3; ++k) {
    a.n[k] = p->n[k];
    a.nq[k] = p->nq[k];
    a.ntile[k] = p->ntile[k];
    a.wsum[k] = p->wsum[k];
  }
  for (int s = 0; s < 6; ++s) a.src_row[s] = p->src_row[s];
  a.geom = p->geom;
  a.frag = p->frag;
  a.packed = nullptr;
  a.x = nullptr;
  a.y = nullptr;
  a.status = p->status;
  return a;
}

}  // namespace mft
}  // namespace iga

using namespace iga;

extern "C" {

iga_status iga_mft_pack(const iga_mft_plan* plan, int dtype_in, const void* coefs, int64_t ld,
                        double* packed, int64_t packed_elems, iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(plan && coefs && packed && ld > 0, "bad argument");
  IGA_CHECK_ARG(plan->op == IGA_OP_MASS || plan->op == IGA_OP_STIFF, "op %d not supported",
                plan->op);
  const int S = plan->op == IGA_OP_MASS ? 1 : 6;
  IGA_CHECK_ARG(plan->nstream == S, "nstream %d does not match the operator", plan->nstream);
  const int64_t need = (int64_t)plan->wsum[0] * plan->wsum[1] * plan->wsum[2] * 2 * S * 32;
  IGA_CHECK_ARG(packed_elems >= need, "packed buffer holds %lld elements, %lld needed",
                (long long)packed_elems, (long long)need);
  for (int k = 0; k < 3; ++k)
    IGA_CHECK_ARG(plan->ntile[k] >= 1 && plan->n[k] >= 1 && plan->nq[k] >= 1, "bad extents");
  mft::Args a = mft::make_args(plan);
  const int tiles = plan->ntile[0] * plan->ntile[1] * plan->ntile[2];
  cudaStream_t st = as_stream(stream);
  if (dtype_in == IGA_F64)
    mft::mft_pack_kernel<double><<<tiles, 256, 0, st>>>(a, S, (const double*)coefs, ld, packed);
  else if (dtype_in == IGA_F32)
    mft::mft_pack_kernel<float><<<tiles, 256, 0, st>>>(a, S, (const float*)coefs, ld, packed);
  else {
    set_error("dtype_in %d not supported", dtype_in);
    return IGA_ERR_UNSUPPORTED;
  }
  IGA_LAUNCH_CHECK();
  return IGA_OK;
}

iga_status iga_mft_smem_bytes(const iga_mft_plan* plan, int64_t* bytes) {
  clear_error();
  IGA_CHECK_ARG(plan && bytes, "bad argument");
  *bytes = (int64_t)mft::smem_bytes(plan->op, plan);
  return IGA_OK;
}

iga_status iga_mft_matvec(const iga_mft_plan* plan, const double* packed, int64_t ncols,
                          const double* x, double* y, iga_stream stream) {
  clear_error();
  IGA_CHECK_ARG(plan && packed && x && y && ncols >= 1, "bad argument");
  IGA_CHECK_ARG(plan->op == IGA_OP_MASS || plan->op == IGA_OP_STIFF, "op %d not supported",
                plan->op);
  const size_t smem = mft::smem_bytes(plan->op, plan);
  IGA_CHECK_ARG(smem <= 227 * 1024, "tile plan needs %zu bytes of shared memory", smem);
  cudaStream_t st = as_stream(stream);
  const int64_t N = (int64_t)plan->n[0] * plan->n[1] * plan->n[2];
  const int tiles = plan->ntile[0] * plan->ntile[1] * plan->ntile[2];
  int dev = 0, sms = 148;
  IGA_CUDA_TRY(cudaGetDevice(&dev));
  IGA_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int grid = tiles < sms ? tiles : sms;
  IGA_CUDA_TRY(cudaMemsetAsync(y, 0, sizeof(double) * N * ncols, st));
  mft::Args a = mft::make_args(plan);
  a.packed = packed;
  for (int64_t k = 0; k < ncols; ++k) {
    a.x = x + k * N;
    a.y = y + k * N;
    if (plan->op == IGA_OP_MASS) {
      IGA_CUDA_TRY(cudaFuncSetAttribute(mft::mf3d_tile_kernel<IGA_OP_MASS>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      mft::mf3d_tile_kernel<IGA_OP_MASS><<<grid, mft::NTHR, smem, st>>>(a);
    } else {
      IGA_CUDA_TRY(cudaFuncSetAttribute(mft::mf3d_tile_kernel<IGA_OP_STIFF>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      mft::mf3d_tile_kernel<IGA_OP_STIFF><<<grid, mft::NTHR, smem, st>>>(a);
    }
    IGA_LAUNCH_CHECK();
  }
  return IGA_OK;
}

}  // extern "C"
