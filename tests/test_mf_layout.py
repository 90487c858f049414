"""CPU checks of the index arithmetic of the fused 3D matvec kernel
(csrc/mf_fused.cuh, csrc/fastdiv.cuh):

* the multiply-high division by a CTA-invariant divisor (FastDiv), compiled
  from the library's own header with the host compiler, equals integer
  division over the tile-local index ranges the kernel uses;
* the FP64 tensor-core form of the q1 flush contraction (mma.sync m8n8k4
  fragments over column-swizzled shared-memory tiles, one warp per 8 x 8
  output block, clamped padding rows, masked stores) is emulated lane by lane
  with the kernel's formulas and must equal the dense contraction;
* the kernel's shared-memory layout (compiled as host code from the kernel
  header): aligned, non-overlapping regions (or shared buffers that fit
  their host regions), and the benchmark plans within their resident-CTA
  budgets;
* the coefficient ring's schedule (issue RA = NST / QC x QC points ahead,
  consume a chunk of QC points, then issue up to RA past its end), replayed
  point by point: no slot is refilled before its point is consumed, at most
  NST points are in flight, every waited point was issued, and a chunk's
  slots are its base slot plus the point's offset in the chunk.
"""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
CSRC = ROOT / "igaops_b200" / "csrc"

HARNESS = r"""
#include <cstdio>
#include "fastdiv.cuh"
int main() {
  long bad = 0, checked = 0;
  for (int d = 1; d <= 4096; ++d) {
    iga::FastDiv f(d);
    const int lim = d <= 64 ? 65536 : 16384;
    for (int e = 0; e < lim; ++e, ++checked)
      if (f.div(e) != e / d) ++bad;
  }
  for (int d = 4097; d < 65536; d += 251) {
    iga::FastDiv f(d);
    for (int e = 0; e < 65536; e += 3, ++checked)
      if (f.div(e) != e / d) ++bad;
  }
  std::printf("%ld %ld\n", checked, bad);
  return bad != 0;
}
"""


def test_fastdiv_matches_integer_division(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    src = tmp_path / "fastdiv_check.cpp"
    exe = tmp_path / "fastdiv_check"
    src.write_text(HARNESS)
    subprocess.run([cxx, "-O2", "-std=c++17", f"-I{CSRC}", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    checked, bad = map(int, out.stdout.split())
    assert out.returncode == 0 and bad == 0 and checked > 10**7


# ------------------------------------------------ DMMA flush (FP64, q1 stage)
FX, FY = 16, 8


def swz(c, r):
    """Column swizzle of the FP64 16-wide tiles: c ^ 4 (r mod 4)."""
    return c ^ ((r & 3) << 2)


def mma_8x8x4(lane_a, lane_b, d):
    """mma.sync.m8n8k4.row.col.f64: lane l holds A[l/4][l%4], B[l%4][l/4],
    D[l/4][2(l%4)+i]. Returns the updated per-lane (d0, d1)."""
    A = np.zeros((8, 4))
    B = np.zeros((4, 8))
    D = np.zeros((8, 8))
    for lane in range(32):
        A[lane >> 2, lane & 3] = lane_a[lane]
        B[lane & 3, lane >> 2] = lane_b[lane]
        D[lane >> 2, 2 * (lane & 3)] = d[lane][0]
        D[lane >> 2, 2 * (lane & 3) + 1] = d[lane][1]
    D += A @ B
    return [(D[lane >> 2, 2 * (lane & 3)], D[lane >> 2, 2 * (lane & 3) + 1]) for lane in range(32)]


@pytest.mark.parametrize("D1r,D2r,dmax1,dmax2,np_,NG", [
    (9, 7, 10, 7, 2, 2),    # p3 interior tile, two flushed planes
    (5, 3, 10, 7, 1, 2),    # edge tile (short ranges)
    (13, 11, 13, 12, 1, 1), # wide band: two row blocks and two column blocks
    (8, 8, 8, 8, 3, 1),     # exact 8 x 8 blocks
])
def test_dmma_flush_q1_emulation(D1r, D2r, dmax1, dmax2, np_, NG):
    rng = np.random.default_rng(D1r * 100 + D2r)
    KS, W1S = FX, 2 * FX  # FP64 row strides (swizzled, unpadded)
    # ks[(pl, g, r2)][l1]: rows r2 >= D2r hold garbage (never written)
    ks_val = rng.standard_normal((np_, NG, dmax2, FX))
    ks = np.full(np_ * NG * dmax2 * KS, np.nan)
    for pl in range(np_):
        for g in range(NG):
            for r2 in range(dmax2):
                for l1 in range(FX):
                    v = ks_val[pl, g, r2, l1] if r2 < D2r else 1e300
                    ks[((pl * NG + g) * dmax2 + r2) * KS + swz(l1, r2)] = v
    # w1d[r1][b][l1]: zero for r1 >= D1r
    w_val = rng.standard_normal((dmax1, 2, FX))
    w_val[D1r:] = 0.0
    w1d = np.zeros(dmax1 * W1S)
    for r1 in range(dmax1):
        for b in range(2):
            for l1 in range(FX):
                w1d[r1 * W1S + b * FX + swz(l1, r1)] = w_val[r1, b, l1]
    gvals = [0, 1] if NG == 2 else [0]
    # dense reference: y[pl][r2][r1] = sum_g sum_l1 ks[pl,g,r2,l1] w[r1,g,l1]
    ref = np.zeros((np_, D2r, D1r))
    for pl in range(np_):
        for gs, g in enumerate(gvals):
            ref[pl] += ks_val[pl, gs, :D2r] @ w_val[:D1r, g].T
    # kernel emulation: one warp per (plane, row block, column block)
    y = np.zeros((np_, D2r, D1r))
    MT, NT1 = (D2r + 7) >> 3, (D1r + 7) >> 3
    for task in range(np_ * MT * NT1):
        nt, rest = task % NT1, task // NT1
        mt, pl = rest % MT, rest // MT
        d = [(0.0, 0.0)] * 32
        for gs, g in enumerate(gvals):
            for kt in range(FX // 4):
                la, lb = [], []
                for lane in range(32):
                    gq, tq = lane >> 2, lane & 3
                    r2c = min(mt * 8 + gq, dmax2 - 1)
                    r1c = min(nt * 8 + gq, dmax1 - 1)
                    l1 = kt * 4 + tq
                    la.append(ks[((pl * NG + gs) * dmax2 + r2c) * KS + swz(l1, r2c)])
                    lb.append(w1d[r1c * W1S + g * FX + swz(l1, r1c)])
                d = mma_8x8x4(la, lb, d)
        for lane in range(32):
            gq, tq = lane >> 2, lane & 3
            r2, r1 = mt * 8 + gq, nt * 8 + 2 * tq
            if r2 < D2r:
                if r1 < D1r:
                    y[pl, r2, r1] += d[lane][0]
                if r1 + 1 < D1r:
                    y[pl, r2, r1 + 1] += d[lane][1]
    np.testing.assert_allclose(y, ref, rtol=1e-13, atol=1e-13)


# ------------------------------------------------ shared-memory layout (host)
SMEM_HARNESS = r"""
#include <cstdio>
#include "mf_fused.cuh"
using namespace iga;
template <typename T, class P>
int check(int W, int cm1, int cm2, int dm1, int dm2) {
  const int rlen = step_row_len<T>(W);
  const Smem3<T, P> L(16, 8, W, rlen, cm1, cm2, dm1, dm2);
  const int A = 16 / (int)sizeof(T);
  const int QC = Depth3<T, P>::qc(W), NT = 128;
  int bad = 0;
  const int off[] = {L.ring, L.stage, L.done, L.ks, L.xs, L.a1s, L.b1tab, L.b2tab, L.w1d, L.w2d, L.total};
  for (int o : off) bad += (o % A) != 0;                       // 16-byte aligned regions
  const long n_stage = (long)QC * ncombo3<P>() * NT, n_done = (long)QC * npair3<P>() * NT;
  const long n_ks = (long)QC * ng<P>() * dm2 * L.ks_row, n_xs = (long)QC * cm1 * cm2;
  const long n_a1s = (long)QC * nb1<P>() * cm2 * 16;
  if (Depth3<T, P>::alias(W)) {
    bad += L.ks != L.stage || L.xs < L.ks + n_ks || L.done < L.xs + n_xs || L.done < L.stage + n_stage;
    bad += L.a1s != L.done || L.b1tab < L.a1s + n_a1s || L.b1tab < L.done + n_done;
  } else {
    bad += L.done < L.stage + n_stage || L.ks < L.done + n_done || L.xs < L.ks + n_ks;
    bad += L.a1s < L.xs + n_xs || L.b1tab < L.a1s + n_a1s;
  }
  bad += L.stage < L.ring + (long)Depth3<T, P>::nst(W) * (P::S * NT + rlen);
  bad += L.b2tab < L.b1tab + 16 * 2 * W || L.w1d < L.b2tab + 8 * 2 * W;
  bad += L.w2d < L.w1d + (long)dm1 * L.w1_row;
  bad += L.total < L.w2d + (long)dm2 * 16;
  bad += mf3d_smem_bytes<T, P>(16, 8, W, 0, rlen, cm1, cm2, dm1, dm2) != 128 + (size_t)L.total * sizeof(T) + 16;
  return bad;
}
int main() {
  int bad = 0;
  using Stiff = Pat<3, IGA_OP_STIFF, 0, 0, 0, 1>;
  using Mass = Pat<3, IGA_OP_MASS, 0, 0, 0, 0>;
  const int cases[][5] = {{3, 8, 6, 8, 6}, {4, 9, 7, 9, 7}, {5, 10, 8, 10, 8}, {6, 11, 9, 11, 9}, {4, 5, 4, 5, 4}};
  for (auto& c : cases) {
    bad += check<double, Stiff>(c[0], c[1], c[2], c[3], c[4]);
    bad += check<double, Mass>(c[0], c[1], c[2], c[3], c[4]);
    bad += check<float, Stiff>(c[0], c[1], c[2], c[3], c[4]);
    bad += check<float, Mass>(c[0], c[1], c[2], c[3], c[4]);
  }
  // the p3 128^3 FP64 stiffness plan fits three CTAs per SM, p2 four (shared buffers)
  const size_t s3 = mf3d_smem_bytes<double, Stiff>(16, 8, 4, 0, step_row_len<double>(4), 9, 7, 9, 7);
  const size_t s2 = mf3d_smem_bytes<double, Stiff>(16, 8, 3, 0, step_row_len<double>(3), 8, 6, 8, 6);
  std::printf("%d %zu %zu\n", bad, s3, s2);
  return bad != 0;
}
"""


def test_smem_layout_of_the_fused_kernel(tmp_path):
    """Every shared-memory region of the 3D kernel starts on a 16-byte
    boundary, regions do not overlap (or, where the kernel shares buffers
    with disjoint lifetimes, each fits inside its host region), and the
    byte count the launcher requests matches the layout; the benchmark
    plans fit their resident-CTA targets (227 KB per SM budget)."""
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        pytest.skip("no nvcc")
    src = tmp_path / "smem_check.cu"
    exe = tmp_path / "smem_check"
    src.write_text(SMEM_HARNESS)
    subprocess.run([nvcc, "-std=c++17", "--expt-relaxed-constexpr", f"-I{CSRC}",
                    f"-I{ROOT / 'include'}", "-gencode", "arch=compute_100a,code=sm_100a",
                    str(src), "-o", str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    bad, s3, s2 = map(int, out.stdout.split())
    assert out.returncode == 0 and bad == 0
    per_sm = 233472  # bytes of shared memory per SM
    assert 3 * (s3 + 1024 + 128) <= per_sm
    assert 4 * (s2 + 1024 + 128) <= per_sm


@pytest.mark.parametrize("QC,NST", [(4, 4), (6, 6), (8, 8), (4, 8), (6, 12), (5, 10),
                                    (4, 12), (8, 16), (4, 4 * 4)])
def test_coefficient_ring_schedule(QC, NST):
    """The TMA ring of mf3d_body: copies of point t land in slot t % NST; the
    chunk loop waits for its points (phase parity (t / NST) & 1), consumes
    them, passes the chunk barrier and issues the points up to RA past the
    chunk's end into the slots it freed."""
    assert NST % QC == 0
    RA = NST // QC * QC
    for L in list(range(1, 3 * NST + 3)) + [97, 389]:
        slot_owner = {}          # slot -> point whose copy it holds
        consumed = set()
        issued = []
        uses = {}                # slot -> completed fills (phase count)

        def issue(lo, hi):
            for t in range(lo, hi):
                s = t % NST
                prev = slot_owner.get(s)
                # the slot's previous point was consumed before the refill
                assert prev is None or prev in consumed, (L, t, prev)
                slot_owner[s] = t
                uses[s] = uses.get(s, 0) + 1
                issued.append(t)

        issue(0, min(RA, L))
        hi = min(RA, L)
        nchunk = -(-L // QC)
        for ch in range(nchunk):
            tb, te = ch * QC, min(ch * QC + QC, L)
            slot0 = tb % NST
            for k, t in enumerate(range(tb, te)):
                s = t % NST
                assert slot0 + k == s            # chunk base + offset
                assert slot_owner[s] == t        # the copy waited for is t's
                assert (uses[s] - 1) % 2 == (t // NST) & 1   # wait parity
                assert len([u for u in issued if u not in consumed]) <= NST
            consumed.update(range(tb, te))
            if hi < min(te + RA, L):
                issue(hi, min(te + RA, L))
                hi = min(te + RA, L)
        assert issued == list(range(L)) and consumed == set(range(L))
