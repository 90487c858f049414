"""CPU checks of the index arithmetic of the fused 3D matvec kernel
(csrc/mf_fused.cuh, csrc/fastdiv.cuh):

* the multiply-high division by a CTA-invariant divisor (FastDiv), compiled
  from the library's own header with the host compiler, equals integer
  division over the tile-local index ranges the kernel uses;
* the FP64 tensor-core form of the q1 flush contraction (mma.sync m8n8k4
  fragments over column-swizzled shared-memory tiles, one warp per 8 x 8
  output block, clamped padding rows, masked stores) is emulated lane by lane
  with the kernel's formulas and must equal the dense contraction.
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
