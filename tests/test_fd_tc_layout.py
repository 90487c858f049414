"""CPU check of the index arithmetic of the tensor-core FD apply
(csrc/fd_tc.cu): the six rotated mode products are emulated in numpy with
the kernel's own formulas (gather, rotated stores with padded fastest dims,
1/Lambda index, scatter) and the B operands decoded from the core-matrix
image that igaops_b200.fastdiag builds; the result must equal the oracle's
FD apply."""
import numpy as np
import pytest

from oracle import fd as ofd
from tests._problems import rules


def _tile(Bm):
    """Core-matrix image as fastdiag._tile_kmajor_bf16 builds it (float64)."""
    nr, kr = Bm.shape
    Np, Kp = -(-nr // 16) * 16, -(-kr // 16) * 16
    P = np.zeros((Np, Kp))
    P[:nr, :kr] = Bm
    return P.reshape(Np // 8, 8, Kp // 8, 8).transpose(2, 0, 1, 3).reshape(-1), Np, Kp


def _untile(img, Np, Kp):
    """Read operand element (n, k) the way the MMA descriptors address it:
    core (g = n/8, kc = k/8) at element (kc*Np/8 + g)*64, row n%8 at 8*(n%8)."""
    B = np.zeros((Np, Kp))
    for nn in range(Np):
        for kk in range(Kp):
            B[nn, kk] = img[(kk // 8 * (Np // 8) + nn // 8) * 64 + (nn % 8) * 8 + kk % 8]
    return B


def _gemm(Asrc, R, Kp, Bimg, Np, N, out_rfast, kpn, mode, inv_lambda=None, box=None, y=None):
    """D[row][a] = sum_k A[row][k] B[k][a]; B[k][a] = image row a, column k."""
    B = _untile(Bimg, Np, Kp)  # (Np, Kp): row a, col k
    D = Asrc(R, Kp) @ B.T       # (R, Np)
    if mode == 2:
        n, lo, m = box
        for row in range(R):
            i1, i2 = row % m[0], row // m[0]
            for a in range(N):
                idx = ((lo[2] + a) * n[1] + lo[1] + i2) * n[0] + lo[0] + i1
                y[idx] = D[row, a]
        return None
    nslow = R // out_rfast
    out = np.zeros(N * nslow * kpn)
    for row in range(R):
        rs, rf = row // out_rfast, row % out_rfast
        for a in range(N):
            v = D[row, a]
            if mode == 1:
                v *= inv_lambda[a * R + row]
            out[(a * nslow + rs) * kpn + rf] = v
    return out


@pytest.mark.parametrize("p,ne,table_kind", [(2, 3, "all"), (3, 4, "mixed"), (2, 5, "none")])
def test_fd_tc_index_arithmetic(p, ne, table_kind):
    rl = rules(3, [p, p, p + 1], [ne, ne + 1, ne + 2], kind="gauss")
    table = np.ones((1, 3, 2), dtype=bool)
    if table_kind == "mixed":
        table[0, 0, 0] = False
        table[0, 2, 1] = False
    elif table_kind == "none":
        table[:] = False
    fd = ofd.setup(rl, table)
    n = fd.n
    lo = [1 if table[0, d, 0] else 0 for d in range(3)]
    m = [U.shape[0] for U in fd.U]
    kp = [-(-mm // 16) * 16 for mm in m]
    rng = np.random.default_rng(p + ne)
    x = rng.standard_normal(int(np.prod(n)))
    inv = 1.0 / fd.eig
    fwd = [_tile(U.T) for U in fd.U]
    bwd = [_tile(U) for U in fd.U]
    m1, m2, m3 = m

    def gather(R, Kp):
        A = np.zeros((R, Kp))
        for row in range(R):
            i2, i3 = row % m2, row // m2
            for k in range(m1):
                A[row, k] = x[((lo[2] + i3) * n[1] + lo[1] + i2) * n[0] + lo[0] + k]
        return A

    def rows_of(buf):
        return lambda R, Kp: buf[: R * Kp].reshape(R, Kp)

    t1 = _gemm(gather, m3 * m2, kp[0], fwd[0][0], fwd[0][1], m1, m2, kp[1], 0)
    t2 = _gemm(rows_of(t1), m1 * m3, kp[1], fwd[1][0], fwd[1][1], m2, m3, kp[2], 0)
    t3 = _gemm(rows_of(t2), m2 * m1, kp[2], fwd[2][0], fwd[2][1], m3, m1, kp[0], 1, inv)
    t4 = _gemm(rows_of(t3), m3 * m2, kp[0], bwd[0][0], bwd[0][1], m1, m2, kp[1], 0)
    t5 = _gemm(rows_of(t4), m1 * m3, kp[1], bwd[1][0], bwd[1][1], m2, m3, kp[2], 0)
    y = np.zeros_like(x)
    _gemm(rows_of(t5), m2 * m1, kp[2], bwd[2][0], bwd[2][1], m3, m1, kp[0], 2, box=(n, lo, m), y=y)
    ref = ofd.apply(fd, x)
    assert np.max(np.abs(y - ref)) <= 1e-12 * np.max(np.abs(ref))


def _gather_emulated(x_bytes_offset, elem, xflat, rowbase, nvalid, Kp, m0):
    """The tensor-core apply's gather (csrc/fd_tc.cu gather_tile), thread by
    thread: thread t owns row t mod 128 and half of its 8-element chunks,
    reads the aligned 16-byte blocks holding the row (only blocks that hold
    an element of the row), shifts a 9-block window by the row's
    misalignment one bit at a time and writes chunk (row r, kc) at byte
    kc * 2048 + r * 16 of the tile.  Returns the tile as (128, Kp) and the
    set of block indices read."""
    VW = 16 // elem
    G = VW
    tile = np.full(128 * Kp, np.nan)  # element view of the tile (2-byte slots)
    nkc = Kp // 8
    halfc = (nkc + 1) // 2
    read = set()
    for tid in range(256):
        r = tid & 127
        kc0, kc1 = (halfc, nkc) if tid >> 7 else (0, halfc)
        b = rowbase[r] if r < nvalid else -1
        lead = qlast = 0
        if b >= 0:
            a = x_bytes_offset + b * elem
            lead = (a % 16) // elem
            qlast = (lead + m0 - 1) // VW
            a16 = a - a % 16
        for kg in range(kc0, kc1, G):
            e0 = lead + 8 * kg
            q0, p0 = e0 // VW, e0 % VW
            w = [0.0] * (9 * VW)
            for t in range(9):
                if b >= 0 and q0 + t <= qlast:
                    blk = (a16 + (q0 + t) * 16 - x_bytes_offset) // elem  # element index
                    # every block read holds an element of the row
                    assert any(b <= blk + i < b + m0 for i in range(VW))
                    read.add(blk)
                    for i in range(VW):
                        j = blk + i
                        w[t * VW + i] = xflat[j] if 0 <= j < xflat.size else np.nan
            sh = VW // 2
            while sh >= 1:
                if p0 & sh:
                    for i in range(9 * VW - sh):
                        w[i] = w[i + sh]
                sh //= 2
            for c in range(G):
                kc = kg + c
                if kc >= kc1:
                    break
                for m in range(8):
                    k = 8 * kc + m
                    val = w[8 * c + m] if (b >= 0 and k < m0) else 0.0
                    tile[(kc * 2048 + r * 16) // 2 + m] = val
    # decode the canonical layout back to (row, k)
    out = np.zeros((128, Kp))
    for r in range(128):
        for k in range(Kp):
            out[r, k] = tile[((k >> 3) * 16 + (r >> 3)) * 64 + (r & 7) * 8 + (k & 7)]
    return out, read


@pytest.mark.parametrize("elem", [4, 8])
@pytest.mark.parametrize("offset", [0, 1, 2, 3])
@pytest.mark.parametrize("m0,n0,nvalid", [(11, 13, 128), (97, 99, 100), (16, 16, 37), (1, 3, 5)])
def test_fd_tc_gather_layout(elem, offset, m0, n0, nvalid):
    """Every element of the 128 x Kp tile is written (the NaN fill never
    survives), box elements land at their canonical positions, padding
    columns and rows past the last are zero, and only blocks that hold an
    element of their row are read, at every alignment of the vector."""
    Kp = -(-m0 // 16) * 16
    rng = np.random.default_rng(m0 + offset)
    nrows = nvalid
    xflat = rng.standard_normal(n0 * (nrows + 2) + 8)
    lo0 = 1 if n0 > m0 else 0
    rowbase = np.array([(r + 1) * n0 + lo0 for r in range(128)])
    out, read = _gather_emulated(offset * elem, elem, xflat, rowbase, nvalid, Kp, m0)
    assert np.isfinite(out).all()
    want = np.zeros((128, Kp))
    for r in range(nvalid):
        want[r, :m0] = xflat[rowbase[r]:rowbase[r] + m0]
    assert np.array_equal(out, want)
