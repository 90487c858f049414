"""Host plan of the tensor-core 3D matvec (``mf3d_tile_kernel``, csrc/mf_tile.cu).

The FP64 stiffness and mass operators of a 3D patch
(BsplineOperations.compute_mf_scalar_gradu_gradv / compute_mf_scalar_u_v,
src/igaops/operators/bsplines_ops.py:290-355) as a sequence of small dense
contractions per 3D tile of quadrature points, every one a block of FP64
tensor-core products (``mma.sync.m8n8k4.f64``, 8 x 8 x 4 per warp
instruction):

* tiles of 16 x 8 x 16 quadrature points (directions 1, 2, 3; the last tile
  of a direction is partial);
* along each direction the tile's points fall into groups of 8; a group's
  trial band (B0 / B1 rows of its points) lies in a window of 8 consecutive
  control points, and so does its test band (rows of W0^T / W1^T), so every
  contraction is an 8-row, 8-column, 2 x 4-deep product; the windows of a
  tile lie inside 12 control points per direction (8 in direction 2);
* the 1D factors enter the products as fragment tables: per (direction,
  tile, group), B0, B1, W0^T, W1^T as the 8 x 8 window blocks in the
  register order of the tensor-core B operand (lane l holds
  row k = l % 4 + 4 s, column n = l / 4 of k-step s);
* the coefficients stream in units of 8 (q1, q2) rows x 8 q3 points x S
  streams, in the register order of the product that consumes them.

This module computes the tile geometry, the fragment tables and the packed
layout on the host (numpy), checks that the band structure fits the windows
(otherwise the operator keeps the pencil kernel) and holds the device buffers.
"""
from __future__ import annotations

import ctypes
import math
from typing import List, Optional

import numpy as np
import torch

from . import _lib
from ._device import iga_dtype, require_cuda, stream_handle
from .bands import rule_bands

QT = (16, 8, 16)      # tile extent in quadrature points per direction
XP = (12, 8, 12)      # allocated control-point extent of a tile per direction
GEOM = 16             # int32 fields per (direction, tile) record
(G_QA, G_Q, G_XA, G_YA, G_DX, G_DY, G_TW0, G_TW1, G_SW0, G_SW1, G_NG, G_CUM,
 G_WT) = range(13)
UNIT_ROWS = 8         # (q1, q2) rows of a coefficient unit
UNIT_Q3 = 8           # q3 points of a coefficient unit


def _dense_band(band, rows: int, cols: int, which: int) -> np.ndarray:
    """Dense (rows, cols) matrix of one value array of a shared band."""
    start, vals, w, _ = band
    M = np.zeros((rows, cols + w))
    r = np.arange(rows)[:, None]
    c = start[:, None].astype(np.int64) + np.arange(w)[None, :]
    M[np.broadcast_to(r, c.shape), c] = vals[which]
    return M[:, :cols]


class DirTiles:
    """Tiles of one direction: geometry records and fragment tables."""

    def __init__(self, q, k: int):
        rb = rule_bands(q)
        n, nq = rb.n, rb.nq
        W = max(rb.trial[2], rb.testT[2])
        self.k, self.n, self.nq, self.W = k, n, nq, W
        ts = rb.trial[0].astype(np.int64)
        ss = rb.testT[0].astype(np.int64)
        B0 = _dense_band(rb.trial, nq, n, 0)
        B1 = _dense_band(rb.trial, nq, n, 1)
        T0 = _dense_band(rb.testT, nq, n, 0)   # W0^T (nq x n)
        T1 = _dense_band(rb.testT, nq, n, 1)   # W1^T
        qt, xp = QT[k], XP[k]
        ntile = -(-nq // qt)
        self.ntile = ntile
        geom = np.zeros((ntile, GEOM), dtype=np.int32)
        frag = np.zeros((ntile, 2, 4, 2, 32))
        ok = True
        lanes = np.arange(32)
        lr, lc = lanes // 4, lanes % 4
        for t in range(ntile):
            qa = t * qt
            Q = min(qt, nq - qa)
            ng = -(-Q // 8)
            xa, ya = int(ts[qa]), int(ss[qa])
            dx = min(int(ts[qa + Q - 1]) + W, n) - xa
            dy = min(int(ss[qa + Q - 1]) + W, n) - ya
            g_rec = [qa, Q, xa, ya, dx, dy, 0, 0, 0, 0, ng]
            for g in range(ng):
                qg = qa + 8 * g
                ql = min(qg + 8, qa + Q) - 1
                tw, sw = int(ts[qg]) - xa, int(ss[qg]) - ya
                # the group's bands fit an 8-wide window inside the tile's
                # allocated extent
                if ts[ql] + W - ts[qg] > 8 or ss[ql] + W - ss[qg] > 8:
                    ok = False
                if tw + 8 > xp or sw + 8 > xp:
                    ok = False
                g_rec[G_TW0 + g] = tw
                g_rec[G_SW0 + g] = sw
                # trial fragments: lane holds B[qp = qg + l/4][dof = xa + tw + 4s + l%4]
                for s in range(2):
                    qp = qg + lr
                    dof = xa + tw + 4 * s + lc
                    okq = qp < qa + Q
                    okd = dof < n
                    m = okq & okd
                    qpc, dofc = np.where(m, qp, 0), np.where(m, dof, 0)
                    frag[t, g, 0, s] = np.where(m, B0[qpc, dofc], 0.0)
                    frag[t, g, 1, s] = np.where(m, B1[qpc, dofc], 0.0)
                    # test fragments: lane holds W^T[qp = qg + kappa(4s + l%4)][dof = ya + sw + l/4];
                    # direction 3 takes its k-steps as the even / odd points of the group
                    kk = 4 * s + lc
                    kap = (2 * lc + s) if k == 2 else kk
                    qp = qg + kap
                    dof = ya + sw + lr
                    m = (qp < qa + Q) & (dof < n)
                    qpc, dofc = np.where(m, qp, 0), np.where(m, dof, 0)
                    frag[t, g, 2, s] = np.where(m, T0[qpc, dofc], 0.0)
                    frag[t, g, 3, s] = np.where(m, T1[qpc, dofc], 0.0)
            if dx > xp or dy > xp:
                ok = False
            geom[t, :len(g_rec)] = g_rec
        # offset weights: H (direction 1), Q2 (direction 2), NT (direction 3)
        if k == 0:
            wt = -(-geom[:, G_Q] // 8)
        elif k == 1:
            wt = geom[:, G_Q].copy()
        else:
            wt = -(-geom[:, G_Q] // 8)
        geom[:, G_WT] = wt
        geom[:, G_CUM] = np.concatenate([[0], np.cumsum(wt)[:-1]])
        self.total = int(wt.sum())
        self.geom = geom
        self.frag = frag
        self.ok = ok


def tile_supported(quadrule_list, op: int, sym: bool, time_ders, dtype) -> bool:
    if len(quadrule_list) != 3 or time_ders is not None or dtype != torch.float64:
        return False
    if op == _lib.IGA_OP_STIFF and not sym:
        return False
    if op not in (_lib.IGA_OP_MASS, _lib.IGA_OP_STIFF):
        return False
    rbs = [rule_bands(q) for q in quadrule_list]
    if not all(rb.fusable for rb in rbs):
        return False
    if max(max(rb.trial[2], rb.testT[2]) for rb in rbs) > 5:
        return False
    dirs = [_dir_tiles(q, k) for k, q in enumerate(quadrule_list)]
    if not all(d.ok for d in dirs):
        return False
    return smem_bytes(op, [d.ntile for d in dirs]) <= SMEM_LIMIT


SMEM_LIMIT = 227 * 1024


def smem_bytes(op: int, ntile) -> int:
    """Dynamic shared memory of the kernel (the formula of csrc/mf_tile.cu)."""
    geo = (sum(ntile) * GEOM * 4 + 127) // 128 * 128
    xs, fr = XP[2] * XP[1] * XP[0], 5 * 256
    t1, t2 = 2 * XP[2] * XP[1] * 16, 3 * XP[2] * 8 * 16
    nslot = 12 if op == _lib.IGA_OP_MASS else 4
    return 2048 + geo + (2 * xs + 2 * fr + t1 + t2) * 8 + 8 * nslot * unit_elems(op) * 8


_DIR_CACHE = {}


def _dir_tiles(q, k: int) -> DirTiles:
    key = (id(q), k)
    hit = _DIR_CACHE.get(key)
    if hit is None or hit[0]() is not q:
        import weakref

        try:
            ref = weakref.ref(q)
        except TypeError:
            return DirTiles(q, k)
        hit = (ref, DirTiles(q, k))
        _DIR_CACHE[key] = hit
    return hit[1]


def unit_elems(op: int) -> int:
    S = 1 if op == _lib.IGA_OP_MASS else 6
    return 2 * S * 32


def stream_rows(op: int, lead2: int) -> List[int]:
    """Leading index (into the flattened reference coefficient array) of the
    streams: mass (c); stiffness (C00, C01, C02, C11, C12, C22)."""
    if op == _lib.IGA_OP_MASS:
        return [0]
    return [0 * lead2 + 0, 0 * lead2 + 1, 0 * lead2 + 2, 1 * lead2 + 1, 1 * lead2 + 2,
            2 * lead2 + 2]


class TilePlan:
    """Device plan of the tensor-core 3D matvec of one operator on one patch."""

    nseg = 1  # one launch covers the patch (no segments of a streamed direction)

    def __init__(self, quadrule_list, op: int):
        dev = require_cuda()
        self.op = op
        self.S = 1 if op == _lib.IGA_OP_MASS else 6
        self.dirs = [_dir_tiles(q, k) for k, q in enumerate(quadrule_list)]
        if not all(d.ok for d in self.dirs):
            raise NotImplementedError("band structure does not fit the tile windows")
        d1, d2, d3 = self.dirs
        self.n = [d.n for d in self.dirs]
        self.nq = [d.nq for d in self.dirs]
        self.N = math.prod(self.n)
        self.Nq = math.prod(self.nq)
        self.ntile = [d.ntile for d in self.dirs]
        self.tiles = math.prod(self.ntile)
        self.units = d1.total * d2.total * d3.total
        self.ue = unit_elems(op)
        self.packed_elems = self.units * self.ue
        geom = np.concatenate([d.geom for d in self.dirs]).astype(np.int32)
        frag = np.concatenate([d.frag.reshape(d.ntile, -1) for d in self.dirs])
        self.geom = torch.from_numpy(np.ascontiguousarray(geom)).to(dev)
        self.frag = torch.from_numpy(np.ascontiguousarray(frag)).to(dev, torch.float64)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        P = _lib.iga_mft_plan()
        P.op = op
        P.nstream = self.S
        for k in range(3):
            P.n[k] = self.n[k]
            P.nq[k] = self.nq[k]
            P.ntile[k] = self.ntile[k]
            P.wsum[k] = self.dirs[k].total
        P.geom = self.geom.data_ptr()
        P.frag = self.frag.data_ptr()
        P.status = self.status.data_ptr()
        self.P = P

    def pack(self, coefs: torch.Tensor, lead2: int) -> torch.Tensor:
        rows = stream_rows(self.op, lead2)
        for s in range(6):
            self.P.src_row[s] = rows[s] if s < len(rows) else 0
        packed = torch.empty(self.packed_elems, dtype=torch.float64, device=coefs.device)
        _lib.check(
            _lib.LIB.iga_mft_pack(ctypes.byref(self.P), iga_dtype(coefs.dtype),
                                  coefs.data_ptr(), coefs.shape[-1], packed.data_ptr(),
                                  self.packed_elems, stream_handle())
        )
        return packed

    def matvec(self, packed: torch.Tensor, x: torch.Tensor, y: torch.Tensor, ncols: int = 1):
        _lib.check(
            _lib.LIB.iga_mft_matvec(ctypes.byref(self.P), packed.data_ptr(), ncols, x.data_ptr(),
                                    y.data_ptr(), stream_handle())
        )

    def check_status(self):
        st = int(self.status.item())
        if st != 0:
            self.status.zero_()
            _lib.check(st)


# ------------------------------------------------------------------ emulation
def emulate(quadrule_list, op: int, coefs: np.ndarray, x: np.ndarray,
            pack_only: bool = False) -> Optional[np.ndarray]:
    """numpy restatement of the tile kernel's arithmetic (test support): the
    same tiles, windows, fragment tables and coefficient units, the products
    done as dense 8 x 8 blocks.  `coefs` in the reference layout."""
    dirs = [DirTiles(q, k) for k, q in enumerate(quadrule_list)]
    assert all(d.ok for d in dirs)
    n = [d.n for d in dirs]
    nq = [d.nq for d in dirs]
    S = 1 if op == _lib.IGA_OP_MASS else 6
    X = x.reshape(n[2], n[1], n[0])
    if op == _lib.IGA_OP_MASS:
        C = coefs.reshape(1, nq[2], nq[1], nq[0])
    else:
        c = coefs.reshape(3, 3, nq[2], nq[1], nq[0])
        C = np.stack([c[0, 0], c[0, 1], c[0, 2], c[1, 1], c[1, 2], c[2, 2]])
    y = np.zeros((n[2], n[1], n[0]))

    def blocks(d, t, g):
        """(B0, B1) as [qp 8][dof 8] and (W0T, W1T) as [qp 8][dof 8] in
        natural point order, decoded from the fragment table."""
        f = d.frag[t, g]  # [4][2][32]
        lanes = np.arange(32)
        lr, lc = lanes // 4, lanes % 4
        out = []
        for m in range(4):
            Bm = np.zeros((8, 8))
            for s in range(2):
                if m < 2:
                    Bm[lr, 4 * s + lc] = f[m, s]          # [qp][dof]
                else:
                    kap = (2 * lc + s) if d.k == 2 else 4 * s + lc
                    Bm[kap, lr] = f[m, s]                 # [qp][dof]
            out.append(Bm)
        return out

    for t3 in range(dirs[2].ntile):
        for t2 in range(dirs[1].ntile):
            for t1 in range(dirs[0].ntile):
                g = [d.geom[t] for d, t in zip(dirs, (t1, t2, t3))]
                Q = [int(r[G_Q]) for r in g]
                qa = [int(r[G_QA]) for r in g]
                xa = [int(r[G_XA]) for r in g]
                ya = [int(r[G_YA]) for r in g]
                # X box, zero beyond n
                Xb = np.zeros((XP[2], XP[1], XP[0]))
                e3, e2, e1 = (min(XP[2], n[2] - xa[2]), min(XP[1], n[1] - xa[1]),
                              min(XP[0], n[0] - xa[0]))
                Xb[:e3, :e2, :e1] = X[xa[2]:xa[2] + e3, xa[1]:xa[1] + e2, xa[0]:xa[0] + e1]
                # trial: dense per-tile factors [qp][dof-in-box] from the groups
                Bt, Wt = [], []
                for k, (d, t) in enumerate(zip(dirs, (t1, t2, t3))):
                    b0 = np.zeros((QT[k], XP[k]))
                    b1 = np.zeros((QT[k], XP[k]))
                    w0 = np.zeros((QT[k], XP[k]))
                    w1 = np.zeros((QT[k], XP[k]))
                    for gg in range(int(g[k][G_NG])):
                        B0, B1, W0, W1 = blocks(d, t, gg)
                        tw, sw = int(g[k][G_TW0 + gg]), int(g[k][G_SW0 + gg])
                        b0[8 * gg:8 * gg + 8, tw:tw + 8] += B0
                        b1[8 * gg:8 * gg + 8, tw:tw + 8] += B1
                        w0[8 * gg:8 * gg + 8, sw:sw + 8] += W0
                        w1[8 * gg:8 * gg + 8, sw:sw + 8] += W1
                    Bt.append((b0, b1))
                    Wt.append((w0, w1))
                # coefficients of the tile (zero beyond the tile)
                Ct = np.zeros((S, QT[2], QT[1], QT[0]))
                Ct[:, :Q[2], :Q[1], :Q[0]] = C[:, qa[2]:qa[2] + Q[2], qa[1]:qa[1] + Q[1],
                                               qa[0]:qa[0] + Q[0]]
                ein = np.einsum
                if op == _lib.IGA_OP_MASS:
                    u = ein("ai,bj,ck,kji->cba", Bt[0][0], Bt[1][0], Bt[2][0], Xb)
                    v = Ct[0] * u
                    yt = ein("ai,bj,ck,cba->kji", Wt[0][0], Wt[1][0], Wt[2][0], v)
                else:
                    u0 = ein("ai,bj,ck,kji->cba", Bt[0][1], Bt[1][0], Bt[2][0], Xb)
                    u1 = ein("ai,bj,ck,kji->cba", Bt[0][0], Bt[1][1], Bt[2][0], Xb)
                    u2 = ein("ai,bj,ck,kji->cba", Bt[0][0], Bt[1][0], Bt[2][1], Xb)
                    c00, c01, c02, c11, c12, c22 = Ct
                    v0 = c00 * u0 + c01 * u1 + c02 * u2
                    v1 = c01 * u0 + c11 * u1 + c12 * u2
                    v2 = c02 * u0 + c12 * u1 + c22 * u2
                    yt = (ein("ai,bj,ck,cba->kji", Wt[0][1], Wt[1][0], Wt[2][0], v0)
                          + ein("ai,bj,ck,cba->kji", Wt[0][0], Wt[1][1], Wt[2][0], v1)
                          + ein("ai,bj,ck,cba->kji", Wt[0][0], Wt[1][0], Wt[2][1], v2))
                e3, e2, e1 = (min(XP[2], n[2] - ya[2]), min(XP[1], n[1] - ya[1]),
                              min(XP[0], n[0] - ya[0]))
                y[ya[2]:ya[2] + e3, ya[1]:ya[1] + e2, ya[0]:ya[0] + e1] += yt[:e3, :e2, :e1]
    return y.ravel()
