"""Banded device views of the 1D factors (host-side setup, cached per object).

The reference stores every 1D factor as a scipy CSR matrix: ``q.basis[k]``
of shape (nq, n) and ``q.weights[k]`` of shape (n, nq)
(src/igaops/quadrature/utils/operations.py:53-105,
src/igaops/quadrature/weighted_quad.py:321-363).  B-spline supports make
every row a short contiguous band, so the device form is a dense band:
``start[r]`` (first column of row r) and ``vals[r, 0:width]``.  Several
matrices with the same sparsity (B0/B1, W00/W10) share one ``start`` so the
fused kernel walks them with a single register window.
"""
from __future__ import annotations

import weakref
from typing import Dict, List, Sequence, Tuple

import numpy as np
import scipy.sparse as sp
import torch

from . import _lib
from ._device import require_cuda


# ------------------------------------------------------------------ cache
class IdCache:
    """Per-object cache keyed by identity, dropped when the object dies."""

    def __init__(self):
        self._d: Dict[int, Tuple[weakref.ref, dict]] = {}

    def slot(self, obj) -> dict:
        key = id(obj)
        hit = self._d.get(key)
        if hit is not None and hit[0]() is obj:
            return hit[1]
        try:
            ref = weakref.ref(obj)
        except TypeError:
            return {}  # not weak-referenceable: no caching
        slot: dict = {}
        self._d[key] = (ref, slot)
        weakref.finalize(obj, self._d.pop, key, None)
        return slot


_CACHE = IdCache()


# ------------------------------------------------------------ band build
def _row_extents(M, rows: int):
    lo = np.full(rows, np.iinfo(np.int64).max, dtype=np.int64)
    hi = np.full(rows, -1, dtype=np.int64)
    if sp.issparse(M):
        coo = sp.coo_array(M)
        keep = coo.data != 0
        r, c = coo.row[keep].astype(np.int64), coo.col[keep].astype(np.int64)
    else:
        r, c = np.nonzero(np.asarray(M))
    np.minimum.at(lo, r, c)
    np.maximum.at(hi, r, c)
    return lo, hi


def _dense_rows(M) -> np.ndarray:
    if sp.issparse(M):
        return np.asarray(M.toarray(), dtype=np.float64)
    return np.asarray(M, dtype=np.float64)


def band_from(mats: Sequence, width: int | None = None, unit_steps: bool = False):
    """Shared band of same-shape matrices.

    Returns (start int32[rows], [vals float64[rows, width]] per matrix, width,
    monotone) where `monotone` tells whether start[] is non-decreasing.
    With unit_steps, a row's start is lowered (the band then also covers some
    leading zeros) wherever that keeps start[r] - start[r-1] <= 1 -- e.g. the
    last quadrature point x = 1, where only the last basis function is
    non-zero.
    """
    shape = mats[0].shape
    rows, cols = shape
    lo = np.full(rows, np.iinfo(np.int64).max, dtype=np.int64)
    hi = np.full(rows, -1, dtype=np.int64)
    for M in mats:
        if M.shape != shape:
            raise ValueError("matrices sharing a band must have the same shape")
        l, h = _row_extents(M, rows)
        lo = np.minimum(lo, l)
        hi = np.maximum(hi, h)
    empty = hi < 0
    start = np.where(empty, 0, lo)
    # empty rows inherit the previous start so that start stays monotone
    if empty.any():
        last = 0
        for r in range(rows):
            if empty[r]:
                start[r] = last
            else:
                last = start[r]
    natural = int(max(1, (hi - start + 1)[~empty].max())) if (~empty).any() else 1
    w = natural if width is None else int(width)
    if unit_steps:
        for r in range(1, rows):
            cand = min(start[r], start[r - 1] + 1)
            if cand >= start[r - 1] and (empty[r] or cand >= hi[r] - w + 1):
                start[r] = cand
    if w < natural:
        raise ValueError(f"band width {w} below the natural width {natural}")
    vals = []
    ridx = np.arange(rows)[:, None]
    cidx = start[:, None] + np.arange(w)[None, :]
    inside = cidx < cols
    for M in mats:
        D = _dense_rows(M) if rows * cols <= 4_000_000 else None
        V = np.zeros((rows, w), dtype=np.float64)
        if D is not None:
            V[inside] = D[np.broadcast_to(ridx, cidx.shape)[inside], cidx[inside]]
        else:
            coo = sp.coo_array(M)
            V[coo.row, coo.col - start[coo.row]] = coo.data
        vals.append(V)
    monotone = bool(np.all(np.diff(start) >= 0))
    return start.astype(np.int32), vals, w, monotone


# ---------------------------------------------------------- device bands
class DeviceBand:
    """A band on the device: start (int32) + one or more value arrays."""

    def __init__(self, start: np.ndarray, vals: List[np.ndarray], width: int, cols: int,
                 dtype: torch.dtype):
        dev = require_cuda()
        self.rows = int(start.shape[0])
        self.cols = int(cols)
        self.width = int(width)
        self.start_host = start
        self.start = torch.from_numpy(np.ascontiguousarray(start)).to(dev)
        self.vals = [torch.from_numpy(np.ascontiguousarray(v)).to(dev, dtype) for v in vals]

    def struct(self, k: int = 0) -> _lib.iga_band:
        b = _lib.iga_band()
        b.rows, b.cols, b.width = self.rows, self.cols, self.width
        b.start = self.start.data_ptr()
        b.vals = self.vals[k].data_ptr()
        return b


def device_band(mats: Sequence, dtype: torch.dtype, width: int | None = None) -> DeviceBand:
    start, vals, w, _ = band_from(mats, width)
    return DeviceBand(start, vals, w, mats[0].shape[1], dtype)


# ----------------------------------------------------- generic factors
class DeviceFactor:
    """iga_factor view of one matrix (band if sparse, strided dense if not)."""

    def __init__(self, M, dtype: torch.dtype, transpose: bool):
        dev = require_cuda()
        self.keep = []
        f = _lib.iga_factor()
        if isinstance(M, torch.Tensor):
            D = M.to(dev, dtype).contiguous()
            self._dense(f, D, transpose)
        elif sp.issparse(M):
            Mt = M.T if transpose else M
            band = device_band([Mt], dtype)
            self.keep.append(band)
            f.kind = 0
            f.rows, f.cols = band.rows, band.cols
            f.band = band.struct(0)
        else:
            D = torch.from_numpy(np.ascontiguousarray(np.asarray(M, dtype=np.float64))).to(dev, dtype)
            self._dense(f, D, transpose)
        self.f = f
        self.rows, self.cols = int(f.rows), int(f.cols)

    def _dense(self, f, D: torch.Tensor, transpose: bool):
        if D.ndim != 2:
            raise ValueError("factor matrices must be 2-dimensional")
        self.keep.append(D)
        r, c = D.shape
        f.kind = 1
        if transpose:
            f.rows, f.cols, f.ld_row, f.ld_col = c, r, 1, c
        else:
            f.rows, f.cols, f.ld_row, f.ld_col = r, c, c, 1
        f.dense = D.data_ptr()


def factor_for(M, dtype: torch.dtype, transpose: bool = False) -> DeviceFactor:
    if isinstance(M, torch.Tensor):
        return DeviceFactor(M, dtype, transpose)  # tensors are used as given
    slot = _CACHE.slot(M)
    key = ("factor", dtype, bool(transpose))
    fac = slot.get(key)
    if fac is None:
        fac = DeviceFactor(M, dtype, transpose)
        slot[key] = fac
    return fac


# ------------------------------------------------- fused-kernel views
class RuleBands:
    """The three banded views of one quadrature rule used by the fused kernel.

    trial : B0/B1 (nq x n)   testT : W0^T/W1^T (nq x n)   testR : W0/W1 (n x nq)
    with W0 = weights[0] and W1 = weights[2].
    """

    def __init__(self, q):
        B = q.basis
        Wt = q.weights
        self.n = int(q.nbctrlpts)
        self.nq = int(q.nbquadpts)
        self.trial = band_from([B[0], B[1]], unit_steps=True)
        self.testT = band_from([sp.csr_array(Wt[0]).T, sp.csr_array(Wt[2]).T], unit_steps=True)
        self.testR = band_from([Wt[0], Wt[2]])
        same01 = _same(Wt[0], Wt[1])
        same23 = _same(Wt[2], Wt[3])
        monotone = self.trial[3] and self.testT[3] and self.testR[3]
        # the fused kernel walks quadrature points in order and moves its
        # control-plane windows by at most one plane per point
        steps = bool(np.all(np.diff(self.trial[0]) <= 1) and np.all(np.diff(self.testT[0]) <= 1))
        # fused kernel needs weights depending on the test derivative only
        self.fusable = bool(same01 and same23 and monotone and steps)
        self._dev: Dict[tuple, tuple] = {}

    @property
    def width(self) -> int:
        return max(self.trial[2], self.testT[2])

    @property
    def rwidth(self) -> int:
        return self.testR[2]

    def device(self, dtype: torch.dtype, W: int, RW: int):
        key = (dtype, W, RW)
        hit = self._dev.get(key)
        if hit is None:
            hit = (
                _repad(self.trial, W, self.n, dtype),
                _repad(self.testT, W, self.n, dtype),
                _repad(self.testR, RW, self.nq, dtype),
            )
            self._dev[key] = hit
        return hit


def _same(A, B) -> bool:
    A = sp.csr_array(A)
    B = sp.csr_array(B)
    if A.shape != B.shape:
        return False
    return (A != B).nnz == 0


def _repad(band, W: int, cols: int, dtype) -> DeviceBand:
    start, vals, w, _ = band
    if W < w:
        raise ValueError("padding below natural width")
    pv = [np.pad(v, ((0, 0), (0, W - w))) for v in vals]
    return DeviceBand(start, pv, W, cols, dtype)


def rule_bands(q) -> RuleBands:
    slot = _CACHE.slot(q)
    rb = slot.get("rulebands")
    if rb is None:
        rb = RuleBands(q)
        slot["rulebands"] = rb
    return rb
