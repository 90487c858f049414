"""Matrix-free operators on the GPU, behind the reference's operator API.

* ``MatrixFree``         -- src/igaops/operators/utils/matrix_free.py:7-119
* ``BsplineOperations``  -- src/igaops/operators/bsplines_ops.py:56-429
* ``MFOperator``         -- device-resident form of one ``compute_mf_*`` call
  (packed coefficients, fixed plan), used by the solvers and the benchmark.

Arrays: numpy in -> numpy (float64) out, computed in FP64; torch CUDA tensors
in -> torch out, computed in the tensor's precision (float64 or float32).
Every numerical step runs in libigab200; torch only holds memory.
"""
from __future__ import annotations

import ctypes
import math
from typing import Optional

import numpy as np
import torch

from . import _lib
from ._device import (
    compute_dtype,
    iga_dtype,
    like_input,
    require_cuda,
    stream_handle,
    to_device,
)
from .bands import factor_for, rule_bands

_OPS = {
    "u_v": _lib.IGA_OP_MASS,
    "mass": _lib.IGA_OP_MASS,
    "gradu_gradv": _lib.IGA_OP_STIFF,
    "stiffness": _lib.IGA_OP_STIFF,
    "gradu_v": _lib.IGA_OP_GRADU_V,
    "u_gradv": _lib.IGA_OP_U_GRADV,
}


# =================================================================== L-mode
def _lmode_device(factors, x: torch.Tensor, ncols: int) -> torch.Tensor:
    """(M_d x ... x M_1) x on the device; factors[0] = M_1; x is (N, ncols) C-order."""
    d = len(factors)
    dt = iga_dtype(x.dtype)
    arr = (_lib.iga_factor * d)(*[f.f for f in factors])
    dims = [f.cols for f in factors][::-1]  # slowest first
    work = 0
    for m in range(d):
        f = factors[d - 1 - m]
        dims[m] = f.rows
        work = max(work, math.prod(dims) * ncols)
    out_elems = math.prod(f.rows for f in factors) * ncols
    y = torch.empty(out_elems, dtype=x.dtype, device=x.device)
    if d > 1:
        w0 = torch.empty(work, dtype=x.dtype, device=x.device)
        w1 = torch.empty(work, dtype=x.dtype, device=x.device)
        p0, p1 = w0.data_ptr(), w1.data_ptr()
    else:
        p0 = p1 = None
    _lib.check(
        _lib.LIB.iga_lmode_apply(dt, d, arr, ncols, x.data_ptr(), y.data_ptr(), p0, p1,
                                 stream_handle())
    )
    return y


class MatrixFree:
    """Kronecker (L-mode) products, same arguments as the reference class."""

    @staticmethod
    def reshape_array_to_tensor(matrix_list, array_in, is_transpose: bool = False):
        shape = [m.shape[0 if is_transpose else 1] for m in matrix_list]
        shape.extend(tuple(array_in.shape[1:]) or (1,))
        return array_in.reshape(shape)

    @staticmethod
    def tensor_matrix_product(tensor, matrix, mode: int, is_transpose: bool = False):
        """n-mode product of `tensor` with `matrix` along `mode` (on the GPU)."""
        dtype = compute_dtype(tensor)
        t = to_device(tensor, dtype)
        shape = list(t.shape)
        fac = factor_for(matrix, dtype, transpose=is_transpose)
        if fac.cols != shape[mode]:
            raise ValueError(
                f"matrix has {fac.cols} columns, tensor mode {mode} has size {shape[mode]}"
            )
        outer = math.prod(shape[:mode])
        inner = math.prod(shape[mode + 1:])
        out_shape = shape[:mode] + [fac.rows] + shape[mode + 1:]
        y = torch.empty(out_shape, dtype=dtype, device=t.device)
        _lib.check(
            _lib.LIB.iga_mode_product(iga_dtype(dtype), fac.f, outer, inner, t.data_ptr(),
                                      y.data_ptr(), 0, stream_handle())
        )
        return like_input(y, tensor)

    @staticmethod
    def apply(matrix_list, array_in, is_transpose: bool = False):
        """(M_n x ... x M_1) v, or its transpose; v is (N,) or (N, k)."""
        dtype = compute_dtype(array_in)
        x = to_device(array_in, dtype)
        ncols = 1 if x.ndim == 1 else math.prod(x.shape[1:])
        facs = [factor_for(M, dtype, transpose=is_transpose) for M in matrix_list]
        n_in = math.prod(f.cols for f in facs)
        if x.shape[0] != n_in:
            raise ValueError(f"array_in has {x.shape[0]} rows, the factors expect {n_in}")
        y = _lmode_device(facs, x, ncols)
        if x.ndim == 1:
            y = y.reshape(-1)
        else:
            y = y.reshape((-1,) + tuple(x.shape[1:]))
        return like_input(y, array_in)


# ============================================================ fused plans
def _spacetime(time_ders):
    if time_ders is None:
        return 0, 0, 0
    tt, tr = int(time_ders[0]), int(time_ders[1])
    return 1, tt, tr


def _fused_supported(ndim, op, st, tt, tr) -> bool:
    if ndim not in (2, 3):
        return False
    if tt not in (0, 1) or tr not in (0, 1):
        return False
    if not st:
        return True
    if ndim != 3:
        return False
    if op == _lib.IGA_OP_MASS:
        return True
    return op == _lib.IGA_OP_STIFF and tt == 0 and tr == 0


def _nstream(ndim, op, st, sym):
    spd = ndim - 1 if st else ndim
    if op == _lib.IGA_OP_MASS:
        return 1
    if op == _lib.IGA_OP_STIFF:
        return spd * (spd + 1) // 2 if sym else spd * spd
    return spd


def _src_rows(ndim, op, st, sym, lead2: int):
    """Leading index (into the reference coefficient array) of each stream."""
    spd = ndim - 1 if st else ndim
    if op == _lib.IGA_OP_MASS:
        return [0]
    if op in (_lib.IGA_OP_GRADU_V, _lib.IGA_OP_U_GRADV):
        return list(range(spd))
    if not sym:
        return [i * lead2 + j for i in range(spd) for j in range(spd)]
    rows = [i * lead2 + i for i in range(spd)]
    pairs = [(0, 1)] if spd == 2 else [(0, 1), (0, 2), (1, 2)]
    rows += [i * lead2 + j for i, j in pairs]
    return rows


FACE3 = (16, 8)
FACE2 = (128,)
_SM_COUNT = 148


class FusedPlan:
    """Device plan of one fused operator on one patch (see include/igab200.h)."""

    def __init__(self, quadrule_list, op: int, time_ders, sym: bool, dtype: torch.dtype,
                 nseg: Optional[int] = None):
        dev = require_cuda()
        ndim = len(quadrule_list)
        st, tt, tr = _spacetime(time_ders)
        self.ndim, self.op, self.st, self.tt, self.tr = ndim, op, st, tt, tr
        self.sym = bool(sym)
        self.dtype = dtype
        rbs = [rule_bands(q) for q in quadrule_list]
        W = max(rb.width for rb in rbs)
        RW = max(rb.rwidth for rb in rbs)
        if not (3 <= W <= 6):
            raise NotImplementedError(f"fused kernels cover band width 3..6, got {W}")
        self.W, self.RW = W, RW
        self.n = [rb.n for rb in rbs]
        self.nq = [rb.nq for rb in rbs]
        self.N = math.prod(self.n)
        self.Nq = math.prod(self.nq)
        devb = [rb.device(dtype, W, RW) for rb in rbs]
        self._keep = devb
        P = _lib.iga_mf_plan()
        P.ndim, P.op, P.spacetime, P.time_test, P.time_trial = ndim, op, st, tt, tr
        P.sym = int(self.sym)
        P.width, P.rwidth = W, RW
        for d in range(3):
            P.n[d] = self.n[d] if d < ndim else 1
            P.nq[d] = self.nq[d] if d < ndim else 1
        face = FACE3 if ndim == 3 else FACE2
        P.face[0] = face[0]
        P.face[1] = face[1] if ndim == 3 else 1
        S = _nstream(ndim, op, st, self.sym)
        P.nstream = S
        self.nstream = S
        # tiles and segments of the streamed direction
        tiles1 = -(-self.nq[0] // face[0])
        tiles2 = -(-self.nq[1] // face[1]) if ndim == 3 else 1
        nlast = self.nq[-1]
        if nseg is None:
            # about 12 CTAs per SM (one resident CTA per SM in 3D), segments of
            # at least 48 points so window warm-up and flush stay amortised
            target = _SM_COUNT * 12
            nseg = max(1, min(-(-target // (tiles1 * tiles2)), nlast // 48))
        nseg = max(1, min(int(nseg), nlast))
        P.nseg = nseg
        self.nseg = nseg
        self.units = tiles1 * tiles2 * nseg
        # tile ranges for shared-memory sizing
        cmax, dmax = [1, 1], [1, 1]
        for d in range(min(ndim - 1, 2)):
            f = face[d]
            ts = rbs[d].trial[0]
            ws = rbs[d].testT[0]
            for t in range(-(-self.nq[d] // f)):
                lo, hi = t * f, min((t + 1) * f, self.nq[d]) - 1
                cmax[d] = max(cmax[d], int(ts[hi] - ts[lo]) + W)
                dmax[d] = max(dmax[d], int(min(ws[hi] + W - 1, self.n[d] - 1) - ws[lo] + 1))
        P.cmax[0], P.cmax[1] = cmax
        P.dmax[0], P.dmax[1] = dmax
        for d in range(ndim):
            trial, testT, testR = devb[d]
            P.trial[d] = trial.struct(0)
            P.trial_d1[d] = trial.vals[1].data_ptr()
            P.testT[d] = testT.struct(0)
            P.testT_d1[d] = testT.vals[1].data_ptr()
            P.testR[d] = testR.struct(0)
            P.testR_d1[d] = testR.vals[1].data_ptr()
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        P.status = self.status.data_ptr()
        # packed layout
        off = np.zeros(tiles1 * tiles2, dtype=np.int64)
        elems = ctypes.c_int64(0)
        _lib.check(
            _lib.LIB.iga_mf_layout(ctypes.byref(P), iga_dtype(dtype), ctypes.byref(elems),
                                   off.ctypes.data_as(ctypes.c_void_p))
        )
        self.packed_elems = int(elems.value)
        self.tile_off = torch.from_numpy(off).to(dev)
        P.tile_off = self.tile_off.data_ptr()
        # per-point step table of the streamed direction
        telems = ctypes.c_int64(0)
        _lib.check(_lib.LIB.iga_mf_table(ctypes.byref(P), iga_dtype(dtype), ctypes.byref(telems),
                                         None, stream_handle()))
        self.step_table = torch.empty(int(telems.value), dtype=dtype, device=dev)
        _lib.check(_lib.LIB.iga_mf_table(ctypes.byref(P), iga_dtype(dtype), ctypes.byref(telems),
                                         self.step_table.data_ptr(), stream_handle()))
        P.step_table = self.step_table.data_ptr()
        self.P = P

    def set_nseg(self, nseg: int):
        """Segments of the streamed direction (work units = tiles x nseg)."""
        nseg = max(1, min(int(nseg), self.nq[-1]))
        tiles = self.units // self.nseg
        self.P.nseg = nseg
        self.nseg = nseg
        self.units = tiles * nseg

    def set_src_rows(self, lead2: int):
        rows = _src_rows(self.ndim, self.op, self.st, self.sym, lead2)
        for s in range(9):
            self.P.src_row[s] = rows[s] if s < len(rows) else 0

    def pack(self, coefs: torch.Tensor, lead2: int) -> torch.Tensor:
        """Pack a reference-layout coefficient tensor (flattened leading dims)."""
        self.set_src_rows(lead2)
        packed = torch.empty(self.packed_elems, dtype=self.dtype, device=coefs.device)
        ld = coefs.shape[-1]
        _lib.check(
            _lib.LIB.iga_mf_pack(ctypes.byref(self.P), iga_dtype(coefs.dtype), coefs.data_ptr(),
                                 ld, iga_dtype(self.dtype), packed.data_ptr(), stream_handle())
        )
        return packed

    def matvec(self, packed: torch.Tensor, x: torch.Tensor, y: torch.Tensor, ncols: int = 1):
        """y = A x; x, y hold `ncols` columns of N entries each (column after column)."""
        _lib.check(
            _lib.LIB.iga_mf_matvec(ctypes.byref(self.P), iga_dtype(self.dtype), packed.data_ptr(),
                                   ncols, x.data_ptr(), y.data_ptr(), stream_handle())
        )

    def check_status(self):
        st = int(self.status.item())
        if st != 0:
            self.status.zero_()
            _lib.check(st)


# ======================================================= operator object
def _coef_layout(op: int, coefs: torch.Tensor, ndim: int, st: int, Nq: int):
    """Validate the reference coefficient shape; return (flat 2D tensor, lead2)."""
    spd = ndim - 1 if st else ndim
    if op == _lib.IGA_OP_MASS:
        if coefs.shape[-1] != Nq or coefs.numel() != Nq:
            raise ValueError(f"mass coefficients must have shape ({Nq},), got {tuple(coefs.shape)}")
        return coefs.reshape(1, Nq), 1
    if op == _lib.IGA_OP_STIFF:
        if coefs.ndim != 3 or coefs.shape[-1] != Nq or coefs.shape[0] < spd or coefs.shape[1] < spd:
            raise ValueError(
                f"stiffness coefficients must have shape (d, d, {Nq}), got {tuple(coefs.shape)}"
            )
        return coefs.reshape(-1, Nq), coefs.shape[1]
    if coefs.ndim != 2 or coefs.shape[-1] != Nq or coefs.shape[0] < spd:
        raise ValueError(f"coefficients must have shape (d, {Nq}), got {tuple(coefs.shape)}")
    return coefs, 1


class MFOperator:
    """y = A x for one matrix-free operator of one patch, device-resident.

    Same arithmetic as ``BsplineOperations.compute_mf_scalar_<op>(quadrule_list,
    coefficients, x, time_ders)``; the coefficients are packed once (fused
    path) so repeated applies stream them straight from HBM.  ``kernel``:
    "pencil" -- the pencil kernel (every fused pattern); "tile" -- the FP64
    tensor-core tile kernel (3D stiffness with symmetric coefficients and
    mass, band width <= 5; ``igaops_b200.tile3d``); "auto" -- with
    ``nseg="auto"``, the autotuner times both on this operator where the
    tile kernel applies and keeps the faster (cached per shape; on B200 the
    pencil kernel wins, e.g. 3D p3 128^3 stiffness 0.91 ms against the tile
    kernel's 1.2-1.6 ms), otherwise the pencil kernel.
    ``nseg``: the pencil kernel's segment count of the streamed direction
    (None: heuristic; "auto": timed by ``igaops_b200.tune`` on this operator
    and cached per shape).
    """

    def __init__(self, quadrule_list, coefficients, op: str = "gradu_gradv", time_ders=None,
                 dtype: torch.dtype = torch.float64, nseg=None,
                 force_generic: bool = False, kernel: str = "auto",
                 symmetric: Optional[bool] = None):
        dev = require_cuda()
        if op not in _OPS:
            raise ValueError(f"unknown operator {op!r}; one of {sorted(_OPS)}")
        self.quadrule_list = list(quadrule_list)
        self.op_name = op
        self.op = _OPS[op]
        self.time_ders = None if time_ders is None else (int(time_ders[0]), int(time_ders[1]))
        self.dtype = dtype
        ndim = len(self.quadrule_list)
        self.ndim = ndim
        st, tt, tr = _spacetime(self.time_ders)
        self.n = [int(q.nbctrlpts) for q in self.quadrule_list]
        self.nq = [int(q.nbquadpts) for q in self.quadrule_list]
        self.N = math.prod(self.n)
        self.Nq = math.prod(self.nq)
        cdtype = torch.float64 if dtype == torch.float64 else torch.float32
        coefs = to_device(coefficients, cdtype, dev)
        flat, lead2 = _coef_layout(self.op, coefs, ndim, st, self.Nq)
        rbs = [rule_bands(q) for q in self.quadrule_list]
        W = max(rb.width for rb in rbs)
        self.symmetric = None  # symmetry of the stiffness coefficients (fused path)
        self.fused = (
            not force_generic
            and all(rb.fusable for rb in rbs)
            and 3 <= W <= 6
            and _fused_supported(ndim, self.op, st, tt, tr)
        )
        if self.fused:
            sym = False
            if self.op == _lib.IGA_OP_STIFF:
                spd = ndim - 1 if st else ndim
                if symmetric is not None:
                    # the caller checked these coefficients already (e.g. for
                    # the operator of the other precision)
                    sym = bool(symmetric)
                elif isinstance(coefficients, np.ndarray):
                    # host input: compare on the host, no device round trip
                    sym = all(np.array_equal(coefficients[i, j], coefficients[j, i])
                              for i in range(spd) for j in range(i + 1, spd))
                else:
                    c = coefs[:spd, :spd]
                    sym = bool(torch.equal(c, c.transpose(0, 1)))
            td = self.time_ders
            if td is not None and self.op in (_lib.IGA_OP_MASS, _lib.IGA_OP_U_GRADV):
                # the reference indexes the weight list with time_ders[0] itself
                # for these two operators (bsplines_ops.py:310-313,421-425):
                # weights[1] = W01, which equals W00 for the rules fused here,
                # so the time test derivative seen by the kernel is 0
                td = (0, td[1])
            auto = isinstance(nseg, str)
            if auto and nseg != "auto":
                raise ValueError(f"nseg must be an int, None or 'auto', got {nseg!r}")
            if kernel not in ("auto", "tile", "pencil"):
                raise ValueError(f"kernel must be 'auto', 'tile' or 'pencil', got {kernel!r}")
            self.symmetric = sym
            from . import tile3d

            # the tile kernel's geometry check only where it can be chosen
            tile_ok = ((kernel == "tile" or (kernel == "auto" and auto and ndim == 3))
                       and tile3d.tile_supported(self.quadrule_list, self.op, sym,
                                                 self.time_ders, dtype))
            if kernel == "tile" and not tile_ok:
                raise NotImplementedError(
                    "the tile kernel covers 3D FP64 stiffness (symmetric coefficients) and mass "
                    "with band width <= 5 and no space-time derivatives")
            self.tiled = tile_ok and kernel == "tile"
            self.coefs = None
            if self.tiled:
                self.plan = tile3d.TilePlan(self.quadrule_list, self.op)
                self.packed = self.plan.pack(flat.contiguous(), lead2)
                return
            self.plan = FusedPlan(self.quadrule_list, self.op, td, sym, dtype,
                                  None if auto else nseg)
            self.packed = self.plan.pack(flat.contiguous(), lead2)
            if auto and ndim == 3:
                from .tune import choose_kernel, tune_nseg

                xt = torch.zeros(self.N, dtype=dtype, device=dev)
                yt = torch.empty_like(xt)
                tune_nseg(self.plan, self.packed, xt, yt)
                if kernel == "auto" and tile_ok:
                    # the autotuner also times the tile kernel's 3D tiling
                    def make_tile():
                        tp = tile3d.TilePlan(self.quadrule_list, self.op)
                        return tp, tp.pack(flat.contiguous(), lead2)

                    win, tile = choose_kernel(self.plan, self.packed, make_tile, xt, yt)
                    if win == "tile":
                        self.tiled = True
                        self.plan, self.packed = tile
        else:
            self.tiled = False
            self.plan = None
            self.packed = None
            self.coefs = coefs.to(dtype)

    # -- bytes streamed per apply (algorithmic): coefficient streams + x + y
    def algorithmic_bytes(self, ncols: int = 1) -> int:
        es = 8 if self.dtype == torch.float64 else 4
        if self.fused:
            S = self.plan.S if self.tiled else self.plan.nstream
        else:
            S = self.coefs.numel() // self.Nq
        return self.Nq * S * es + 2 * self.N * es * ncols

    def apply_into(self, x: torch.Tensor, y: torch.Tensor, ncols: int = 1):
        """Device hot path: x, y are contiguous device tensors, columns stacked."""
        if self.fused:
            self.plan.matvec(self.packed, x, y, ncols)
        else:
            xv = x.reshape(ncols, self.N).t().contiguous()
            yv = _generic_apply(self.quadrule_list, self.op, self.coefs, xv, self.time_ders, ncols)
            y.copy_(yv.reshape(self.N, ncols).t().reshape(y.shape))

    def __call__(self, array_in):
        return self.apply(array_in)

    def apply(self, array_in):
        x = to_device(array_in, self.dtype)
        if x.shape[0] != self.N:
            raise ValueError(f"array_in has {x.shape[0]} rows, the operator has {self.N} DOFs")
        if x.ndim == 1:
            y = torch.empty_like(x)
            self.apply_into(x, y, 1)
        else:
            k = math.prod(x.shape[1:])
            xc = x.reshape(self.N, k).t().contiguous()
            yc = torch.empty_like(xc)
            self.apply_into(xc, yc, k)
            y = yc.t().reshape(x.shape)
        return like_input(y.contiguous(), array_in)


# ============================================================ generic path
def _generic_apply(rules, op, coefs: torch.Tensor, x: torch.Tensor, time_ders, ncols: int):
    """Unfused device path: the reference's sequence of L-mode products and
    pointwise scalings (src/igaops/operators/bsplines_ops.py:290-429), each
    step a libigab200 kernel.  x is (N, ncols) C-order; returns (N, ncols)."""
    ndim = len(rules)
    st = time_ders is not None
    spd = ndim - 1 if st else ndim
    dtype = x.dtype
    dt = iga_dtype(dtype)
    Nq = math.prod(int(q.nbquadpts) for q in rules)
    N = math.prod(int(q.nbctrlpts) for q in rules)
    h = stream_handle()

    def basis(der):
        return [factor_for(q.basis[b], dtype) for q, b in zip(rules, der)]

    def weights(der):
        return [factor_for(q.weights[z], dtype) for q, z in zip(rules, der)]

    def scale(c: torch.Tensor, u: torch.Tensor, out: torch.Tensor, acc: bool):
        _lib.check(
            _lib.LIB.iga_pointwise_scale(dt, Nq, ncols, c.data_ptr(), 1, u.data_ptr(),
                                         out.data_ptr(), int(acc), h)
        )

    def add(src: torch.Tensor, dst: torch.Tensor, first: bool):
        _lib.check(
            _lib.LIB.iga_axpby(dt, src.numel(), 1.0, src.data_ptr(), 0.0 if first else 1.0,
                               dst.data_ptr(), h)
        )

    def zeros_list():
        return [0] * ndim

    y = torch.empty(N * ncols, dtype=dtype, device=x.device)
    if op == _lib.IGA_OP_MASS:
        b = zeros_list()
        if st:
            b[-1] = time_ders[1]
        tmp = _lmode_device(basis(b), x, ncols)
        bc = torch.empty_like(tmp)
        scale(coefs.reshape(-1), tmp, bc, False)
        a = zeros_list()
        if st:
            a[-1] = time_ders[0]
        return _lmode_device(weights(a), bc, ncols).reshape(N, ncols)
    if op == _lib.IGA_OP_STIFF:
        first = True
        bc = None
        for j in range(spd):
            beta = zeros_list()
            beta[j] = 1
            if st:
                beta[-1] = time_ders[1]
            tmp = _lmode_device(basis(beta), x, ncols)
            bc = torch.empty_like(tmp) if bc is None else bc
            for i in range(spd):
                alpha = zeros_list()
                alpha[i] = 1
                if st:
                    alpha[-1] = time_ders[0]
                zeta = [b + 2 * a for b, a in zip(beta, alpha)]
                scale(coefs[i, j].contiguous(), tmp, bc, False)
                add(_lmode_device(weights(zeta), bc, ncols), y, first)
                first = False
        return y.reshape(N, ncols)
    if op == _lib.IGA_OP_GRADU_V:
        beta = zeros_list()
        if st:
            beta[-1] = time_ders[1]
        tmp = _lmode_device(basis(beta), x, ncols)
        bc = torch.empty_like(tmp)
        for i in range(spd):
            alpha = zeros_list()
            alpha[i] = 1
            if st:
                alpha[-1] = time_ders[0]
            zeta = [b + 2 * a for b, a in zip(beta, alpha)]
            scale(coefs[i].contiguous(), tmp, bc, False)
            add(_lmode_device(weights(zeta), bc, ncols), y, i == 0)
        return y.reshape(N, ncols)
    # u_gradv
    acc = torch.empty(Nq * ncols, dtype=dtype, device=x.device)
    for i in range(spd):
        beta = zeros_list()
        beta[i] = 1
        if st:
            beta[-1] = time_ders[1]
        tmp = _lmode_device(basis(beta), x, ncols)
        scale(coefs[i].contiguous(), tmp, acc, i > 0)
    alpha = zeros_list()
    if st:
        alpha[-1] = time_ders[0]
    return _lmode_device(weights(alpha), acc, ncols).reshape(N, ncols)


# ====================================================== reference facade
class BsplineOperations:
    """GPU drop-in for the matrix-free methods of the reference class
    (src/igaops/operators/bsplines_ops.py:56-429)."""

    @staticmethod
    def eval_jacobien(basis_list, u_at_ctrlpts, nurbs_weights=np.array([]), along_axis=False):
        """J[i, j] = d u_i / d xi_j at the quadrature points (bsplines_ops.py:88-114)."""
        if along_axis:
            raise NotImplementedError("along_axis evaluation is outside the matrix-free path")
        ndim = len(basis_list)
        u = u_at_ctrlpts
        nm = u.shape[0]
        rows = []
        for i in range(nm):
            comp = []
            for j in range(ndim):
                der = [1 if k == j else 0 for k in range(ndim)]
                comp.append(MatrixFree.apply([b[d] for b, d in zip(basis_list, der)], u[i]))
            rows.append(comp)
        return _stack(rows)

    @staticmethod
    def eval_interpolation(basis_list, u_at_ctrlpts, nurbs_weights=np.array([]), along_axis=False):
        if along_axis:
            raise NotImplementedError("along_axis evaluation is outside the matrix-free path")
        return _stack([MatrixFree.apply([b[0] for b in basis_list], u) for u in u_at_ctrlpts])

    @staticmethod
    def eval_hessian(basis_list, u_at_ctrlpts, nurbs_weights=np.array([]), along_axis=False):
        if along_axis:
            raise NotImplementedError("along_axis evaluation is outside the matrix-free path")
        ndim = len(basis_list)
        nm = u_at_ctrlpts.shape[0]
        out = [[[None] * ndim for _ in range(ndim)] for _ in range(nm)]
        for i in range(nm):
            for j in range(ndim):
                for k in range(j, ndim):
                    z = [0] * ndim
                    z[j] += 1
                    z[k] += 1
                    v = MatrixFree.apply([b[zz] for b, zz in zip(basis_list, z)], u_at_ctrlpts[i])
                    out[i][j][k] = out[i][k][j] = v
        return _stack(out)

    @staticmethod
    def _mf(op, quadrule_list, coefficients, array_in, time_ders):
        dtype = compute_dtype(array_in)
        oper = _operator_for(quadrule_list, coefficients, op, time_ders, dtype)
        return oper.apply(array_in)

    @staticmethod
    def compute_mf_scalar_u_v(quadrule_list, coefficients, array_in, time_ders=None,
                              nurbs_weights=np.array([])):
        return BsplineOperations._mf("u_v", quadrule_list, coefficients, array_in, time_ders)

    @staticmethod
    def compute_mf_scalar_gradu_gradv(quadrule_list, coefficients, array_in, time_ders=None,
                                      nurbs_weights=np.array([])):
        return BsplineOperations._mf("gradu_gradv", quadrule_list, coefficients, array_in,
                                     time_ders)

    @staticmethod
    def compute_mf_scalar_gradu_v(quadrule_list, coefficients, array_in, time_ders=None,
                                  nurbs_weights=np.array([])):
        return BsplineOperations._mf("gradu_v", quadrule_list, coefficients, array_in, time_ders)

    @staticmethod
    def compute_mf_scalar_u_gradv(quadrule_list, coefficients, array_in, time_ders=None,
                                  nurbs_weights=np.array([])):
        return BsplineOperations._mf("u_gradv", quadrule_list, coefficients, array_in, time_ders)


def _stack(nested):
    """Stack nested lists of equal arrays (numpy or torch)."""
    def leaf(x):
        return x

    def rec(v):
        if isinstance(v, list):
            parts = [rec(w) for w in v]
            if isinstance(parts[0], torch.Tensor):
                return torch.stack(parts)
            return np.stack(parts)
        return leaf(v)

    return rec(nested)


# Operators built from torch coefficient tensors are reused while the tensor
# is unchanged (same storage, shape, dtype and version counter).  numpy
# coefficients are packed on every call: numpy arrays can change in place
# without notice.
_OP_CACHE: "dict[tuple, MFOperator]" = {}
_OP_CACHE_MAX = 4


def _operator_for(quadrule_list, coefficients, op, time_ders, dtype) -> MFOperator:
    if isinstance(coefficients, torch.Tensor) and coefficients.is_cuda:
        key = (
            tuple(id(q) for q in quadrule_list),
            op,
            None if time_ders is None else tuple(int(t) for t in time_ders),
            dtype,
            coefficients.data_ptr(),
            tuple(coefficients.shape),
            tuple(coefficients.stride()),
            coefficients.dtype,
            coefficients._version,
        )
        hit = _OP_CACHE.get(key)
        if hit is not None and all(a is b for a, b in zip(hit.quadrule_list, quadrule_list)):
            return hit
        oper = MFOperator(quadrule_list, coefficients, op, time_ders, dtype)
        if len(_OP_CACHE) >= _OP_CACHE_MAX:
            _OP_CACHE.pop(next(iter(_OP_CACHE)))
        _OP_CACHE[key] = oper
        return oper
    return MFOperator(quadrule_list, coefficients, op, time_ders, dtype)
