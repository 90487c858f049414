"""Rational (NURBS) matrix-free operators on the GPU.

GPU drop-in for ``NurbsOperations`` (src/igaops/operators/nurbs_ops.py:
79-463).  A NURBS operator is the B-spline operator applied to the weighted
input ``w_c * x`` and scaled by ``w_c`` again, with the per-point coefficients
replaced by terms of the interpolated weight ``W`` and its gradient
(nurbs_ops.py:14-62, 320-463):

* mass:      ``w_c * M[c/W^2] (w_c x)``
* stiffness: ``w_c * (K[C/W^2] + M[z^T C z] - UG[C^T z/W] - GU[C z/W]) (w_c x)``
  with ``z = dW / W^2``
* advection: ``w_c * (A[c/W^2] - M[c.z/W]) (w_c x)``

``NurbsMFOperator`` derives those coefficient streams once on the device
(``iga_nurbs_coefficients``) and keeps one fused operator per term, so an
apply is one pointwise scaling, one fused matvec per term and the
accumulation, all libigab200 kernels.
"""
from __future__ import annotations

import math
from typing import List

import numpy as np
import torch

from . import _lib
from ._device import compute_dtype, iga_dtype, like_input, require_cuda, stream_handle, to_device
from .bands import factor_for
from .operators import BsplineOperations, MFOperator, _lmode_device

__all__ = ["NurbsOperations", "NurbsMFOperator", "project_nurbs_weights"]


def _weights_at_qp(basis_list, nurbs_weights: torch.Tensor, nders: int):
    """W (Nq,) and, for nders >= 1, dW (ndim, Nq) at the quadrature points:
    the projections of the control weights (nurbs_ops.py:14-62), FP64."""
    ndim = len(basis_list)
    w = nurbs_weights.reshape(-1, 1)
    Wq = _lmode_device([factor_for(b[0], torch.float64) for b in basis_list], w, 1)
    if nders == 0:
        return Wq, None
    rows = []
    for k in range(ndim):
        fac = [factor_for(b[1 if j == k else 0], torch.float64) for j, b in enumerate(basis_list)]
        rows.append(_lmode_device(fac, w, 1))
    return Wq, torch.stack(rows).contiguous()


def project_nurbs_weights(basis_list, nurbs_weights, nders: int = 0):
    """(1/W, dW/W^2, H/W^3) at the quadrature points, as
    _Helpers.project_nurbs_weights (nurbs_ops.py:14-62); device tensors."""
    if nders < 0 or nders > 2:
        raise NotImplementedError("Number of derivatives should be positive and lower than 3")
    dev = require_cuda()
    w = to_device(nurbs_weights, torch.float64, dev).reshape(-1)
    Wq, dW = _weights_at_qp(basis_list, w, nders)
    inv = 1.0 / Wq
    if nders == 0:
        return inv, None, None
    z = dW * inv ** 2
    if nders == 1:
        return inv, z, None
    H = BsplineOperations.eval_hessian(basis_list, w.reshape(1, -1))[0]
    return inv, z, H * inv ** 3


class NurbsMFOperator:
    """y = A x for one NURBS matrix-free operator of one patch, device-resident
    (the arithmetic of ``NurbsOperations.compute_mf_scalar_<op>``)."""

    def __init__(self, quadrule_list, coefficients, nurbs_weights, op: str = "gradu_gradv",
                 time_ders=None, dtype: torch.dtype = torch.float64):
        dev = require_cuda()
        rules = list(quadrule_list)
        self.quadrule_list = rules
        self.op_name = op
        self.dtype = dtype
        ndim = len(rules)
        st = time_ders is not None
        sp = ndim - 1 if st else ndim
        self.N = math.prod(int(q.nbctrlpts) for q in rules)
        self.Nq = math.prod(int(q.nbquadpts) for q in rules)
        w64 = to_device(nurbs_weights, torch.float64, dev).reshape(-1)
        if w64.numel() != self.N:
            raise ValueError(f"nurbs_weights has {w64.numel()} entries, the patch has {self.N} DOFs")
        self.wc = w64.to(dtype)
        opc = {"u_v": _lib.IGA_OP_MASS, "gradu_gradv": _lib.IGA_OP_STIFF,
               "gradu_v": _lib.IGA_OP_GRADU_V, "u_gradv": _lib.IGA_OP_U_GRADV}.get(op)
        if opc is None:
            raise ValueError(f"unknown operator {op!r}")
        Wq, dW = _weights_at_qp([q.basis for q in rules], w64, 0 if opc == _lib.IGA_OP_MASS else 1)
        c = to_device(coefficients, torch.float64, dev)
        Nq = self.Nq
        if opc == _lib.IGA_OP_MASS:
            c = c.reshape(Nq)
        elif opc == _lib.IGA_OP_STIFF:
            if c.ndim != 3 or c.shape[0] < sp or c.shape[1] < sp or c.shape[2] != Nq:
                raise ValueError(f"stiffness coefficients must have shape ({sp}, {sp}, {Nq})")
            c = c[:sp, :sp].contiguous()
        else:
            if c.ndim != 2 or c.shape[0] < sp or c.shape[1] != Nq:
                raise ValueError(f"coefficients must have shape ({sp}, {Nq})")
            c = c[:sp].contiguous()
        main = torch.empty_like(c)
        uv = torch.empty(Nq, dtype=torch.float64, device=dev)
        ug = torch.empty((sp, Nq), dtype=torch.float64, device=dev)
        gu = torch.empty((sp, Nq), dtype=torch.float64, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        _lib.check(_lib.LIB.iga_nurbs_coefficients(
            opc, sp, Nq, c.data_ptr(), Wq.data_ptr(),
            None if dW is None else dW.data_ptr(), main.data_ptr(), uv.data_ptr(),
            ug.data_ptr(), gu.data_ptr(), status.data_ptr(), stream_handle()))
        if int(status.item()) != 0:
            raise ZeroDivisionError("the NURBS weight function vanishes at a quadrature point")
        td = time_ders
        self.terms: List[tuple] = [(1.0, MFOperator(rules, main, op, td, dtype))]
        if opc == _lib.IGA_OP_STIFF:
            self.terms += [(1.0, MFOperator(rules, uv, "u_v", td, dtype)),
                           (-1.0, MFOperator(rules, ug, "u_gradv", td, dtype)),
                           (-1.0, MFOperator(rules, gu, "gradu_v", td, dtype))]
        elif opc != _lib.IGA_OP_MASS:
            self.terms.append((-1.0, MFOperator(rules, uv, "u_v", td, dtype)))
        self._work = {}

    def algorithmic_bytes(self, ncols: int = 1) -> int:
        es = 8 if self.dtype == torch.float64 else 4
        return sum(t.algorithmic_bytes(ncols) for _, t in self.terms) + 2 * self.N * es * ncols

    def _buf(self, name, n, like):
        b = self._work.get(name)
        if b is None or b.numel() < n or b.device != like.device:
            b = torch.empty(n, dtype=self.dtype, device=like.device)
            self._work[name] = b
        return b[:n]

    def _scale(self, src: torch.Tensor, dst: torch.Tensor, ncols: int):
        dt, h = iga_dtype(self.dtype), stream_handle()
        for k in range(ncols):
            _lib.check(_lib.LIB.iga_pointwise_scale(
                dt, self.N, 1, self.wc.data_ptr(), 1, src[k * self.N:].data_ptr(),
                dst[k * self.N:].data_ptr(), 0, h))

    def apply_into(self, x: torch.Tensor, y: torch.Tensor, ncols: int = 1):
        """x, y: contiguous device tensors, columns stacked ((ncols, N))."""
        n = self.N * ncols
        xs = self._buf("xs", n, x)
        self._scale(x.reshape(-1), xs, ncols)
        yf = y.reshape(-1)
        self.terms[0][1].apply_into(xs, yf, ncols)
        if len(self.terms) > 1:
            tmp = self._buf("tmp", n, x)
            dt, h = iga_dtype(self.dtype), stream_handle()
            for sign, t in self.terms[1:]:
                t.apply_into(xs, tmp, ncols)
                _lib.check(_lib.LIB.iga_axpby(dt, n, sign, tmp.data_ptr(), 1.0, yf.data_ptr(), h))
        self._scale(yf, yf, ncols)

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


class NurbsOperations:
    """GPU drop-in for the matrix-free and evaluation methods of the
    reference class (src/igaops/operators/nurbs_ops.py:79-463).  Empty
    ``nurbs_weights`` fall back to the B-spline operators (all weights 1)."""

    # -------------------------------------------------------- evaluation
    @staticmethod
    def _scaled(u_at_ctrlpts, nurbs_weights):
        dev = require_cuda()
        u = to_device(u_at_ctrlpts, torch.float64, dev)
        w = to_device(nurbs_weights, torch.float64, dev).reshape(-1)
        return u * w[None, :], w

    @staticmethod
    def eval_interpolation(basis_list, u_at_ctrlpts, nurbs_weights=np.array([]), along_axis=False):
        """u(q) = sum_c N_c w_c u_c / W(q) (nurbs_ops.py:196-213)."""
        if np.size(nurbs_weights) == 0:
            return BsplineOperations.eval_interpolation(basis_list, u_at_ctrlpts,
                                                        along_axis=along_axis)
        if along_axis:
            raise NotImplementedError("along_axis evaluation is outside the matrix-free path")
        us, w = NurbsOperations._scaled(u_at_ctrlpts, nurbs_weights)
        inv, _, _ = project_nurbs_weights(basis_list, w, 0)
        out = BsplineOperations.eval_interpolation(basis_list, us) * inv[None, :]
        return like_input(out, u_at_ctrlpts)

    @staticmethod
    def eval_jacobien(basis_list, u_at_ctrlpts, nurbs_weights=np.array([]), along_axis=False):
        """d u_i / d xi_j of the rational interpolant (nurbs_ops.py:167-194)."""
        if np.size(nurbs_weights) == 0:
            return BsplineOperations.eval_jacobien(basis_list, u_at_ctrlpts, along_axis=along_axis)
        if along_axis:
            raise NotImplementedError("along_axis evaluation is outside the matrix-free path")
        us, w = NurbsOperations._scaled(u_at_ctrlpts, nurbs_weights)
        inv, z, _ = project_nurbs_weights(basis_list, w, 1)
        jac = BsplineOperations.eval_jacobien(basis_list, us) * inv[None, None, :]
        u_proj = BsplineOperations.eval_interpolation(basis_list, us)
        jac = jac - u_proj[:, None, :] * z[None, :, :]
        return like_input(jac, u_at_ctrlpts)

    @staticmethod
    def eval_hessian(basis_list, u_at_ctrlpts, nurbs_weights=np.array([]), along_axis=False):
        """Second parametric derivatives of the rational interpolant
        (nurbs_ops.py:80-165)."""
        if np.size(nurbs_weights) == 0:
            return BsplineOperations.eval_hessian(basis_list, u_at_ctrlpts, along_axis=along_axis)
        if along_axis:
            raise NotImplementedError("along_axis evaluation is outside the matrix-free path")
        us, w = NurbsOperations._scaled(u_at_ctrlpts, nurbs_weights)
        inv, z, h = project_nurbs_weights(basis_list, w, 2)
        hess = BsplineOperations.eval_hessian(basis_list, us) * inv
        u_proj = BsplineOperations.eval_interpolation(basis_list, us)   # (nm, Nq)
        du = BsplineOperations.eval_jacobien(basis_list, us)            # (nm, d, Nq)
        ndim = len(basis_list)
        out = torch.empty_like(hess)
        for j in range(ndim):
            for k in range(j, ndim):
                v = (hess[:, j, k] - du[:, j] * z[k] - du[:, k] * z[j]
                     + 2.0 * u_proj * z[j] * z[k] * (1.0 / inv)
                     - u_proj * h[j, k] * (1.0 / inv))
                out[:, j, k] = v
                out[:, k, j] = v
        return like_input(out, u_at_ctrlpts)

    # -------------------------------------------------------- matrix-free
    @staticmethod
    def _mf(op, quadrule_list, coefficients, array_in, time_ders, nurbs_weights):
        if np.size(nurbs_weights) == 0:
            return getattr(BsplineOperations, f"compute_mf_scalar_{op}")(
                quadrule_list, coefficients, array_in, time_ders=time_ders)
        oper = NurbsMFOperator(quadrule_list, coefficients, nurbs_weights, op, time_ders,
                               compute_dtype(array_in))
        return oper.apply(array_in)

    @staticmethod
    def compute_mf_scalar_u_v(quadrule_list, coefficients, array_in, time_ders=None,
                              nurbs_weights=np.array([])):
        return NurbsOperations._mf("u_v", quadrule_list, coefficients, array_in, time_ders,
                                   nurbs_weights)

    @staticmethod
    def compute_mf_scalar_gradu_gradv(quadrule_list, coefficients, array_in, time_ders=None,
                                      nurbs_weights=np.array([])):
        return NurbsOperations._mf("gradu_gradv", quadrule_list, coefficients, array_in,
                                   time_ders, nurbs_weights)

    @staticmethod
    def compute_mf_scalar_gradu_v(quadrule_list, coefficients, array_in, time_ders=None,
                                  nurbs_weights=np.array([])):
        return NurbsOperations._mf("gradu_v", quadrule_list, coefficients, array_in, time_ders,
                                   nurbs_weights)

    @staticmethod
    def compute_mf_scalar_u_gradv(quadrule_list, coefficients, array_in, time_ders=None,
                                  nurbs_weights=np.array([])):
        return NurbsOperations._mf("u_gradv", quadrule_list, coefficients, array_in, time_ders,
                                   nurbs_weights)
