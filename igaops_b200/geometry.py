"""Geometry of a tensor-product spline patch at the quadrature points.

* ``GeometryOps``      -- src/igaops/geometry/mixin/operations.py:7-159
* ``SingleSpline``     -- src/igaops/geometry/mixin/template.py:16-130
* ``precompute_coefficients`` -- the coefficient tensors the matrix-free
  operators take: det J (mass) and det J * J^+ J^{+T} (stiffness), built
  on the device (the reference leaves this einsum to the caller,
  tests/test_assemble.py:116-123).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional

import numpy as np
import torch

from . import _lib
from ._device import like_input, stream_handle, to_device
from .bands import factor_for
from .operators import _lmode_device


class GeometryOps:
    @staticmethod
    def make_open_knotvector(degree: int, nbel: int, multiplicity: int = 1) -> np.ndarray:
        """Open uniform knot vector on [0, 1] (operations.py:8-30)."""
        inner = np.linspace(0.0, 1.0, nbel + 1)[1:-1]
        return np.concatenate([np.zeros(degree + 1), np.repeat(inner, multiplicity),
                               np.ones(degree + 1)])

    @staticmethod
    def evaluate_greville(degree: int, knotvector: np.ndarray) -> np.ndarray:
        """Greville abscissae: means of p consecutive interior knots (:54-71)."""
        U = np.asarray(knotvector, dtype=float)
        n = len(U) - degree - 1
        c = np.concatenate([[0.0], np.cumsum(U)])
        return (c[np.arange(n) + degree + 1] - c[np.arange(n) + 1]) / degree

    @staticmethod
    def inverse_rectangular_matrix(jac):
        """(det J, J^+) from J (m, n, ...) on the device (:137-159)."""
        J = to_device(jac, torch.float64)
        m, n = J.shape[0], J.shape[1]
        tail = tuple(J.shape[2:])
        nq = int(math.prod(tail)) if tail else 1
        det, inv, _ = _pointwise(J.reshape(m, n, nq), want_inv=True, want_coef=False)
        det = det.reshape(tail)
        inv = inv.reshape((n, m) + tail)
        return like_input(det, jac), like_input(inv, jac)


def _pointwise(J: torch.Tensor, want_inv: bool, want_coef: bool, want_det: bool = True):
    """Run the geometry kernel on J (M, D, nq); raise like the reference."""
    M, D, nq = J.shape
    dev = J.device
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    det = torch.empty(nq, dtype=torch.float64, device=dev) if want_det else None
    inv = torch.empty((D, M, nq), dtype=torch.float64, device=dev) if want_inv else None
    coef = torch.empty((D, D, nq), dtype=torch.float64, device=dev) if want_coef else None
    _lib.check(
        _lib.LIB.iga_geometry_pointwise(
            D, M, nq, J.data_ptr(), None if det is None else det.data_ptr(),
            None if inv is None else inv.data_ptr(), None if coef is None else coef.data_ptr(),
            status.data_ptr(), stream_handle())
    )
    st = int(status.item())
    if st & 1:
        raise ZeroDivisionError("There are near to zero determinants")
    if st & 2:
        raise ValueError("Potential geometry issue: some quadrature points have detJ <= 0")
    return det, inv, coef


def jacobian(quadrule_list, ctrlpts) -> torch.Tensor:
    """J[m, j] = d x_m / d xi_j at all quadrature points, shape (M, D, Nq)."""
    P = to_device(ctrlpts, torch.float64)
    D = len(quadrule_list)
    M = P.shape[0]
    nq = math.prod(int(q.nbquadpts) for q in quadrule_list)
    J = torch.empty((M, D, nq), dtype=torch.float64, device=P.device)
    for j in range(D):
        facs = [factor_for(q.basis[1 if k == j else 0], torch.float64)
                for k, q in enumerate(quadrule_list)]
        for m in range(M):
            J[m, j] = _lmode_device(facs, P[m].contiguous(), 1)
    return J


def precompute_coefficients(quadrule_list, ctrlpts, stiffness: bool = True,
                            mass: bool = True):
    """Device coefficient tensors of the perturbed geometry.

    Returns a dict with ``"stiffness"`` (D, D, Nq) = det J * J^+ J^{+T} and
    ``"mass"`` (Nq,) = det J, both float64 on the device.
    """
    J = jacobian(quadrule_list, ctrlpts)
    det, _, coef = _pointwise(J, want_inv=False, want_coef=stiffness, want_det=True)
    del J
    out = {}
    if stiffness:
        out["stiffness"] = coef
    if mass:
        out["mass"] = det
    return out


@dataclass
class EvaluatedSpline:
    ctrlpts: object
    nurbs_weights: np.ndarray
    qp_phy: object
    jac: object
    det_jac: object
    inv_jac: object
    quadrule_list: list


class SingleSpline:
    """Spline patch: control points + quadrature rules (template.py:16-130)."""

    def __init__(self, ctrlpts, nurbs_weights, quadrule_list: List):
        self.ctrlpts = ctrlpts
        self.nurbs_weights = np.asarray(nurbs_weights)
        self.quadrule_list = list(quadrule_list)

    @property
    def ndim(self):
        return len(self.quadrule_list)

    @property
    def nbctrlpts(self):
        return np.asarray([q.nbctrlpts for q in self.quadrule_list], dtype=int)

    @property
    def nbquadpts(self):
        return np.asarray([q.nbquadpts for q in self.quadrule_list], dtype=int)

    def evaluate_spline(self) -> EvaluatedSpline:
        if self.nurbs_weights.size > 0:
            # rational geometry (template.py:100-107 with NurbsOperations)
            from .nurbs import NurbsOperations

            basis = [q.basis for q in self.quadrule_list]
            P = to_device(self.ctrlpts, torch.float64)
            J = NurbsOperations.eval_jacobien(basis, P, nurbs_weights=self.nurbs_weights)
            qp = NurbsOperations.eval_interpolation(basis, P, nurbs_weights=self.nurbs_weights)
            det, inv, _ = _pointwise(J.contiguous(), want_inv=True, want_coef=False)
        else:
            J = jacobian(self.quadrule_list, self.ctrlpts)
            det, inv, _ = _pointwise(J, want_inv=True, want_coef=False)
            P = to_device(self.ctrlpts, torch.float64)
            facs = [factor_for(q.basis[0], torch.float64) for q in self.quadrule_list]
            qp = torch.stack([_lmode_device(facs, P[m].contiguous(), 1) for m in range(P.shape[0])])
        tmpl = self.ctrlpts
        return EvaluatedSpline(
            ctrlpts=self.ctrlpts,
            nurbs_weights=self.nurbs_weights.copy(),
            qp_phy=like_input(qp, tmpl),
            jac=like_input(J, tmpl),
            det_jac=like_input(det, tmpl),
            inv_jac=like_input(inv, tmpl),
            quadrule_list=list(self.quadrule_list),
        )


def unit_cube_ctrlpts(quadrule_list, amplitude: float = 0.0, phase: float = 0.0,
                      ncoord: Optional[int] = None) -> np.ndarray:
    """Greville control net of the unit cube/square, each coordinate displaced
    by amplitude * h * prod_k sin(2 pi (x_k + phase)), h = 1 / elements of
    direction 1.  The displacement vanishes on the boundary when phase = 0.
    Returns (ncoord, N) with the first direction fastest."""
    D = len(quadrule_list)
    ncoord = ncoord or D
    g = [GeometryOps.evaluate_greville(q.degree, q.knotvector) for q in quadrule_list]
    grids = np.meshgrid(*g[::-1], indexing="ij")[::-1]  # grids[k]: coordinate k, C order
    coords = [gk.reshape(-1) for gk in grids]
    h = 1.0 / (len(quadrule_list[0].unique_kv) - 1)
    disp = amplitude * h * np.prod([np.sin(2 * np.pi * (c + phase)) for c in coords], axis=0)
    out = np.zeros((ncoord, coords[0].shape[0]))
    for k in range(D):
        out[k] = coords[k] + (disp if amplitude else 0.0)
    return out
