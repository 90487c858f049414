"""Oracle: rational (NURBS) matrix-free operators and evaluations (numpy).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).  Restates
src/igaops/operators/nurbs_ops.py:14-62 (weight projections), 80-213
(evaluations) and 320-463 (matrix-free operators) on top of oracle.mf.
"""
from __future__ import annotations

import numpy as np

from . import mf


def project_weights(basis_list, w, nders):
    """(1/W, dW/W^2, H/W^3) at the quadrature points (nurbs_ops.py:14-62)."""
    ndim = len(basis_list)
    W = mf.lmode_apply([b[0] for b in basis_list], w)
    inv = 1.0 / W
    z = h = None
    if nders >= 1:
        z = mf.eval_jacobian(basis_list, w[None, :])[0] * inv ** 2
    if nders >= 2:
        h = np.zeros((ndim, ndim, W.size))
        for j in range(ndim):
            for k in range(j, ndim):
                der = [0] * ndim
                der[j] += 1
                der[k] += 1
                h[j, k] = h[k, j] = mf.lmode_apply([b[d] for b, d in zip(basis_list, der)], w)
        h = h * inv ** 3
    return inv, z, h


def eval_interpolation(basis_list, u, w):
    """nurbs_ops.py:196-213."""
    inv, _, _ = project_weights(basis_list, w, 0)
    return mf.eval_interpolation(basis_list, u * w[None, :]) * inv[None, :]


def eval_jacobian(basis_list, u, w):
    """nurbs_ops.py:167-194: J_ij = d_j(u w)/W - u_proj z_j."""
    inv, z, _ = project_weights(basis_list, w, 1)
    us = u * w[None, :]
    jac = mf.eval_jacobian(basis_list, us) * inv[None, None, :]
    up = mf.eval_interpolation(basis_list, us)
    return jac - up[:, None, :] * z[None, :, :]


def eval_hessian(basis_list, u, w):
    """nurbs_ops.py:80-165."""
    ndim = len(basis_list)
    inv, z, h = project_weights(basis_list, w, 2)
    us = u * w[None, :]
    up = mf.eval_interpolation(basis_list, us)
    du = mf.eval_jacobian(basis_list, us)
    out = np.zeros((u.shape[0], ndim, ndim, inv.size))
    for i in range(u.shape[0]):
        for j in range(ndim):
            for k in range(j, ndim):
                der = [0] * ndim
                der[j] += 1
                der[k] += 1
                first = mf.lmode_apply([b[d] for b, d in zip(basis_list, der)], us[i]) * inv
                v = (first - du[i, j] * z[k] - du[i, k] * z[j]
                     + 2.0 * up[i] * z[j] * z[k] / inv - up[i] * h[j, k] / inv)
                out[i, j, k] = out[i, k, j] = v
    return out


def _scale_rows(x, w):
    return x * w.reshape((-1,) + (1,) * (x.ndim - 1))


def mf_nurbs(op, rules, coefs, x, w, time_ders=None):
    """NurbsOperations.compute_mf_scalar_<op> (nurbs_ops.py:320-463)."""
    basis = [q.basis for q in rules]
    ndim = len(rules)
    sp = ndim - 1 if time_ders is not None else ndim
    xs = _scale_rows(x, w)
    if op == "u_v":
        inv, _, _ = project_weights(basis, w, 0)
        y = mf.mf_u_v(rules, coefs * inv ** 2, xs, time_ders)
        return _scale_rows(y, w)
    inv, z, _ = project_weights(basis, w, 1)
    z = z[:sp]
    if op == "gradu_gradv":
        y = mf.mf_gradu_gradv(rules, coefs * inv ** 2, xs, time_ders)
        y = y + mf.mf_u_v(rules, np.einsum("ijq,iq,jq->q", coefs, z, z), xs, time_ders)
        y = y - mf.mf_u_gradv(rules, np.einsum("ijq,iq,q->jq", coefs, z, inv), xs, time_ders)
        y = y - mf.mf_gradu_v(rules, np.einsum("ijq,jq,q->iq", coefs, z, inv), xs, time_ders)
        return _scale_rows(y, w)
    first = mf.mf_gradu_v if op == "gradu_v" else mf.mf_u_gradv
    y = first(rules, coefs * inv ** 2, xs, time_ders)
    y = y - mf.mf_u_v(rules, np.einsum("iq,iq,q->q", coefs, z, inv), xs, time_ders)
    return _scale_rows(y, w)
