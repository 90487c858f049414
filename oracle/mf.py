"""Oracle: Kronecker (L-mode) products and matrix-free operators (numpy).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).  Restates
src/igaops/operators/utils/matrix_free.py:9-119 and
src/igaops/operators/bsplines_ops.py:88-136,290-429.
"""
from __future__ import annotations

import numpy as np


def mode_product(tensor: np.ndarray, matrix, mode: int, transpose: bool = False) -> np.ndarray:
    """n-mode product along `mode` (matrix_free.py:39-75)."""
    mat = matrix.T if transpose else matrix
    moved = np.moveaxis(tensor, mode, 0)
    lead = moved.shape[0]
    flat = moved.reshape(lead, -1)
    out = np.asarray(mat @ flat)
    out = out.reshape((out.shape[0],) + moved.shape[1:])
    return np.moveaxis(out, 0, mode)


def lmode_apply(matrix_list, x: np.ndarray, transpose: bool = False) -> np.ndarray:
    """(M_n x ... x M_1) x  (matrix_free.py:77-119): the slowest direction is
    the first tensor mode (C order), each factor applied as a mode product."""
    mats = list(matrix_list)[::-1]
    shape = [m.shape[0 if transpose else 1] for m in mats]
    tail = x.shape[1:]
    t = np.reshape(x, shape + list(tail or (1,)))
    for i, m in enumerate(mats):
        t = mode_product(t, m, i, transpose)
    if x.ndim == 1:
        return t.ravel()
    return t.reshape((-1,) + tail)


def _lists(ndim, time_ders):
    st = time_ders is not None
    return (ndim - 1 if st else ndim), st


def mf_u_v(rules, coefs, x, time_ders=None):
    """Mass operator (bsplines_ops.py:290-317)."""
    ndim = len(rules)
    _, st = _lists(ndim, time_ders)
    b = np.zeros(ndim, dtype=int)
    if st:
        b[-1] = time_ders[1]
    tmp = lmode_apply([q.basis[k] for q, k in zip(rules, b)], x)
    a = np.zeros(ndim, dtype=int)
    if st:
        a[-1] = time_ders[0]
    scaled = coefs.reshape((-1,) + (1,) * (tmp.ndim - 1)) * tmp
    return lmode_apply([q.weights[k] for q, k in zip(rules, a)], scaled)


def mf_gradu_gradv(rules, coefs, x, time_ders=None):
    """Stiffness operator (bsplines_ops.py:319-355):
    y = sum_j sum_i W^(e_j + 2 e_i) [ C[i, j] * (B^(e_j) x) ]."""
    ndim = len(rules)
    spd, st = _lists(ndim, time_ders)
    y = np.zeros(x.shape, dtype=float)
    for j in range(spd):
        beta = np.zeros(ndim, dtype=int)
        beta[j] = 1
        if st:
            beta[-1] = time_ders[1]
        tmp = lmode_apply([q.basis[k] for q, k in zip(rules, beta)], x)
        for i in range(spd):
            alpha = np.zeros(ndim, dtype=int)
            alpha[i] = 1
            if st:
                alpha[-1] = time_ders[0]
            zeta = beta + 2 * alpha
            c = coefs[i, j].reshape((-1,) + (1,) * (tmp.ndim - 1))
            y += lmode_apply([q.weights[k] for q, k in zip(rules, zeta)], c * tmp)
    return y


def mf_gradu_v(rules, coefs, x, time_ders=None):
    """bsplines_ops.py:357-390: y = sum_i W^(beta + 2 e_i) [ c_i * (B^beta x) ]."""
    ndim = len(rules)
    spd, st = _lists(ndim, time_ders)
    y = np.zeros(x.shape, dtype=float)
    beta = np.zeros(ndim, dtype=int)
    if st:
        beta[-1] = time_ders[1]
    tmp = lmode_apply([q.basis[k] for q, k in zip(rules, beta)], x)
    for i in range(spd):
        alpha = np.zeros(ndim, dtype=int)
        alpha[i] = 1
        if st:
            alpha[-1] = time_ders[0]
        zeta = beta + 2 * alpha
        c = coefs[i].reshape((-1,) + (1,) * (tmp.ndim - 1))
        y += lmode_apply([q.weights[k] for q, k in zip(rules, zeta)], c * tmp)
    return y


def mf_u_gradv(rules, coefs, x, time_ders=None):
    """bsplines_ops.py:392-429: y = W^alpha [ sum_i c_i * (B^(e_i) x) ]."""
    ndim = len(rules)
    spd, st = _lists(ndim, time_ders)
    nq = int(np.prod([q.nbquadpts for q in rules]))
    acc = np.zeros((nq,) + x.shape[1:])
    for i in range(spd):
        beta = np.zeros(ndim, dtype=int)
        beta[i] = 1
        if st:
            beta[-1] = time_ders[1]
        tmp = lmode_apply([q.basis[k] for q, k in zip(rules, beta)], x)
        acc += coefs[i].reshape((-1,) + (1,) * (tmp.ndim - 1)) * tmp
    alpha = np.zeros(ndim, dtype=int)
    if st:
        alpha[-1] = time_ders[0]
    return lmode_apply([q.weights[k] for q, k in zip(rules, alpha)], acc)


OPS = {
    "u_v": mf_u_v,
    "gradu_gradv": mf_gradu_gradv,
    "gradu_v": mf_gradu_v,
    "u_gradv": mf_u_gradv,
}


def eval_jacobian(basis_list, u):
    """J[i, j] = d u_i / d xi_j (bsplines_ops.py:88-114)."""
    ndim = len(basis_list)
    out = np.zeros((u.shape[0], ndim, int(np.prod([b[0].shape[0] for b in basis_list]))))
    for i in range(u.shape[0]):
        for j in range(ndim):
            der = [1 if k == j else 0 for k in range(ndim)]
            out[i, j] = lmode_apply([b[d] for b, d in zip(basis_list, der)], u[i])
    return out


def eval_interpolation(basis_list, u):
    return np.stack([lmode_apply([b[0] for b in basis_list], ui) for ui in u])
