"""Oracle: spatial fast-diagonalisation preconditioner (numpy / scipy).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).  Restates
src/igaops/fastdiag/utils/space_precond.py:124-320 and
src/igaops/common/math.py:10-90 for one DOF per node.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List

import numpy as np
import scipy.linalg as sclin
import scipy.sparse as sp

from .mf import lmode_apply

TINY = 1e-8
SAFEGUARD = 1e-14


def kron_sum(vals: List[np.ndarray], coefs) -> np.ndarray:
    """sum_i c_i (1 x .. x lambda_i x .. x 1), direction 1 fastest (math.py:10-58)."""
    total = None
    for i, v in enumerate(vals):
        parts = [np.ones_like(w) for w in vals]
        parts[i] = v * coefs[i]
        out = parts[0]
        for w in parts[1:]:
            out = np.kron(w, out)
        total = out if total is None else total + out
    return total


@dataclass
class FDData:
    U: List[np.ndarray]
    lam: List[np.ndarray]
    free: np.ndarray
    eig: np.ndarray
    n: List[int]


def setup(gauss_rules, table: np.ndarray, scalar_coefs=(0.0, 1.0), stiff_corr=None,
          mass_corr=1.0) -> FDData:
    """One DOF per node: eigh of the Gauss pencils minus Dirichlet rows
    (space_precond.py:124-193), then the combined eigenvalues (:195-236)."""
    ndim = len(gauss_rules)
    U, lam, idx_all, n = [], [], [], []
    for d, q in enumerate(gauss_rules):
        M = sp.csr_array(q.weights[0] @ q.basis[0]).toarray()
        K = sp.csr_array(q.weights[-1] @ q.basis[-1]).toarray()
        nn = M.shape[0]
        a = 1 if table[0, d, 0] else 0
        b = nn - 1 if table[0, d, 1] else nn
        idx = np.arange(a, b)
        Bm = M[np.ix_(idx, idx)]
        Am = K[np.ix_(idx, idx)]
        if nn == len(idx):
            Am = Am + TINY * Bm
        w, V = sclin.eigh(Am, Bm)
        U.append(V)
        lam.append(w)
        idx_all.append(idx)
        n.append(nn)
    corr = np.ones(ndim) if stiff_corr is None else np.asarray(stiff_corr)
    mixed = kron_sum(lam, corr)
    eig = scalar_coefs[0] * mass_corr * np.ones_like(mixed) + scalar_coefs[1] * mixed
    eig = np.maximum(eig, SAFEGUARD * np.max(eig))
    # free nodes: tensor of index ranges, direction 1 fastest
    free = np.zeros(1, dtype=np.int64)
    stride = 1
    flat = None
    for d in range(ndim):
        term = idx_all[d] * stride
        flat = term if flat is None else (term[:, None] + flat[None, :]).reshape(-1)
        stride *= n[d]
    return FDData(U=U, lam=lam, free=flat, eig=eig, n=n)


def apply(fd: FDData, x: np.ndarray) -> np.ndarray:
    """P^{-1} x on the free nodes, zero elsewhere (space_precond.py:273-320)."""
    out = np.zeros_like(x, dtype=float)
    v = x[fd.free]
    t = lmode_apply(fd.U, v, transpose=True)
    t = t / fd.eig.reshape((-1,) + (1,) * (t.ndim - 1))
    out[fd.free] = lmode_apply(fd.U, t, transpose=False)
    return out
