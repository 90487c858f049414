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


# ------------------------------------------------------------ space-time
@dataclass
class SpTmData:
    space: FDData
    Ut: np.ndarray        # time eigenvectors (complex, mt x mt), Ut^H Mt Ut = I
    dt: np.ndarray        # diagonal of the arrowhead time block (complex, mt)
    g: np.ndarray         # its border (complex, mt - 1)
    nt: int
    adv: float = 1.0


def sptime_setup(space_gauss_rules, table, time_gauss_rule, scalar_coefs=(0.0, 1.0),
                 adv_corr=1.0) -> SpTmData:
    """Arrowhead space-time FD (time_arrow.py:44-98, time_template.py:49-64):
    the time pencil (advection, mass) minus the first time DOF, eigenvectors
    of its leading block normalised in the mass inner product, plus the
    mass-orthogonal last vector [v, 1]."""
    space = setup(space_gauss_rules, table, scalar_coefs)
    q = time_gauss_rule
    Mt_full = sp.csr_array(q.weights[0] @ q.basis[0]).toarray()
    Wt_full = sp.csr_array(q.weights[1] @ q.basis[1]).toarray()
    nt = Mt_full.shape[0]
    idx = np.arange(1, nt)
    Wt = Wt_full[np.ix_(idx, idx)]
    Mt = Mt_full[np.ix_(idx, idx)]
    Wp, Mp = Wt[:-1, :-1], Mt[:-1, :-1]
    m, w = Mt[:-1, -1], Wt[:-1, -1]
    D, V = sclin.eig(Wp, Mp)
    for i in range(V.shape[1]):
        u = V[:, i].copy()
        V[:, i] /= np.sqrt(np.abs(u.conj() @ Mp @ u))
    v = np.linalg.solve(Mp, -m)
    v1 = np.concatenate([v, [1.0]])
    kr = v1 / np.sqrt(v1 @ (Mt @ v1))
    k = kr[:-1]
    Ut = np.zeros((len(idx), len(idx)), dtype=complex)
    Ut[:-1, :-1] = V
    Ut[:-1, -1] = k
    Ut[-1, -1] = kr[-1]
    g = V.conj().T @ (np.hstack([Wp, w[:, None]]) @ kr)
    sigma = kr @ (Wt @ kr)
    dt = np.concatenate([D, [sigma]])
    return SpTmData(space=space, Ut=Ut, dt=dt, g=np.ravel(g), nt=nt, adv=adv_corr)


def arrowhead_solve(H, bfac, rhs):
    """operations.py:5-93 for one right-hand side: H (k+1, m), bfac (k,)."""
    Htop, Hlast = H[:-1], H[-1]
    schur = Hlast + np.sum((np.abs(bfac) ** 2)[:, None] / Htop, axis=0)
    r = rhs.reshape(H.shape)
    y = r[:-1] / Htop
    rs = r[-1] + np.tensordot(np.conj(bfac), y, axes=(0, 0))
    xl = rs / schur
    xt = y - (bfac[:, None] / Htop) * xl[None, :]
    return np.concatenate([xt, xl[None, :]], axis=0).ravel()


def sptime_apply(fd: SpTmData, x: np.ndarray, transpose: bool = False) -> np.ndarray:
    """time_arrow.py:112-192 for one DOF per node: free nodes = time indices
    1..nt-1 times the spatial free nodes (time slowest)."""
    Ns = int(np.prod(fd.space.n))
    free = (np.arange(1, fd.nt)[:, None] * Ns + fd.space.free[None, :]).reshape(-1)
    g = fd.adv * fd.g
    bfac = -np.conj(g) if transpose else g
    H = np.add.outer(fd.adv * fd.dt, fd.space.eig)
    Uf = fd.Ut if transpose else fd.Ut.conj()
    Ub = fd.Ut.conj() if transpose else fd.Ut
    a1 = lmode_apply(list(fd.space.U) + [Uf], x[free].astype(complex), transpose=True)
    a2 = arrowhead_solve(H, bfac, a1)
    out = np.zeros_like(x, dtype=float)
    out[free] = np.real(lmode_apply(list(fd.space.U) + [Ub], a2, transpose=False))
    return out


@dataclass
class SpTmQZData:
    space: FDData
    S: np.ndarray         # complex Schur form of the advection pencil
    T: np.ndarray         # complex Schur form of the mass pencil
    Q: np.ndarray         # left Schur vectors (W = Q S Z^H, M = Q T Z^H)
    Z: np.ndarray         # right Schur vectors
    nt: int
    adv: float = 1.0


def sptime_qz_setup(space_gauss_rules, table, time_gauss_rule, scalar_coefs=(0.0, 1.0),
                    adv_corr=1.0) -> SpTmQZData:
    """QZ ("legacy") space-time FD (time_legacy.py:43-52, time_template.py:
    46-59): the same time pencil, reduced by scipy.linalg.qz(W, M,
    output="complex")."""
    space = setup(space_gauss_rules, table, scalar_coefs)
    q = time_gauss_rule
    Mt_full = sp.csr_array(q.weights[0] @ q.basis[0]).toarray()
    Wt_full = sp.csr_array(q.weights[1] @ q.basis[1]).toarray()
    nt = Mt_full.shape[0]
    idx = np.arange(1, nt)
    S, T, Q, Z = sclin.qz(Wt_full[np.ix_(idx, idx)], Mt_full[np.ix_(idx, idx)], output="complex")
    return SpTmQZData(space=space, S=S, T=T, Q=Q, Z=Z, nt=nt, adv=adv_corr)


def sptime_qz_apply(fd: SpTmQZData, x: np.ndarray, transpose: bool = False) -> np.ndarray:
    """time_legacy.py:61-170 for one DOF per node and one column: Q^H (or
    Z^T) in time, one triangular solve per spatial eigen-index, Z (or
    conj(Q))."""
    Ns = int(np.prod(fd.space.n))
    free = (np.arange(1, fd.nt)[:, None] * Ns + fd.space.free[None, :]).reshape(-1)
    mt = fd.nt - 1
    Uf = fd.Z if transpose else fd.Q.conj()
    Ub = fd.Q.conj() if transpose else fd.Z
    a1 = lmode_apply(list(fd.space.U) + [Uf], x[free].astype(complex), transpose=True)
    rows = np.reshape(a1, (-1, mt), order="F")
    out_rows = np.zeros_like(rows)
    for j, row in enumerate(rows):
        mat = fd.adv * fd.S + fd.space.eig[j] * fd.T
        if transpose:
            out_rows[j] = sclin.solve_triangular(mat.T, row, lower=True)
        else:
            out_rows[j] = sclin.solve_triangular(mat, row, lower=False)
    a2 = np.reshape(out_rows, (-1,), order="F")
    out = np.zeros_like(x, dtype=float)
    out[free] = np.real(lmode_apply(list(fd.space.U) + [Ub], a2, transpose=False))
    return out
