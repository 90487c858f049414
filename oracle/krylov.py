"""Oracle: the reference's GMRES and GCRO-DR solvers (numpy / scipy).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).  Restates
src/igaops/solvers/linear_solver.py:149-257,438-525 (GMRES with the
ConvergenceManager stopping rules of
src/igaops/solvers/utils/convergence_manager.py:156-327) and
src/igaops/solvers/deflated/gcrodr.py:188-373 with
src/igaops/solvers/deflated/helpers.py:13-265.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sclin
from numpy.linalg import lstsq, norm

SAFEGUARD = 1e-14


def _converged(tol, abs_err, rel_err=None, incr=None):
    """Any of: absolute < 1e-14, relative < max(tol, 1e-14), increment < same."""
    thr = max(tol, SAFEGUARD)
    if abs_err is not None and abs_err < SAFEGUARD:
        return True
    if rel_err is not None and rel_err < thr:
        return True
    if incr is not None and incr < thr:
        return True
    return False


def gmres(A, b, P=None, tol=1e-10, maxiters=100, cleandod=None, x0=None):
    """Unrestarted right-preconditioned GMRES keeping Z = P V, two modified
    Gram-Schmidt passes, least squares on the Hessenberg matrix each step.
    Returns (x, residual history, success, iterations)."""
    P = P or (lambda v: v)

    def mask(v):
        if cleandod is not None:
            v[cleandod] = 0.0

    def mv(v):
        mask(v)
        y = np.asarray(A(v))
        mask(y)
        return y

    def pc(v):
        mask(v)
        y = np.asarray(P(v))
        mask(y)
        return y

    b = np.array(b, dtype=float, copy=True)
    mask(b)
    if x0 is not None:
        x0 = np.array(x0, dtype=float, copy=True)
        mask(x0)
        b = b - mv(x0)
    x = np.zeros_like(b)
    r0 = float(norm(b))
    res = [1.0]
    if _converged(tol, r0):
        return (x + (x0 if x0 is not None else 0.0)), np.array(res), True, 0
    H = np.zeros((maxiters + 1, maxiters))
    V = np.zeros((maxiters + 1, b.shape[0]))
    Z = np.zeros_like(V)
    V[0] = b / r0
    success, it = False, 0
    for it in range(1, maxiters + 1):
        Z[it - 1] = pc(V[it - 1].copy())
        w = mv(Z[it - 1].copy())
        for _ in range(2):
            for j in range(it):
                h = w.dot(V[j])
                H[j, it - 1] += h
                w = w - h * V[j]
        nw = norm(w)
        H[it, it - 1] = nw
        if nw != 0:
            V[it] = w / nw
        Hm = H[: it + 1, :it]
        rhs = np.zeros(it + 1)
        rhs[0] = r0
        y = lstsq(Hm, rhs, rcond=None)[0]
        xold = x
        x = Z[: len(y)].T @ y
        incr = float(norm(x - xold) / (norm(x) + SAFEGUARD))
        r1 = float(norm(rhs - Hm @ y))
        res.append(r1 / r0)
        if _converged(tol, r1, res[-1], incr):
            success = True
            break
    if x0 is not None:
        x = x + x0
    return x, np.array(res), success, it


# --------------------------------------------------------------- GCRO-DR
def _gmres_cycle(A, M, x, r, m, tol, C=None):
    """m Arnoldi steps of M A (deflated against C when given)."""
    n = r.shape[0]
    V = np.zeros((m + 1, n), dtype=complex)
    H = np.zeros((m + 1, m), dtype=complex)
    B = None if C is None else np.zeros((C.shape[1], m), dtype=complex)
    resv = np.zeros(m)
    beta = norm(r)
    k = 1
    y = np.zeros(1, dtype=complex)
    res = np.array([beta], dtype=complex)
    if beta <= SAFEGUARD:
        return V, H, B, k, resv[:k], y, res
    V[0] = r / beta
    for k in range(1, m + 1):
        w = M(A(V[k - 1]))
        if C is not None:
            B[:, k - 1] = C.conj().T @ w
            w = w - C @ B[:, k - 1]
        for _ in range(2):
            for j in range(k):
                h = V[j].conj().dot(w)
                H[j, k - 1] += h
                w = w - h * V[j]
        nw = norm(w)
        H[k, k - 1] = nw
        if nw > 0.0:
            V[k] = w / nw
        Hm = H[: k + 1, :k]
        rhs = np.zeros(k + 1, dtype=complex)
        rhs[0] = beta
        y = np.linalg.lstsq(Hm, rhs, rcond=None)[0]
        res = rhs - Hm @ y
        resv[k - 1] = norm(res)
        if resv[k - 1] < tol:
            break
    return V, H, B, k, resv[:k], y, res


def _harm1(m, k, H):
    Hm = H[:m, :m]
    em = np.zeros(m, dtype=complex)
    em[-1] = 1.0
    f = np.linalg.solve(Hm.conj().T, em)
    G = Hm + (abs(H[m, m - 1]) ** 2) * np.outer(f, em.conj())
    vals, vecs = sclin.eig(G)
    good = np.isfinite(vals)
    vals, vecs = vals[good], vecs[:, good]
    return vecs[:, np.argsort(np.abs(vals))[:k]]


def _harm2(m, k, G, V, U, C):
    p = m - k
    Vt = np.hstack([U, V[:p].T])
    Wt = np.hstack([C, V[: p + 1].T])
    Phi = Wt.conj().T @ Vt
    vals, vecs = sclin.eig(G.conj().T @ G, G.conj().T @ Phi)
    good = np.isfinite(vals)
    vals, vecs = vals[good], vecs[:, good]
    return vecs[:, np.argsort(np.abs(vals))[:k]]


class GCRODR:
    """GCRO with deflated restarting; left preconditioned; complex128."""

    def __init__(self, tol, maxiters, m=40, k=20, max_cycles=10):
        self.tol, self.maxiters, self.m, self.k, self.max_cycles = tol, maxiters, m, k, max_cycles
        self.U = {}

    def solve(self, Afun, b, Pfun=None, key="default"):
        Pfun = Pfun or (lambda v: v)

        def A(v):
            v = np.asarray(v)
            if np.iscomplexobj(v):
                return Afun(np.real(v)) + 1j * Afun(np.imag(v))
            return Afun(v)

        def M(v):
            v = np.asarray(v)
            if np.iscomplexobj(v):
                return Pfun(np.real(v)) + 1j * Pfun(np.imag(v))
            return Pfun(v)

        m, k, tol = self.m, self.k, self.tol
        b = np.asarray(b, dtype=complex)
        x = np.zeros_like(b)
        r = M(b)
        r0 = float(norm(r))
        resvec = [r0]

        def rel(v):
            v = np.abs(np.asarray(v))
            return v / max(v[0], SAFEGUARD)

        if r0 < SAFEGUARD:
            return np.real(x), rel(resvec), True
        U = C = None
        nmv = 0
        if key in self.U:
            Y = self.U[key].copy()
            Cm = np.column_stack([M(A(Y[:, i])) for i in range(Y.shape[1])])
            C, R = np.linalg.qr(Cm, mode="reduced")
            U = sclin.solve_triangular(R.T, Y.T, lower=True).T
            cr = C.conj().T.dot(r)
            x = x + U @ cr
            r = r - C @ cr
            resvec.append(float(norm(r)))
            p = np.inf
        else:
            V, H, _, p, rv, y, res = _gmres_cycle(A, M, x, r, m, tol * r0)
            x = x + V[:p].T @ y
            r = V[: p + 1].T @ res
            resvec.extend(rv.tolist())
            nmv += p
            if p >= k:
                Pk = _harm1(p, k, H)
                Y = V[:p].T @ Pk
                Q, R = np.linalg.qr(H[: p + 1, :p] @ Pk, mode="reduced")
                C = V[: p + 1].T @ Q
                U = sclin.solve_triangular(R.T, Y.T, lower=True).T
        rn = float(norm(r))
        if nmv > self.maxiters:
            raise RuntimeError(f"Maximum iterations ({self.maxiters}) exceeded.")
        if _converged(tol, rn, rn / r0) or p < m:
            if U is not None:
                self.U[key] = U
            return np.real(x), rel(resvec), True
        success = False
        for _cycle in range(self.max_cycles):
            V, H, B, p, rv, _, _ = _gmres_cycle(A, M, None, r, m - k, tol * r0, C)
            resvec.extend(rv.tolist())
            nmv += p
            D = np.diag(1.0 / np.sqrt(np.diag(U.conj().T @ U)))
            Ut = U @ D
            Vh = np.hstack([Ut, V[:p].T])
            Wh = np.hstack([C, V[: p + 1].T])
            G = np.block([[D, B[:, :p]], [np.zeros((p + 1, k), dtype=complex), H[: p + 1, :p]]])
            y = np.linalg.lstsq(G, Wh.conj().T.dot(r), rcond=None)[0]
            x = x + Vh @ y
            r = r - Wh @ (G @ y)
            rn = float(norm(r))
            if nmv > self.maxiters:
                raise RuntimeError(f"Maximum iterations ({self.maxiters}) exceeded.")
            if _converged(tol, rn, rn / r0) or p < m - k:
                success = True
                break
            Pk = _harm2(p + k, k, G, V[: p + 1], Ut, C)
            Y = Vh @ Pk
            Q, R = np.linalg.qr(G @ Pk, mode="reduced")
            C = Wh @ Q
            U = sclin.solve_triangular(R.T, Y.T, lower=True).T
        self.U[key] = U
        return np.real(x), rel(resvec), success
