"""1D quadrature rules: the host-side setup inputs of the matrix-free path.

Each rule exposes the attributes the reference rules do
(src/igaops/quadrature/utils/template.py:15-129): ``degree``,
``knotvector``, ``nbctrlpts``, ``nbquadpts``, ``quadpts``, ``basis``
(``[B0, B1]``, CSR (nq, n): basis values / first derivatives at the
quadrature points) and ``weights`` (four CSR (n, nq) matrices indexed by
``trial_der + 2*test_der``).  The GPU operators consume them as banded
factors; they are built once per patch on the host, as in the reference.

* ``StandardGauss``       -- src/igaops/quadrature/gauss_quad.py:14-126
* ``WeightedQuadrature``  -- src/igaops/quadrature/weighted_quad.py:238-363
  with the point layout of src/igaops/quadrature/utils/wq_helpers.py:11-259

B-spline evaluation restates Piegl & Tiller, *The NURBS Book*, A2.1 (span
search) and A2.3 (basis derivatives), vectorised over evaluation points; the
reference delegates these to the third-party ``geomdl.helpers``.
"""
from __future__ import annotations

import logging
from typing import Callable, List, Literal, Optional, Tuple

import numpy as np
import scipy.sparse as sp

from .common import validate_entry

logger = logging.getLogger(__name__)


# ============================================================ B-splines
def find_spans(degree: int, knotvector: np.ndarray, x: np.ndarray) -> np.ndarray:
    """Knot span of each point: the last s in [p, n-1] with U[s] <= x."""
    U = np.asarray(knotvector, dtype=float)
    n = len(U) - degree - 1
    s = np.searchsorted(U, np.asarray(x, dtype=float), side="right") - 1
    return np.clip(s, degree, n - 1)


def basis_ders(degree: int, knotvector: np.ndarray, x: np.ndarray, nders: int = 1):
    """Non-zero basis functions and derivatives at points x, computed in the
    library's host code (``iga_bspline_basis``: Piegl & Tiller A2.1 / A2.3).

    Returns (span[m], ders[nders+1, p+1, m]) with ders[k, j] the k-th
    derivative of N_{span-p+j, p}.
    """
    import ctypes

    from . import _lib

    p = int(degree)
    U = np.ascontiguousarray(knotvector, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    m = x.shape[0]
    span = np.zeros(m, dtype=np.int32)
    ders = np.zeros((nders + 1, p + 1, m))
    vp = ctypes.c_void_p
    _lib.check(_lib.LIB.iga_bspline_basis(p, U.shape[0], vp(U.ctypes.data), m, vp(x.ctypes.data),
                                          int(nders), vp(span.ctypes.data), vp(ders.ctypes.data)))
    return span.astype(np.int64), ders


def eval_basis_sparse(degree: int, knotvector: np.ndarray, x: np.ndarray,
                      nders: int = 1) -> List[sp.csr_array]:
    """CSR (len(x), n) matrices of the basis and its derivatives at x
    (same layout as src/igaops/quadrature/utils/operations.py:53-105)."""
    U = np.asarray(knotvector, dtype=float)
    n = len(U) - degree - 1
    x = np.asarray(x, dtype=float)
    span, ders = basis_ders(degree, U, x, nders)
    m = x.shape[0]
    rows = np.repeat(np.arange(m), degree + 1)
    cols = (span[:, None] - degree + np.arange(degree + 1)[None, :]).reshape(-1)
    out = []
    for k in range(nders + 1):
        vals = ders[k].T.reshape(-1)
        b = sp.coo_array((vals, (rows, cols)), shape=(m, n))
        b.eliminate_zeros()
        out.append(sp.csr_array(b))
    return out


def find_multiplicity(knot: float, knotvector: np.ndarray, tol: float = 1e-7) -> int:
    return int(np.sum(np.abs(np.asarray(knotvector) - knot) <= tol))


def increase_multiplicity(repeat: int, degree: int, knotvector: np.ndarray) -> np.ndarray:
    """Raise the multiplicity of every interior knot by `repeat`."""
    kv = np.asarray(knotvector, dtype=float)
    uniq = np.unique(kv)
    out = []
    for i, knot in enumerate(uniq):
        r = 0 if i in (0, len(uniq) - 1) else repeat
        m = find_multiplicity(knot, kv) + r
        if m > degree + 1:
            raise Warning("Introduces numerical instability.")
        out.extend([knot] * m)
    return np.sort(np.asarray(out))


# ================================================================ base
class _Rule1D:
    def __init__(self, degree: int, knotvector: np.ndarray):
        self._degree = int(degree)
        self._knotvector = np.asarray(knotvector).astype(float)
        self._parametric_space = (0.0, 1.0)
        self._unique_kv = np.unique(np.clip(self._knotvector, 0.0, 1.0))
        self._nbctrlpts = len(self._knotvector) - self._degree - 1
        self._quadpts = np.array([])
        self._basis: List[sp.csr_array] = []
        self._weights: List[sp.csr_array] = []

    degree = property(lambda self: self._degree)
    knotvector = property(lambda self: self._knotvector)
    parametric_space = property(lambda self: self._parametric_space)
    unique_kv = property(lambda self: self._unique_kv)
    nbctrlpts = property(lambda self: self._nbctrlpts)
    quadpts = property(lambda self: self._quadpts)
    basis = property(lambda self: self._basis)
    weights = property(lambda self: self._weights)

    @property
    def nbquadpts(self) -> int:
        return len(self._quadpts)

    @property
    def max_h_size(self) -> float:
        return float(np.max(np.abs(np.diff(self._unique_kv))))

    def eval_minimal_continuity(self) -> int:
        cont = self._degree - 1
        for knot in self._unique_kv[1:-1]:
            cont = min(cont, self._degree - find_multiplicity(knot, self._knotvector))
        return cont

    def eval_basis(self, knots_to_interp: np.ndarray, nders: int = 1):
        return eval_basis_sparse(self._degree, self._knotvector, knots_to_interp, nders)


# =============================================================== Gauss
def lobatto(n: int) -> Tuple[np.ndarray, np.ndarray]:
    """Gauss-Lobatto nodes/weights on [-1, 1]: endpoints plus the roots of
    P'_{n-1}; weights 2 / (n (n-1) P_{n-1}(x)^2)."""
    if n < 2:
        raise ValueError("n must be >= 2")
    if n == 2:
        return np.array([-1.0, 1.0]), np.array([1.0, 1.0])
    P = np.polynomial.legendre.Legendre.basis(n - 1)
    inner = np.sort(np.real(P.deriv().roots()))
    x = np.concatenate([[-1.0], inner, [1.0]])
    w = 2.0 / (n * (n - 1) * P(x) ** 2)
    w[0] = w[-1] = 2.0 / (n * (n - 1))
    return x, w


class StandardGauss(_Rule1D):
    """Element-wise Gauss-Legendre or Gauss-Lobatto rule on the knot spans."""

    def __init__(self, degree: int, knotvector: np.ndarray,
                 quadtype: Literal["legendre", "lobatto"], nbptsperel: Optional[int] = None,
                 nders: Optional[int] = None):
        super().__init__(degree, knotvector)
        self._quadrature_type = validate_entry(quadtype, ["legendre", "lobatto"])
        self._nders = int(nders) if nders is not None else 1
        default = self._degree + (1 if self._quadrature_type == "legendre" else 2)
        npts = int(nbptsperel) if nbptsperel is not None else default
        if self._quadrature_type == "legendre":
            self._iso_x, self._iso_w = np.polynomial.legendre.leggauss(npts)
        else:
            self._iso_x, self._iso_w = lobatto(npts)
        self._quadpts, self._parametric_weights = self.interpolate_points_and_weights(
            self._unique_kv)
        basis = self.eval_basis(self._quadpts, nders=self._nders)
        weights = []
        for b in basis:
            w = sp.csr_array(b.T @ sp.diags(self._parametric_weights))
            weights.extend([w, w])
        self._basis = basis
        self._weights = weights

    quadrature_class = property(lambda self: "GAUSS")
    quadrature_type = property(lambda self: self._quadrature_type)
    parametric_weights = property(lambda self: self._parametric_weights)
    nbptsperel = property(lambda self: len(self._iso_x))

    def interpolate_points_and_weights(self, knots: np.ndarray):
        k = np.unique(knots)
        a, b = k[:-1, None], k[1:, None]
        pts = (0.5 * ((b - a) * self._iso_x[None, :] + a + b)).reshape(-1)
        wts = (0.5 * (b - a) * self._iso_w[None, :]).reshape(-1)
        return pts, wts


# ============================================== weighted quadrature
def _element_ranges(U: np.ndarray, degree: int, breaks: np.ndarray) -> np.ndarray:
    """(first, last) element index covered with positive measure by each
    B-spline of (degree, U)."""
    n = len(U) - degree - 1
    a = U[:n, None]
    b = U[degree + 1: degree + 1 + n, None]
    lo = np.maximum(a, breaks[None, :-1])
    hi = np.minimum(b, breaks[None, 1:])
    cover = hi > lo
    first = np.argmax(cover, axis=1)
    last = cover.shape[1] - 1 - np.argmax(cover[:, ::-1], axis=1)
    return np.stack([first, last], axis=1)


def _target_space(degree: int, U: np.ndarray, quadtype: str):
    if quadtype == "1":
        return degree - 1, U[1:-1]
    if quadtype == "2":
        return degree, increase_multiplicity(1, degree, U)
    raise ValueError("Unknown method for weighted quadrature.")


def wq_points_per_element(degree: int, knotvector: np.ndarray, quadtype: str) -> np.ndarray:
    """Number of WQ points per element from the exactness constraints
    (src/igaops/quadrature/utils/wq_helpers.py:11-82,221-259).

    For every (test, target) pair the shared element interval (r, s) is
    counted; for each test function the points needed on elements r..s is
    the number of pairs whose interval lies inside [r, s]; the lower bound
    per element is the maximum over test functions (plus one for
    stability, as the reference does), raised by an integer program only if
    a multi-element constraint is violated.  The tables and the check run in
    the library's host code (``iga_wq_point_counts``); the integer program,
    which no open knot vector of the tested families reaches, keeps scipy's
    ``milp`` as the reference does.
    """
    import ctypes

    from . import _lib

    U = np.asarray(knotvector, dtype=float)
    breaks = np.unique(U)
    ne = len(breaks) - 1
    pt, Ut = _target_space(degree, U, quadtype)
    test = np.ascontiguousarray(_element_ranges(U, degree, breaks), dtype=np.int32)
    targ = np.ascontiguousarray(_element_ranges(np.asarray(Ut, dtype=float), pt, breaks),
                                dtype=np.int32)
    counts = np.zeros(ne, dtype=np.int32)
    feasible = np.zeros(1, dtype=np.int32)
    vp = ctypes.c_void_p
    _lib.check(_lib.LIB.iga_wq_point_counts(ne, test.shape[0], vp(test.ctypes.data), targ.shape[0],
                                            vp(targ.ctypes.data), vp(counts.ctypes.data),
                                            vp(feasible.ctypes.data)))
    if feasible[0]:
        return counts.astype(int)
    return _points_by_integer_program(ne, test, targ)


def _point_tables(ne: int, test: np.ndarray, targ: np.ndarray):
    """S4(r, s) = max over test functions of the pairs inside [r, s], and
    the per-element lower bound (numpy form of the native tables)."""
    r = np.maximum(test[:, None, 0], targ[None, :, 0])
    s = np.minimum(test[:, None, 1], targ[None, :, 1])
    ok = r <= s
    ti = np.nonzero(ok)
    mu = np.zeros((test.shape[0], ne, ne), dtype=np.int64)
    np.add.at(mu, (ti[0], r[ok], s[ok]), 1)
    # mubar_i(r, s) = sum_{r <= k <= l <= s} mu_i(k, l): suffix sum over k,
    # prefix sum over l (mu is upper triangular)
    mubar = np.flip(np.cumsum(np.flip(mu, axis=1), axis=1), axis=1).cumsum(axis=2)
    S4 = mubar.max(axis=0)
    return S4, np.diag(S4).copy() + 1


def _points_by_integer_program(ne: int, test: np.ndarray, targ: np.ndarray) -> np.ndarray:
    S4, lb = _point_tables(ne, test, targ)
    csum = np.concatenate([[0], np.cumsum(lb)])
    rr, ss = np.triu_indices(ne, 1)
    need = S4[rr, ss]
    have = csum[ss + 1] - csum[rr]
    if np.all(have >= need):
        return lb.astype(int)
    from scipy.optimize import Bounds, LinearConstraint, milp

    A = np.zeros((len(rr), ne))
    for k, (a0, b0) in enumerate(zip(rr, ss)):
        A[k, a0: b0 + 1] = 1.0
    res = milp(c=np.ones(ne), constraints=LinearConstraint(A, lb=need, ub=np.inf),
               integrality=np.ones(ne), bounds=Bounds(lb=lb.astype(float), ub=np.inf))
    if not res.success:
        raise ValueError(f"Solver failed {res.message}")
    return np.round(res.x).astype(int)


def _endpoint_points(breaks: np.ndarray, n_list: np.ndarray) -> np.ndarray:
    pts = [np.linspace(breaks[e], breaks[e + 1], int(n_list[e]) + 1) for e in range(len(breaks) - 1)]
    return np.sort(np.unique(np.concatenate(pts)))


def _cellcenter_points(breaks: np.ndarray, n_list: np.ndarray) -> np.ndarray:
    pts = []
    for e in range(len(breaks) - 1):
        n = int(n_list[e])
        t = (2.0 * np.arange(1, n + 1) - 1.0) / (2.0 * n)
        pts.append((1.0 - t) * breaks[e] + t * breaks[e + 1])
    return np.sort(np.unique(np.concatenate(pts)))


def _support_lengths(x: np.ndarray, unique_kv: np.ndarray) -> np.ndarray:
    """Length of the cell around each point (midpoints, reflected at the ends)."""
    ext = np.concatenate([[2 * unique_kv[0] - x[0]], x, [2 * unique_kv[-1] - x[-1]]])
    mid = 0.5 * (ext[:-1] + ext[1:])
    return np.diff(mid)


# Row solvers of the weighted-quadrature rules.  "native": the minimum-norm
# solution of every row's exactness system, computed directly in the
# library's host code; it meets the exactness conditions to rounding
# (relative residual ~1e-15).  "lsqr": scipy's LSQR from zero with
# atol = btol = 1e-14, as the reference runs it; up to degree 3 it converges
# to the same solution (rules equal to 1e-12), from degree 4 on the row
# systems are ill-conditioned enough (condition numbers to ~2e6 at degree 5)
# that LSQR stops short of it at a point that depends on the rounding of its
# dot products (constraint residuals up to 4e-8, rules differing from the
# minimum-norm ones by up to 1e-3 relative at degree 5 on 8 elements, 2e-10
# on 32 or more).  "lsqr" reproduces the reference's rules where that
# matters (its golden vectors); "native" is the default.
WQ_SOLVERS = ("native", "lsqr")


def _min_norm_weights(Z: np.ndarray, A: np.ndarray, B: np.ndarray,
                      native: bool = True) -> np.ndarray:
    """Row i: w_i = z_i * v with v the least-squares solution of
    (A diag z_i) v = b_i of the published construction
    (src/igaops/quadrature/utils/operations.py:287-323: scipy lsqr from zero,
    atol = btol = 1e-14).  native=True solves each row directly for its
    minimum-norm solution (``iga_wq_min_norm_rows``, host code in
    libigab200), native=False runs scipy's lsqr as the reference does."""
    if not native:
        from scipy.sparse.linalg import lsqr

        out = np.zeros_like(Z)
        for i in range(Z.shape[0]):
            z = Z[i]
            out[i] = z * lsqr(A * z, B[i], atol=1e-14, btol=1e-14)[0]
        return out
    import ctypes

    from . import _lib

    Z = np.ascontiguousarray(Z, dtype=np.float64)
    A = np.ascontiguousarray(A, dtype=np.float64)
    B = np.ascontiguousarray(B, dtype=np.float64)
    nrows, npts = Z.shape
    nt = A.shape[0]
    out = np.zeros_like(Z)
    dp = ctypes.POINTER(ctypes.c_double)
    _lib.check(_lib.LIB.iga_wq_min_norm_rows(nrows, nt, npts, A.ctypes.data_as(dp),
                                             Z.ctypes.data_as(dp), B.ctypes.data_as(dp), 1e-13,
                                             out.ctypes.data_as(dp)))
    return out


class WeightedQuadrature(_Rule1D):
    """Weighted quadrature of type "1" (4 rules) or "2" (2 rules)."""

    def __init__(self, degree: int, knotvector: np.ndarray, quadtype: Literal["1", "2"],
                 position_rule: Literal["endpoint", "cellcenter"] = "endpoint",
                 eval_nbpts_per_elem: Optional[Callable] = None, *,
                 solver: Literal["native", "lsqr"] = "native"):
        super().__init__(degree, knotvector)
        self._solver = validate_entry(solver, list(WQ_SOLVERS))
        self._quadrature_type = validate_entry(quadtype, ["1", "2"])
        self._position_rule = validate_entry(position_rule, ["endpoint", "cellcenter"])
        self._use_fallback = self._degree <= 1 or len(self._unique_kv) <= 2
        if self._use_fallback:
            logger.warning("Weighted quadrature needs degree >= 2 and more than one element; "
                           "Gauss quadrature is used instead.")
        if self.eval_minimal_continuity() < 0:
            raise RuntimeError("The knotvector is not regular enough.")
        self._npe = eval_nbpts_per_elem if callable(eval_nbpts_per_elem) else wq_points_per_element
        if self._use_fallback:
            g = StandardGauss(self._degree, self._knotvector, quadtype="legendre")
            self._quadpts, self._weights, self._basis = g.quadpts, g.weights, g.basis
            return
        n_list = np.asarray(self._npe(self._degree, self._knotvector, self._quadrature_type))
        if self._position_rule == "endpoint":
            self._quadpts = _endpoint_points(self._unique_kv, n_list)
        else:
            self._quadpts = _cellcenter_points(self._unique_kv, n_list)
        self._build_weights()

    quadrature_class = property(lambda self: "WEIGHTED")
    quadrature_type = property(lambda self: self._quadrature_type)
    position_rule = property(lambda self: self._position_rule)

    def _w0_rules(self, g_test: StandardGauss, x: np.ndarray, B0wq_test, B0wq_target,
                  B0gs_test, B0gs_target):
        """W0-type weights of the space of g_test; returns (basis at x, [rules])."""
        basis = g_test.eval_basis(x, nders=1)
        Z = (basis[0].T @ sp.diags(_support_lengths(x, g_test.unique_kv))).toarray()
        M = g_test.weights[0]

        def rule(A_fn, B_gs):
            integral = sp.csr_array(M @ B_gs).toarray()
            return _min_norm_weights(Z, A_fn, integral, native=self._solver == "native")

        rules = []
        if self._quadrature_type == "1":
            rules.append(rule(B0wq_test, B0gs_test))
        rules.append(rule(B0wq_target, B0gs_target))
        return basis, rules

    def _build_weights(self):
        p, U, x = self._degree, self._knotvector, self._quadpts
        g_test = StandardGauss(p, U, quadtype="legendre")
        pt, Ut = _target_space(p, U, self._quadrature_type)
        g_target = StandardGauss(pt, Ut, quadtype="legendre", nbptsperel=g_test.nbptsperel)
        B0gs_test = g_test.basis[0]
        B0wq_test = g_test.eval_basis(x)[0].T.toarray()
        B0gs_target = g_target.eval_basis(g_test.quadpts)[0]
        B0wq_target = g_target.eval_basis(x)[0].T.toarray()
        basis, rules = self._w0_rules(g_test, x, B0wq_test, B0wq_target, B0gs_test, B0gs_target)
        # derivative-test rules: W0-type weights of S^{p-1} on U[1:-1], combined
        # with the B-spline derivative formula
        g_low = StandardGauss(p - 1, U[1:-1], quadtype="legendre", nbptsperel=g_test.nbptsperel)
        _, low = self._w0_rules(g_low, x, B0wq_test, B0wq_target, B0gs_test, B0gs_target)
        zero = np.zeros((1, x.shape[0]))
        n = len(U) - p - 1
        for Q in low:
            Qp = np.vstack([zero, Q, zero])
            W1 = np.zeros((n, x.shape[0]))
            for i in range(n):
                d1 = U[i + p] - U[i]
                if abs(d1) > 0 and i < Qp.shape[0]:
                    W1[i] += (p / d1) * Qp[i]
                d2 = U[i + p + 1] - U[i + 1]
                if abs(d2) > 0 and i + 1 < Qp.shape[0]:
                    W1[i] -= (p / d2) * Qp[i + 1]
            rules.append(W1)
        order = [0, 1, 2, 3] if self._quadrature_type == "1" else [0, 0, 1, 1]
        weights = []
        for k in order:
            w = sp.csr_array(rules[k])
            w.eliminate_zeros()
            weights.append(w)
        self._basis = basis
        self._weights = weights
