"""CPU tests of the host-side pieces: the 1D rule builders against the
reference's own rules, the Kronecker helpers, the band conversion, and the
C-ABI library (loads, exports every declared symbol; no GPU calls)."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

from igaops_b200 import common, quadrature
from igaops_b200.bands import band_from
from igaops_b200.geometry import GeometryOps
from tests._golden import FixtureRule, load

ROOT = Path(__file__).resolve().parent.parent


def _dense(M):
    return sp.csr_array(M).toarray()


def test_quadrature_builders_match_reference():
    """Rules equal the reference's golden rules.  From degree 4 on the
    reference's rows are LSQR stopping points (the minimum-norm rows of the
    default solver differ from them; see the native-rule tests below), so
    those degrees are built with solver="lsqr", the reference's own row
    solver, which reproduces them."""
    d = load("quadrature")
    for i, name in enumerate(d["names"]):
        kind, p, ne, rule = str(name).split(":")
        p, ne = int(p), int(ne)
        ref = FixtureRule(d, f"r{i}")
        kv = GeometryOps.make_open_knotvector(p, ne)
        assert np.allclose(kv, ref.knotvector, rtol=0, atol=0)
        if kind in ("gauss", "lobatto"):
            q = quadrature.StandardGauss(p, kv, "legendre" if kind == "gauss" else "lobatto")
        else:
            q = quadrature.WeightedQuadrature(p, kv, kind[-1], rule,
                                              solver="lsqr" if p >= 4 else "native")
        assert np.allclose(q.quadpts, ref.quadpts, rtol=0, atol=1e-14), name
        for a, b in zip(q.basis, ref.basis):
            assert np.abs(_dense(a) - _dense(b)).max() <= 1e-13 * max(1, np.abs(_dense(b)).max())
        for a, b in zip(q.weights, ref.weights):
            scale = max(1e-300, np.abs(_dense(b)).max())
            assert np.abs(_dense(a) - _dense(b)).max() / scale < 1e-11, name


def test_wq_rule_errors():
    kv = GeometryOps.make_open_knotvector(3, 4)
    with pytest.raises(ValueError):
        quadrature.WeightedQuadrature(3, kv, "3")
    with pytest.raises(ValueError):
        quadrature.WeightedQuadrature(3, kv, "2", "middle")
    bad = np.array([0, 0, 0, 0, 0.5, 0.5, 0.5, 0.5, 0.5, 1, 1, 1, 1.0])
    with pytest.raises(RuntimeError):
        quadrature.WeightedQuadrature(3, bad, "2")


def test_basis_partition_of_unity_and_derivative_sum():
    kv = np.array([0, 0, 0, 0.2, 0.45, 0.7, 1, 1, 1.0])
    x = np.linspace(0, 1, 41)
    B = quadrature.eval_basis_sparse(2, kv, x, nders=2)
    assert np.allclose(_dense(B[0]).sum(1), 1.0, atol=1e-14)
    assert np.allclose(_dense(B[1]).sum(1), 0.0, atol=1e-12)
    assert np.allclose(_dense(B[2]).sum(1), 0.0, atol=1e-10)
    # finite-difference check of the first derivative away from knots
    h = 1e-6
    xm = np.array([0.1, 0.33, 0.6, 0.9])
    Bp = _dense(quadrature.eval_basis_sparse(2, kv, xm + h)[0])
    Bm = _dense(quadrature.eval_basis_sparse(2, kv, xm - h)[0])
    D = _dense(quadrature.eval_basis_sparse(2, kv, xm)[1])
    assert np.allclose((Bp - Bm) / (2 * h), D, atol=1e-6)


def test_kron_helpers_match_reference():
    d = load("fastdiag")
    got = common.KronProduct.kron_nonzero_indices([[0, 2], [1, 3], [0, 1]], [4, 4, 3])
    assert np.array_equal(got, d["kron_idx"])
    ref = np.nonzero(np.kron(np.kron([1, 0, 1, 0], [0, 1, 0, 1]), [1, 1, 0]))[0]
    assert np.array_equal(got, ref)
    comb = common.combine_arrays([np.array([1.0, 2.0]), np.array([3.0, 4.0, 5.0])], np.array([2.0, 0.5]))
    assert np.allclose(comb, d["comb"])
    assert isinstance(got, list)
    arr = common.KronProduct.kron_nonzero_array([[0, 2], [1, 3], [0, 1]], [4, 4, 3])
    assert arr.dtype == np.int64 and np.array_equal(arr, got)


@pytest.mark.parametrize("sizes", [(7,), (5, 9), (4, 6, 3), (33, 2, 17)])
def test_kron_sum_equals_kronecker_products_bitwise(sizes):
    """combine_arrays without b-vectors (the FD eigenvalue Kronecker sum)
    broadcasts instead of forming Kronecker products: same values, bit for
    bit, as sum_i c_i (1 x .. x a_i x .. x 1) built with np.kron."""
    rng = np.random.default_rng(len(sizes))
    arr = [rng.uniform(0.1, 10.0, n) for n in sizes]
    coefs = rng.uniform(0.5, 2.0, len(sizes))
    ref = None
    for i in range(len(sizes)):
        parts = [np.ones(n) for n in sizes]
        parts[i] = arr[i] * coefs[i]
        term = parts[0]
        for v in parts[1:]:
            term = np.kron(v, term)
        ref = term if ref is None else ref + term
    got = common.combine_arrays(arr, coefs)
    assert got.shape == ref.shape and np.array_equal(got, ref)


def test_validate_entry():
    assert common.validate_entry("a", ["a", "b"]) == "a"
    with pytest.raises(TypeError):
        common.validate_entry(1, ["a"])
    with pytest.raises(ValueError):
        common.validate_entry("c", ["a"])


def test_band_roundtrip():
    rng = np.random.default_rng(0)
    kv = GeometryOps.make_open_knotvector(3, 7)
    q = quadrature.WeightedQuadrature(3, kv, "2")
    for mats in ([q.basis[0], q.basis[1]], [q.weights[0], q.weights[2]],
                 [sp.csr_array(q.weights[0]).T, sp.csr_array(q.weights[2]).T]):
        start, vals, w, mono = band_from(mats)
        assert mono
        for M, V in zip(mats, vals):
            D = np.zeros(M.shape)
            for r in range(M.shape[0]):
                for t in range(w):
                    c = start[r] + t
                    if c < M.shape[1]:
                        D[r, c] = V[r, t]
            assert np.array_equal(D, _dense(M))
    start, vals, w, _ = band_from([q.basis[0]], width=7)
    assert w == 7 and vals[0].shape[1] == 7


def _declared_functions():
    text = (ROOT / "include" / "igab200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"typedef[^;]*;", "", text)  # function-pointer types are not entry points
    return sorted(set(re.findall(r"\b(iga_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from igaops_b200 import _lib

    lib = ctypes.CDLL(_lib.library_path())
    declared = _declared_functions()
    assert declared, "no declarations parsed"
    for name in declared:
        assert hasattr(lib, name), name
    assert set(_lib.exported_symbols()) >= set(declared) - {"iga_last_error"} | {"iga_last_error"}
    assert lib.iga_abi_version() == 1


def test_library_rejects_bad_arguments_without_gpu():
    """Argument validation runs on the host and returns INVALID_ARG."""
    from igaops_b200 import _lib

    rc = _lib.LIB.iga_lmode_apply(0, 0, None, 1, None, None, None, None, None)
    assert rc == _lib.IGA_ERR_INVALID_ARG
    assert b"ndim" in _lib.LIB.iga_last_error()
    rc = _lib.LIB.iga_mf_matvec(None, 0, None, 1, None, None, None)
    assert rc == _lib.IGA_ERR_INVALID_ARG
    with pytest.raises(ValueError):
        _lib.check(_lib.IGA_ERR_INVALID_ARG)


def test_product_has_no_oracle_import():
    for f in (ROOT / "igaops_b200").rglob("*.py"):
        src = f.read_text()
        assert "import oracle" not in src and "from oracle" not in src, f


@pytest.mark.parametrize("p,ne,kind", [(2, 7, "2"), (3, 9, "2"), (3, 6, "1"), (2, 5, "1"),
                                       (4, 8, "2"), (4, 6, "1")])
def test_native_wq_rows_equal_lsqr_rows(p, ne, kind):
    """The native row solver (iga_wq_min_norm_rows, host code of the
    library) gives the rules of the reference's LSQR construction wherever
    LSQR converges (degrees <= 4)."""
    kv = GeometryOps.make_open_knotvector(p, ne)
    qn = quadrature.WeightedQuadrature(p, kv, kind)
    ql = quadrature.WeightedQuadrature(p, kv, kind, solver="lsqr")
    tol = 1e-12 if p <= 3 else 1e-10
    for a, b in zip(qn.weights, ql.weights):
        scale = np.abs(_dense(b)).max()
        assert np.abs(_dense(a) - _dense(b)).max() <= tol * scale


def _exactness(q, p, kv):
    """Largest relative error of the rule's products (test function or its
    derivative against trial function or its derivative) against Gauss
    integration, which is exact for these polynomial products."""
    g = quadrature.StandardGauss(p, kv, "legendre")
    err = 0.0
    for b, wk in ((0, 0), (1, 1), (0, 2), (1, 3)):
        A = _dense(q.weights[wk]) @ _dense(q.basis[b])
        E = _dense(g.weights[wk]) @ _dense(g.basis[b])
        err = max(err, np.abs(A - E).max() / np.abs(E).max())
    return err


def test_native_rules_meet_exactness_where_lsqr_stops_short():
    """At degrees 4 and 5 the reference's rules are LSQR stopping points:
    its golden rules integrate the products they are built for only to
    1e-7 .. 1e-13.  The native minimum-norm rules meet them to rounding,
    and differ from the golden rules by less than 1e-3 relative (by 2e-4
    at most, on degree 5, 6 elements, cell-centred points)."""
    d = load("quadrature")
    seen = 0
    for i, name in enumerate(d["names"]):
        kind, p, ne, rule = str(name).split(":")
        p, ne = int(p), int(ne)
        if not kind.startswith("wq") or p < 4:
            continue
        ref = FixtureRule(d, f"r{i}")
        kv = GeometryOps.make_open_knotvector(p, ne)
        q = quadrature.WeightedQuadrature(p, kv, kind[-1], rule)
        assert np.allclose(q.quadpts, ref.quadpts, rtol=0, atol=1e-14), name
        e_native, e_ref = _exactness(q, p, kv), _exactness(ref, p, kv)
        assert e_native < 1e-14 and e_native <= e_ref, (name, e_native, e_ref)
        for a, b in zip(q.weights, ref.weights):
            assert np.abs(_dense(a) - _dense(b)).max() < 1e-3 * np.abs(_dense(b)).max(), name
        seen += 1
    assert seen == 8


@pytest.mark.parametrize("p,ne,kind,rule", [(5, 6, "2", "cellcenter"), (5, 6, "1", "cellcenter"),
                                            (5, 8, "2", "endpoint"), (4, 5, "2", "endpoint")])
def test_native_rules_leave_discrete_solutions_unchanged(p, ne, kind, rule):
    """-(c u')' + u = f on (0, 1), u(0) = u(1) = 0, c = 1 + sin(3x) / 2,
    discretised with the rule's weights: the native and the LSQR rule give
    solutions whose difference is at least 10x below the rule's own
    quadrature error (against the solution with exactly integrated
    matrices), and the native rule's error is no larger than the LSQR
    rule's (within 1 %; on degree 5, 8 elements it is 2 % smaller)."""
    kv = GeometryOps.make_open_knotvector(p, ne)

    def solve(q):
        x = q.quadpts
        B0, B1 = _dense(q.basis[0]), _dense(q.basis[1])
        W0, W3 = _dense(q.weights[0]), _dense(q.weights[3])
        K = W3 @ ((1.0 + 0.5 * np.sin(3.0 * x))[:, None] * B1) + W0 @ B0
        b = W0 @ (np.exp(x) * np.cos(2.0 * x))
        fr = np.arange(1, K.shape[0] - 1)
        u = np.zeros(K.shape[0])
        u[fr] = np.linalg.solve(K[np.ix_(fr, fr)], b[fr])
        return u

    un = solve(quadrature.WeightedQuadrature(p, kv, kind, rule))
    ul = solve(quadrature.WeightedQuadrature(p, kv, kind, rule, solver="lsqr"))
    ue = solve(quadrature.StandardGauss(p, kv, "legendre", nbptsperel=p + 12))
    err_l = np.linalg.norm(ul - ue) / np.linalg.norm(ue)
    err_n = np.linalg.norm(un - ue) / np.linalg.norm(ue)
    assert np.linalg.norm(un - ul) / np.linalg.norm(ul) < 0.1 * err_l
    assert err_n <= 1.01 * err_l


def _knot_families():
    rng = np.random.default_rng(0)
    for p in range(1, 7):
        for ne in (2, 3, 5, 8, 16, 33):
            for shape in ("uniform", "random", "graded"):
                if shape == "uniform":
                    br = np.linspace(0, 1, ne + 1)
                elif shape == "random":
                    br = np.sort(np.concatenate([[0, 1], rng.uniform(0, 1, ne - 1)]))
                else:
                    br = np.linspace(0, 1, ne + 1) ** 2
                yield p, np.concatenate([np.zeros(p), br, np.ones(p)])
    for p in range(2, 6):
        for mult in range(2, p + 1):
            br = np.linspace(0, 1, 9)
            yield p, np.concatenate([np.zeros(p + 1), np.repeat(br[1:-1], mult), np.ones(p + 1)])


def test_native_point_counts_equal_tables():
    """iga_wq_point_counts == the full (test x element x element) tables of
    the point layout and their range check, over uniform, random, graded
    and repeated-knot vectors of degrees 1..6 and both rule types."""
    n = 0
    for p, U in _knot_families():
        for qt in ("1", "2"):
            breaks = np.unique(U)
            ne = len(breaks) - 1
            pt, Ut = quadrature._target_space(p, U, qt)
            test = quadrature._element_ranges(U, p, breaks)
            targ = quadrature._element_ranges(np.asarray(Ut, float), pt, breaks)
            S4, lb = quadrature._point_tables(ne, test, targ)
            got = quadrature.wq_points_per_element(p, U, qt)
            assert np.array_equal(got, lb), (p, qt)
            n += 1
    assert n > 200


def test_native_point_counts_flag_infeasible_ranges():
    """Pairs whose shared intervals all span several elements leave the
    per-element bound short of a multi-element range: the native check
    flags it and the integer program raises the counts."""
    from igaops_b200 import _lib

    ne = 3
    test = np.array([[0, 2]], dtype=np.int32)
    targ = np.array([[0, 2]] * 5 + [[0, 1], [1, 2]], dtype=np.int32)
    counts = np.zeros(ne, dtype=np.int32)
    feasible = np.ones(1, dtype=np.int32)
    vp = ctypes.c_void_p
    assert _lib.LIB.iga_wq_point_counts(ne, 1, vp(test.ctypes.data), len(targ), vp(targ.ctypes.data),
                                        vp(counts.ctypes.data), vp(feasible.ctypes.data)) == 0
    S4, lb = quadrature._point_tables(ne, test, targ)
    assert np.array_equal(counts, lb) and feasible[0] == 0
    raised = quadrature._points_by_integer_program(ne, test, targ)
    assert raised.sum() >= S4[0, 2] and np.all(raised >= lb)
    bad = np.array([[0, 3]], dtype=np.int32)
    assert _lib.LIB.iga_wq_point_counts(ne, 1, vp(bad.ctypes.data), len(targ), vp(targ.ctypes.data),
                                        vp(counts.ctypes.data),
                                        vp(feasible.ctypes.data)) == _lib.IGA_ERR_INVALID_ARG


def test_native_wq_rows_edge_cases():
    """Rows with no active point or a zero right-hand side give zero weights;
    a consistent square system is solved exactly."""
    A = np.array([[1.0, 2.0, 0.0], [0.0, 1.0, 3.0]])
    Z = np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0], [1.0, 0.0, 1.0]])
    B = np.array([[1.0, 1.0], [0.0, 0.0], [2.0, 6.0]])
    W = quadrature._min_norm_weights(Z, A, B)
    assert np.all(W[0] == 0.0) and np.all(W[1] == 0.0)
    assert np.allclose(A @ W[2], B[2], atol=1e-14)
    ref = quadrature._min_norm_weights(Z, A, B, native=False)
    assert np.allclose(W, ref, atol=1e-13)


def test_fd_pencil_cache_is_exact():
    """The FD setup keeps the 1D Gauss pencils and eigenpairs per spline
    across builds (a serving loop builds one preconditioner per request):
    a cached build equals an uncached one bit for bit, for every Dirichlet
    pattern, and callers get private copies."""
    import igaops_b200.fastdiag as F

    q3 = quadrature.WeightedQuadrature(3, GeometryOps.make_open_knotvector(3, 12), "2")
    q2 = quadrature.WeightedQuadrature(2, GeometryOps.make_open_knotvector(2, 7), "2")
    tables = [np.ones((1, 3, 2), bool), np.array([[[True, False], [False, True], [False, False]]])]
    saved = F._PENCIL_CACHE_MAX
    try:
        for table in tables:
            F._PENCIL_CACHE, F._PENCIL_CACHE_MAX = None, 0  # every entry evicted at once
            ref = F.SingleFD("spatial")
            ref.compute_space_eigendecomposition([q3, q2, q3], table)
            F._PENCIL_CACHE_MAX = saved
            for _ in range(2):  # fill, then hit
                fd = F.SingleFD("spatial")
                fd.compute_space_eigendecomposition([q3, q2, q3], table)
                a, b = ref.space_preconditioner, fd.space_preconditioner
                for va, vb in zip(a._eigenvec_by_dir_space[0], b._eigenvec_by_dir_space[0]):
                    assert np.array_equal(va, vb)
                for wa, wb in zip(a._eigenval_by_dir_space[0], b._eigenval_by_dir_space[0]):
                    assert np.array_equal(wa, wb)
                assert np.array_equal(a.free_nodes(0), b.free_nodes(0))
                assert a.space_free_nodes[0] == b.space_free_nodes[0]
            # private copies: writing into one build leaves the cache intact
            fd.space_preconditioner._eigenvec_by_dir_space[0][0][:] = 0.0
            fd2 = F.SingleFD("spatial")
            fd2.compute_space_eigendecomposition([q3, q2, q3], table)
            assert np.array_equal(fd2.space_preconditioner._eigenvec_by_dir_space[0][0],
                                  ref.space_preconditioner._eigenvec_by_dir_space[0][0])
    finally:
        F._PENCIL_CACHE_MAX = saved


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5, 6])
def test_native_basis_matches_piegl_tiller_helpers(p):
    """iga_bspline_basis (host code of the library) == the oracle's scalar
    restatement of geomdl's span search and basis derivatives (Piegl &
    Tiller A2.1 / A2.3) on random, graded and repeated-knot vectors, at
    interior points, knots, and both ends of the domain."""
    import sys

    sys.path.insert(0, str(ROOT / "oracle" / "geomdl_shim"))
    from geomdl import helpers as H

    rng = np.random.default_rng(p)
    br = np.sort(np.concatenate([[0.0, 1.0], rng.uniform(0, 1, 6)]))
    kvs = [np.concatenate([np.zeros(p + 1), br[1:-1], np.ones(p + 1)]),
           np.concatenate([np.zeros(p + 1), np.repeat(br[2:4], min(2, p)), np.ones(p + 1)])]
    for U in kvs:
        x = np.concatenate([rng.uniform(0, 1, 40), np.unique(U), [0.0, 1.0]])
        span, ders = quadrature.basis_ders(p, U, x, nders=min(p, 3))
        n = len(U) - p - 1
        for i, xi in enumerate(x):
            s = H.find_span_linear(p, list(U), n, xi)
            assert span[i] == s
            ref = np.asarray(H.basis_function_ders(p, list(U), s, xi, min(p, 3)))
            scale = np.abs(ref).max(axis=1, keepdims=True) + 1.0
            assert np.all(np.abs(ders[:, :, i] - ref) <= 1e-13 * scale), (p, xi)


@pytest.mark.parametrize("dims", [2, 3])
def test_dirichlet_nodes_are_the_complement_of_the_free_box(dims):
    """SpaceFD.dirichlet_nodes (built from the box's faces) == the sorted
    complement of the free nodes, for every Dirichlet pattern of the
    directions (none, one side, both sides) and uneven extents."""
    import itertools

    import igaops_b200.fastdiag as F

    rl = [quadrature.WeightedQuadrature(p, GeometryOps.make_open_knotvector(p, ne), "2")
          for p, ne in zip((2, 3, 2), (5, 4, 6))][:dims]
    N = int(np.prod([q.nbctrlpts for q in rl]))
    for flags in itertools.product([False, True], repeat=2 * dims):
        table = np.array(flags, dtype=bool).reshape(1, dims, 2)
        fd = F.SingleFD("spatial")
        fd.compute_space_eigendecomposition(rl, table)
        sp = fd.space_preconditioner
        mask = np.ones(N, dtype=bool)
        mask[sp.free_nodes(0)] = False
        got = sp.dirichlet_nodes(0)
        assert got.dtype == np.int64 and np.array_equal(got, np.flatnonzero(mask)), flags


def test_refined_solver_residual_modes():
    """The refined solvers take residual "true" (default: convergence
    confirmed by b - A x) or "arnoldi" (the reference GMRES's stopping rule)
    and refuse anything else before touching a device."""
    import igaops_b200.batch as batch
    from igaops_b200.refine import MixedPrecisionFGMRES, RefinedOutput

    assert batch.RESIDUAL_KINDS == ("true", "arnoldi")
    assert MixedPrecisionFGMRES().residual == "true"
    assert MixedPrecisionFGMRES(residual="arnoldi").residual == "arnoldi"
    with pytest.raises(ValueError):
        MixedPrecisionFGMRES(residual="estimate")
    assert RefinedOutput(solution=None, residual=np.ones(1), success=False).residual_kind == "true"
    assert batch.BatchResult(solution=None, success=np.ones(1, bool),
                             true_residual=np.ones(1)).residual_kind == "true"
