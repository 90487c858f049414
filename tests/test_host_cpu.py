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
            q = quadrature.WeightedQuadrature(p, kv, kind[-1], rule)
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


@pytest.mark.parametrize("p,ne,kind", [(2, 7, "2"), (3, 9, "2"), (3, 6, "1"), (2, 5, "1")])
def test_native_wq_rows_equal_lsqr_rows(p, ne, kind):
    """The native row solver (iga_wq_min_norm_rows, host code of the
    library) gives the rules of the reference's LSQR construction."""
    kv = GeometryOps.make_open_knotvector(p, ne)
    saved = quadrature.NATIVE_WQ_MAX_DEGREE
    try:
        quadrature.NATIVE_WQ_MAX_DEGREE = 5
        qn = quadrature.WeightedQuadrature(p, kv, kind)
        quadrature.NATIVE_WQ_MAX_DEGREE = 0
        ql = quadrature.WeightedQuadrature(p, kv, kind)
    finally:
        quadrature.NATIVE_WQ_MAX_DEGREE = saved
    for a, b in zip(qn.weights, ql.weights):
        scale = np.abs(_dense(b)).max()
        assert np.abs(_dense(a) - _dense(b)).max() <= 1e-12 * scale


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
                assert a._space_free_nodes[0] == b._space_free_nodes[0]
            # private copies: writing into one build leaves the cache intact
            fd.space_preconditioner._eigenvec_by_dir_space[0][0][:] = 0.0
            fd2 = F.SingleFD("spatial")
            fd2.compute_space_eigendecomposition([q3, q2, q3], table)
            assert np.array_equal(fd2.space_preconditioner._eigenvec_by_dir_space[0][0],
                                  ref.space_preconditioner._eigenvec_by_dir_space[0][0])
    finally:
        F._PENCIL_CACHE_MAX = saved
