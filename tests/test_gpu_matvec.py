"""GPU parity of the L-mode product and the matrix-free operators against
the numpy oracle (oracle/mf.py) on identical seeded inputs.

Tolerances (relative max-norm): FP64 1e-12, FP32 1e-5.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

from oracle import mf as omf
from tests._problems import coefficients, rel_err, rules

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 1e-5


@pytest.fixture(scope="module")
def ops():
    from igaops_b200 import BsplineOperations, MatrixFree, MFOperator

    return BsplineOperations, MatrixFree, MFOperator


# --------------------------------------------------------------- L-mode
@pytest.mark.parametrize("ndim", [1, 2, 3, 4])
@pytest.mark.parametrize("transpose", [False, True])
@pytest.mark.parametrize("ncols", [0, 3])
def test_lmode_sparse_and_dense(cuda, ops, ndim, transpose, ncols):
    _, MatrixFree, _ = ops
    rng = np.random.default_rng(ndim)
    rl = rules(ndim, [2, 3, 2, 3][:ndim], [3, 4, 5, 2][:ndim], kind="gauss")
    sparse = [q.basis[1] for q in rl]
    dense = [rng.standard_normal((3 + k, 4 + k)) for k in range(ndim)]
    for mats in (sparse, dense):
        n = int(np.prod([m.shape[0 if transpose else 1] for m in mats]))
        x = rng.standard_normal((n, ncols) if ncols else n)
        ref = omf.lmode_apply(mats, x, transpose)
        got = MatrixFree.apply(mats, x, is_transpose=transpose)
        assert got.shape == ref.shape
        assert rel_err(got, ref) < TOL64


def test_tensor_matrix_product(cuda, ops):
    _, MatrixFree, _ = ops
    rng = np.random.default_rng(1)
    t = rng.standard_normal((4, 5, 6))
    M = rng.standard_normal((7, 5))
    ref = omf.mode_product(t, M, 1)
    got = MatrixFree.tensor_matrix_product(t, M, mode=1)
    assert rel_err(got, ref) < TOL64
    got_t = MatrixFree.tensor_matrix_product(t, sp.csr_array(M.T), mode=1, is_transpose=True)
    assert rel_err(got_t, ref) < TOL64


# ------------------------------------------------------ fused operators
# (p, 1): one element per direction (Gauss rules stand in for weighted
# quadrature there), the fewest points and control points a tile can hold
CASES_3D = [(2, 5), (3, 7), (4, 4), (5, 3), (3, 20), (2, 1), (5, 1)]
CASES_2D = [(2, 9), (3, 6), (3, 64), (5, 5), (2, 1)]


def _check(ops, rl, op, x, coefs, time_ders=None, dtype=torch.float64, tol=TOL64,
           expect_fused=True):
    BsplineOperations, _, MFOperator = ops
    ref = omf.OPS[op](rl, coefs, x, time_ders)
    oper = MFOperator(rl, coefs, op, time_ders=time_ders, dtype=dtype)
    assert oper.fused == expect_fused
    if dtype == torch.float64:
        got = getattr(BsplineOperations, f"compute_mf_scalar_{op}")(rl, coefs, x, time_ders)
        assert rel_err(got, ref) < tol, rel_err(got, ref)
    xd = torch.from_numpy(x).to("cuda", dtype)
    got = oper.apply(xd).double().cpu().numpy()
    err = rel_err(got, ref)
    assert err < tol, err
    return err


@pytest.mark.parametrize("p,ne", CASES_3D)
@pytest.mark.parametrize("op", ["u_v", "gradu_gradv", "gradu_v", "u_gradv"])
def test_fused_3d(cuda, ops, p, ne, op):
    rl = rules(3, p, ne)
    rng = np.random.default_rng(p * 100 + ne)
    N = int(np.prod([q.nbctrlpts for q in rl]))
    x = rng.standard_normal(N)
    c = coefficients(op, rl, rng)
    _check(ops, rl, op, x, c)
    _check(ops, rl, op, x, c, dtype=torch.float32, tol=TOL32)


@pytest.mark.parametrize("p,ne", CASES_2D)
@pytest.mark.parametrize("op", ["u_v", "gradu_gradv", "gradu_v", "u_gradv"])
def test_fused_2d(cuda, ops, p, ne, op):
    rl = rules(2, p, ne)
    rng = np.random.default_rng(p * 10 + ne)
    N = int(np.prod([q.nbctrlpts for q in rl]))
    x = rng.standard_normal(N)
    c = coefficients(op, rl, rng)
    _check(ops, rl, op, x, c)
    _check(ops, rl, op, x, c, dtype=torch.float32, tol=TOL32)


def test_fused_nonsymmetric_and_multicol(cuda, ops):
    rl = rules(3, 3, 6)
    rng = np.random.default_rng(7)
    N = int(np.prod([q.nbctrlpts for q in rl]))
    c = coefficients("gradu_gradv", rl, rng, symmetric=False)
    x = rng.standard_normal((N, 3))
    _check(ops, rl, "gradu_gradv", x, c)


def test_fused_anisotropic_mesh(cuda, ops):
    rl = rules(3, [2, 3, 4], [9, 5, 7])
    rng = np.random.default_rng(11)
    N = int(np.prod([q.nbctrlpts for q in rl]))
    x = rng.standard_normal(N)
    for op in ("u_v", "gradu_gradv"):
        _check(ops, rl, op, x, coefficients(op, rl, rng))


def test_fused_gauss(cuda, ops):
    rl = rules(3, 3, 5, kind="gauss")
    rng = np.random.default_rng(3)
    N = int(np.prod([q.nbctrlpts for q in rl]))
    x = rng.standard_normal(N)
    _check(ops, rl, "gradu_gradv", x, coefficients("gradu_gradv", rl, rng))


@pytest.mark.parametrize("td", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_fused_spacetime_mass(cuda, ops, td):
    rl = rules(3, [3, 3, 2], [6, 5, 4])
    rng = np.random.default_rng(5)
    N = int(np.prod([q.nbctrlpts for q in rl]))
    x = rng.standard_normal(N)
    _check(ops, rl, "u_v", x, coefficients("u_v", rl, rng), time_ders=td)


def test_fused_spacetime_stiffness(cuda, ops):
    rl = rules(3, [3, 3, 2], [6, 5, 4])
    rng = np.random.default_rng(6)
    N = int(np.prod([q.nbctrlpts for q in rl]))
    x = rng.standard_normal(N)
    c = coefficients("gradu_gradv", rl, rng)
    _check(ops, rl, "gradu_gradv", x, c, time_ders=(0, 0))


@pytest.mark.parametrize("op", ["u_v", "gradu_gradv", "gradu_v", "u_gradv"])
def test_generic_path_type1_and_1d(cuda, ops, op):
    rng = np.random.default_rng(9)
    for rl in (rules(3, 3, 4, kind="wq1"), rules(1, 3, 6), rules(2, 2, 5, kind="wq1")):
        N = int(np.prod([q.nbctrlpts for q in rl]))
        x = rng.standard_normal(N)
        _check(ops, rl, op, x, coefficients(op, rl, rng), expect_fused=False)


def test_generic_spacetime_other_ders(cuda, ops):
    rl = rules(3, [3, 3, 2], [6, 5, 4])
    rng = np.random.default_rng(12)
    N = int(np.prod([q.nbctrlpts for q in rl]))
    x = rng.standard_normal(N)
    c = coefficients("gradu_gradv", rl, rng)
    _check(ops, rl, "gradu_gradv", x, c, time_ders=(1, 0), expect_fused=False)


def test_fused_forced_generic_matches(cuda, ops):
    _, _, MFOperator = ops
    rl = rules(3, 3, 8)
    rng = np.random.default_rng(21)
    N = int(np.prod([q.nbctrlpts for q in rl]))
    x = torch.from_numpy(rng.standard_normal(N)).cuda()
    c = coefficients("gradu_gradv", rl, rng)
    a = MFOperator(rl, c, "gradu_gradv").apply(x)
    b = MFOperator(rl, c, "gradu_gradv", force_generic=True).apply(x)
    assert rel_err(a.cpu().numpy(), b.cpu().numpy()) < TOL64


def test_fused_many_segments(cuda, ops):
    """Segment boundaries of the streamed direction (nseg > 1) are exact."""
    _, _, MFOperator = ops
    rl = rules(3, 3, 16)
    rng = np.random.default_rng(4)
    N = int(np.prod([q.nbctrlpts for q in rl]))
    x = rng.standard_normal(N)
    c = coefficients("gradu_gradv", rl, rng)
    ref = omf.mf_gradu_gradv(rl, c, x)
    for nseg in (1, 2, 5, 13):
        oper = MFOperator(rl, c, "gradu_gradv", nseg=nseg)
        assert oper.plan.nseg == nseg
        got = oper.apply(torch.from_numpy(x).cuda()).cpu().numpy()
        assert rel_err(got, ref) < TOL64


def test_autotuned_launch_shape_same_result(cuda):
    """nseg="auto" picks a segment count by timing; the result is the
    same operator (FP64 1e-12) and a second operator of the same shape hits
    the tuner's cache."""
    from igaops_b200 import MFOperator
    from igaops_b200 import tune

    rng = np.random.default_rng(21)
    rl = rules(3, 3, 10)
    c = coefficients("gradu_gradv", rl, rng)
    x = rng.standard_normal(int(np.prod([q.nbctrlpts for q in rl])))
    ref = omf.mf_gradu_gradv(rl, c, x)
    # the pencil kernel's segment count (kernel="auto" may pick the tile kernel)
    op = MFOperator(rl, c, "gradu_gradv", nseg="auto", kernel="pencil")
    assert rel_err(op.apply(x), ref) < TOL64
    key = tune.shape_key(op.plan)
    assert tune._CACHE[key] == op.plan.nseg
    op2 = MFOperator(rl, c, "gradu_gradv", nseg="auto", kernel="pencil")
    assert op2.plan.nseg == op.plan.nseg
    assert rel_err(op2.apply(x), ref) < TOL64
