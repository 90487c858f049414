"""GPU Krylov solvers against the reference's own results (golden fixtures)
and the oracle."""
import numpy as np
import pytest
import torch

from oracle import fd as ofd
from oracle import krylov as okr
from oracle import mf as omf
from tests._golden import FixtureRule, load
from tests._problems import rel_err, rules

pytestmark = pytest.mark.gpu


def _poisson2d(d):
    from igaops_b200 import MFOperator
    from igaops_b200.fastdiag import SingleFD

    q = FixtureRule(d, "gm_rule")
    rl = [q, q]
    free = torch.as_tensor(d["gm_free"], device="cuda")
    N = q.nbctrlpts ** 2
    op = MFOperator(rl, d["gm_coefs"], "gradu_gradv")
    fd = SingleFD("spatial")
    fd.compute_space_eigendecomposition(rl, np.ones((1, 2, 2), dtype=bool))

    def A(x):
        full = torch.zeros(N, dtype=torch.float64, device="cuda")
        full[free] = x
        return op.apply(full)[free]

    def P(x):
        full = torch.zeros(N, dtype=torch.float64, device="cuda")
        full[free] = x
        return fd.apply(full)[free]

    return A, P


def test_gmres_matches_reference_golden(cuda):
    from igaops_b200.solvers import LinearSolver

    d = load("solvers")
    A, P = _poisson2d(d)
    for tol in (1e-6, 1e-10):
        ls = LinearSolver(tol, 100, linear_type="gmres", verbose=False)
        out = ls.solve(A, d["gm_b"], P)
        ref = d[f"gm_res_{tol:g}"]
        assert out.success
        assert len(out.residual) == len(ref)
        assert np.allclose(out.residual, ref, rtol=1e-6, atol=1e-13)
        assert rel_err(out.solution, d[f"gm_x_{tol:g}"]) < 1e-10
        it = ls.convergence_manager.parameters["iteration"].current
        assert it == len(ref) - 1
    ls = LinearSolver(1e-10, 200, linear_type="gmres", verbose=False)
    out = ls.solve(A, d["gm_b"])
    assert len(out.residual) == len(d["gm_res_noprec"])
    assert rel_err(out.solution, d["gm_x_noprec"]) < 1e-8


def test_gmres_mask_and_x0_match_reference(cuda):
    from igaops_b200.solvers import LinearSolver

    d = load("solvers")
    T = torch.as_tensor(d["tri_T"], device="cuda")
    ls = LinearSolver(1e-9, 100, cleandod=[int(i) for i in d["tri_mask"]], linear_type="gmres",
                      verbose=False)
    out = ls.solve(lambda v: T @ v, d["tri_b"], x0=d["tri_x0"])
    assert len(out.residual) == len(d["tri_res"])
    assert rel_err(out.solution, d["tri_x"]) < 1e-10


def test_gcrodr_matches_reference_golden(cuda):
    from igaops_b200.solvers import GCRODR

    d = load("solvers")
    T = torch.as_tensor(d["gc_T"], device="cuda")
    g = GCRODR(tolerance=1e-8, maxiters=2000, krylov_size=30, recycled_size=10, verbose=False)
    o1 = g.solve(lambda v: T @ v, d["gc_rhs"])
    o2 = g.solve(lambda v: T @ v, 0.5 * d["gc_rhs"] + 0.1)
    assert o1.success and o2.success
    assert len(o1.residual) == len(d["gc_res1"]) and len(o2.residual) == len(d["gc_res2"])
    assert rel_err(o1.solution, d["gc_x1"]) < 1e-8
    assert rel_err(o2.solution, d["gc_x2"]) < 1e-8
    # the recycled space is reused: the second solve starts from a warm start
    Tn = d["gc_T"]
    assert np.linalg.norm(Tn @ o2.solution - (0.5 * d["gc_rhs"] + 0.1)) <= 10 * 1e-8 * np.linalg.norm(
        0.5 * d["gc_rhs"] + 0.1) + 1e-8


def test_gcrodr_reference_suite(cuda):
    """The reference's tests/test_gcrodr.py scenario (n=1000, m=60, k=30)."""
    from igaops_b200.solvers import GCRODR, LinearSolver

    n, tol = 1000, 1e-6
    T = np.diag(np.full(n, 2.05)) + np.diag(np.full(n - 1, -1.0), 1) + np.diag(np.full(n - 1, -1.0), -1)
    Td = torch.as_tensor(T, device="cuda")
    x = np.zeros(n)
    x[0] = 1.0
    rhs = np.outer(np.linspace(0, 1, 5)[1:], T @ x)
    A = lambda v: Td @ v  # noqa: E731
    ls = LinearSolver(tolerance=tol, maxiters=500)
    g = GCRODR(tolerance=tol, maxiters=500, krylov_size=60, recycled_size=30)
    xr = ls.solve(A, rhs[0]).solution
    o = g.solve(A, rhs[0])
    assert o.residual.min() <= tol
    assert np.allclose(xr, o.solution, atol=1e-4)
    for i in range(4):
        o = g.solve(A, rhs[i])
        assert np.linalg.norm(rhs[i] - T @ o.solution) <= tol * 10


@pytest.mark.parametrize("kind", ["cg", "bicgstab"])
def test_cg_bicgstab_match_oracle_direct(cuda, kind):
    from igaops_b200.solvers import LinearSolver

    d = load("solvers")
    A, P = _poisson2d(d)
    ls = LinearSolver(1e-11, 200, linear_type=kind, verbose=False)
    out = ls.solve(A, d["gm_b"], P)
    assert out.success
    assert rel_err(out.solution, d["gm_x_1e-10"]) < 1e-8


def test_block_cg(cuda):
    from igaops_b200.solvers import LinearSolver

    d = load("solvers")
    A, P = _poisson2d(d)
    rng = np.random.default_rng(3)
    nfree = len(d["gm_free"])
    Bm = rng.standard_normal((nfree, 3))

    def A2(X):
        return torch.stack([A(X[:, k].contiguous()) for k in range(X.shape[1])], 1)

    def P2(X):
        return torch.stack([P(X[:, k].contiguous()) for k in range(X.shape[1])], 1)

    ls = LinearSolver(1e-11, 200, linear_type="block_cg", verbose=False)
    out = ls.solve(A2, Bm, P2)
    assert out.success
    ls1 = LinearSolver(1e-12, 200, linear_type="gmres", verbose=False)
    for k in range(3):
        xk = ls1.solve(A, Bm[:, k], P).solution
        assert rel_err(out.solution[:, k], xk) < 1e-8


def test_fd_gmres_3d_converges_fast(cuda):
    """The reference's tests/test_fast_diagonalization.py flow: 3D p3 ne4
    Gauss, anisotropic stiffness (3, 2, 5), mixed Dirichlet, FD-GMRES to 1e-9
    in fewer than 5 iterations, matching a direct solve."""
    from igaops_b200 import MFOperator
    from igaops_b200.fastdiag import SingleFD
    from igaops_b200.solvers import LinearSolver

    q = rules(1, 3, 4, kind="gauss")[0]
    rl = [q] * 3
    vals = [3.0, 2.0, 5.0]
    table = np.zeros((1, 3, 2), dtype=bool)
    table[0, 0, 0] = True
    table[0, 2, 1] = True
    fd = SingleFD("spatial")
    fd.compute_space_eigendecomposition(rl, table)
    fd.add_scalar_space_time_correctors(stiffness_corrector=[np.array(vals)])
    fd.update_space_eigenvalues(scalar_coefs=(0, 1))
    free = np.asarray(fd.space_preconditioner.space_free_nodes[0])
    nq = q.nbquadpts ** 3
    C = np.zeros((3, 3, nq))
    for i, v in enumerate(vals):
        C[i, i] = v
    op = MFOperator(rl, C, "gradu_gradv")
    N = q.nbctrlpts ** 3
    fr = torch.as_tensor(free, device="cuda")

    def A(x):
        full = torch.zeros(N, dtype=torch.float64, device="cuda")
        full[fr] = x
        return op.apply(full)[fr]

    def P(x):
        full = torch.zeros(N, dtype=torch.float64, device="cuda")
        full[fr] = x
        return fd.apply(full)[fr]

    b = np.random.default_rng(0).random(len(free))
    ls = LinearSolver(1e-9, 100, linear_type="gmres", verbose=False)
    out = ls.solve(A, b, P)
    assert ls.convergence_manager.parameters["iteration"].current < 5
    # direct solve of the oracle operator
    Kd = np.zeros((len(free), len(free)))
    for j in range(len(free)):
        e = np.zeros(N)
        e[free[j]] = 1.0
        Kd[:, j] = omf.mf_gradu_gradv(rl, C, e)[free]
    xd = np.linalg.solve(Kd, b)
    assert rel_err(out.solution, xd) < 1e-7


def test_solver_argument_errors(cuda):
    from igaops_b200.solvers import GCRODR, LinearSolver

    with pytest.raises(ValueError):
        LinearSolver(0.0, 10)
    with pytest.raises(ValueError):
        LinearSolver(1e-6, 0)
    with pytest.raises(ValueError):
        LinearSolver(1e-6, 10, linear_type="minres")
    with pytest.raises(TypeError):
        LinearSolver(1e-6, 10, cleandod=(1, 2))
    with pytest.raises(TypeError):
        LinearSolver(1e-6, 10).solve(3, np.ones(4))
    with pytest.raises(ValueError):
        GCRODR(1e-6, 10, krylov_size=5, recycled_size=10)
    # non-convergence is not an exception: success = False with a warning
    T = torch.eye(50, dtype=torch.float64, device="cuda") + 0.01 * torch.randn(
        50, 50, dtype=torch.float64, device="cuda", generator=torch.Generator(device="cuda").manual_seed(1))
    with pytest.warns(UserWarning):
        out = LinearSolver(1e-14, 2, linear_type="gmres", verbose=False).solve(lambda v: T @ v, np.ones(50))
    assert not out.success


def test_c1_fd_is_exact_inverse_on_unit_square(cuda):
    """Known answer of the 2D benchmark configuration (p3, 64^2 elements,
    Greville unit square, Dirichlet on all sides, RHS U(-1,1) seed 0): with
    the identity map the weighted-quadrature stiffness equals the Gauss
    pencils the FD preconditioner diagonalises, so FD-GMRES converges in
    exactly one iteration."""
    from igaops_b200 import MFOperator, precompute_coefficients, unit_cube_ctrlpts
    from igaops_b200.fastdiag import SingleFD
    from igaops_b200.solvers import LinearSolver

    rl = rules(2, 3, 64)
    co = precompute_coefficients(rl, unit_cube_ctrlpts(rl, amplitude=0.0))
    op = MFOperator(rl, co["stiffness"], "gradu_gradv")
    fd = SingleFD("spatial")
    fd.compute_space_eigendecomposition(rl, np.ones((1, 2, 2), dtype=bool))
    free_np = np.asarray(fd.space_preconditioner.space_free_nodes[0])
    assert free_np.size == 65 * 65
    free = torch.as_tensor(free_np, device="cuda")
    N = rl[0].nbctrlpts ** 2

    def A(x):
        full = torch.zeros(N, dtype=torch.float64, device="cuda")
        full[free] = x
        return op.apply(full)[free]

    def P(x):
        full = torch.zeros(N, dtype=torch.float64, device="cuda")
        full[free] = x
        return fd.apply(full)[free]

    b = np.random.default_rng(0).uniform(-1.0, 1.0, free_np.size)
    ls = LinearSolver(1e-10, 200, linear_type="gmres", verbose=False)
    out = ls.solve(A, b, P)
    assert out.success
    assert ls.convergence_manager.parameters["iteration"].current == 1
    x = torch.as_tensor(np.asarray(out.solution), device="cuda")
    bt = torch.as_tensor(b, device="cuda")
    assert float(torch.linalg.vector_norm(A(x) - bt) / torch.linalg.vector_norm(bt)) < 1e-10
