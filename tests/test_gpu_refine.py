"""Mixed-precision refined solves (FGMRES in FP64 around an FP32 / BF16
inner solve) against the plain FP64 GPU path and the oracle's FP64 operator.

Bar: the true relative residual ||b - A x|| / ||b||, recomputed with the
oracle's FP64 matvec on the CPU, is below 1e-10 for every refined solve."""
import numpy as np
import pytest
import torch

from oracle import mf as omf
from tests._problems import rules

pytestmark = pytest.mark.gpu


def _problem(p, ne, amplitude=0.1, seed=0):
    from igaops_b200 import precompute_coefficients, unit_cube_ctrlpts
    from igaops_b200.refine import EllipticPatchSolver

    rl = rules(3, p, ne)
    co = precompute_coefficients(rl, unit_cube_ctrlpts(rl, amplitude=amplitude))
    S = EllipticPatchSolver(rl, co["stiffness"], np.ones((1, 3, 2), dtype=bool))
    rng = np.random.default_rng(seed)
    b = np.zeros(S.N)
    b[S.free] = rng.uniform(-1.0, 1.0, S.free.size)
    return rl, co["stiffness"].cpu().numpy(), S, b


def _oracle_residual(rl, C, free, x, b):
    r = b - omf.mf_gradu_gradv(rl, C, x)
    return np.linalg.norm(r[free]) / np.linalg.norm(b[free])


@pytest.mark.parametrize("p,ne", [(2, 10), (3, 12), (4, 9), (5, 8)])
def test_mixed_solve_reaches_fp64_tolerance(cuda, p, ne):
    rl, C, S, b = _problem(p, ne)
    out = S.solve_mixed(b, tolerance=1e-10)
    assert out.success
    assert out.true_residual < 1e-10
    assert _oracle_residual(rl, C, S.free, out.solution, b) < 1e-10
    x = out.solution
    mask = np.ones(S.N, dtype=bool)
    mask[S.free] = False
    assert np.all(x[mask] == 0.0)


def test_mixed_inner_gmres_and_fp64_path_agree(cuda):
    rl, C, S, b = _problem(3, 12, seed=1)
    ref = S.solve_fp64(b, tolerance=1e-10)
    assert ref.success
    assert _oracle_residual(rl, C, S.free, ref.solution, b) < 1e-9
    S.mixed.inner_iters = 3
    S.mixed._cache = {}
    out = S.solve_mixed(b, tolerance=1e-10)
    assert out.success and out.inner_iterations > 0
    assert _oracle_residual(rl, C, S.free, out.solution, b) < 1e-10
    d = np.linalg.norm(out.solution - ref.solution) / np.linalg.norm(ref.solution)
    assert d < 1e-7
    # the FP32 inner path without tensor cores converges as well
    out2 = S.solve_mixed(b, tolerance=1e-10, precond="fp")
    assert out2.success
    assert _oracle_residual(rl, C, S.free, out2.solution, b) < 1e-10


def test_mixed_solve_zero_rhs(cuda):
    _, _, S, b = _problem(2, 6)
    out = S.solve_mixed(np.zeros_like(b))
    assert out.success and np.all(out.solution == 0.0)


@pytest.mark.parametrize("precond", ["tc", "fp"])
def test_mixed_solve_arnoldi_stopping_rule(cuda, precond):
    """residual="arnoldi": the solve stops on the FP64 Arnoldi estimate (the
    reference GMRES's rule) without the confirming matvec; the solution is
    the one of the default mode, and the reported estimate matches the
    oracle's residual of the returned solution."""
    rl, C, S, b = _problem(3, 12, seed=2)
    ref = S.solve_mixed(b, tolerance=1e-10, precond=precond)
    out = S.solve_mixed(b, tolerance=1e-10, precond=precond, residual="arnoldi")
    assert ref.residual_kind == "true" and out.residual_kind == "arnoldi"
    assert out.success and out.true_residual < 1e-10
    assert out.outer_iterations == ref.outer_iterations
    if precond == "fp":
        assert out.fp64_matvecs == ref.fp64_matvecs - 1
    orc = _oracle_residual(rl, C, S.free, out.solution, b)
    assert orc < 1e-10
    assert abs(orc - out.true_residual) < 1e-12
    d = np.linalg.norm(out.solution - ref.solution) / np.linalg.norm(ref.solution)
    assert d < 1e-12
    with pytest.raises(ValueError):
        S.solve_mixed(b, residual="estimate")
