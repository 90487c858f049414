"""Oracle parity at the full benchmark sizes.

* 3D degree 3, 128^3 elements (131^3 = 2,248,091 DOFs, 389^3 = 58,863,869
  quadrature points), perturbed cube, coefficients computed on the device:
  the fused FP64 and FP32 stiffness and mass matvecs against the oracle's
  FP64 restatement of BsplineOperations.compute_mf_scalar_gradu_gradv /
  compute_mf_scalar_u_v (src/igaops/operators/bsplines_ops.py:290-355) fed
  the same coefficients (copied to the host) and the same seeded vector.
  Tolerances, relative max norm: FP64 1e-12, FP32 1e-5.  Each oracle product
  takes about 15 s of host time.
* 3D 96^3, degrees 2..5, all faces Dirichlet, RHS U(-1,1) from seed 0: the
  mixed-precision refined solve's true relative residual, recomputed with the
  oracle's FP64 stiffness operator on the host, is below 1e-10 and within
  5e-12 of the FP64 Arnoldi estimate the solve stopped on.
"""
import numpy as np
import pytest
import torch

from oracle import mf as omf

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def c2(cuda):
    from igaops_b200 import GeometryOps, WeightedQuadrature, precompute_coefficients, unit_cube_ctrlpts

    q = WeightedQuadrature(3, GeometryOps.make_open_knotvector(3, 128), "2")
    rules = [q, q, q]
    coefs = precompute_coefficients(rules, unit_cube_ctrlpts(rules, amplitude=0.1))
    x = np.random.default_rng(0).standard_normal(q.nbctrlpts ** 3)
    yield rules, coefs, x
    del coefs
    torch.cuda.empty_cache()


def test_fullsize_stiffness_matches_oracle(c2):
    from igaops_b200 import MFOperator

    rules, coefs, x = c2
    K = MFOperator(rules, coefs["stiffness"], "gradu_gradv", dtype=torch.float64)
    assert K.fused and K.N == 131 ** 3 and K.Nq == 389 ** 3
    xd = torch.from_numpy(x).cuda()
    y64 = K.apply(xd).cpu().numpy()
    K.plan.check_status()
    del K
    K32 = MFOperator(rules, coefs["stiffness"], "gradu_gradv", dtype=torch.float32)
    y32 = K32.apply(xd.float()).double().cpu().numpy()
    K32.plan.check_status()
    del K32
    C = coefs["stiffness"].cpu().numpy()
    ref = omf.mf_gradu_gradv(rules, C, x)
    del C
    assert _rel(y64, ref) < 1e-12
    assert _rel(y32, ref) < 1e-5


def test_fullsize_mass_matches_oracle(c2):
    from igaops_b200 import MFOperator

    rules, coefs, x = c2
    M = MFOperator(rules, coefs["mass"], "u_v", dtype=torch.float64)
    assert M.fused
    xd = torch.from_numpy(x).cuda()
    y64 = M.apply(xd).cpu().numpy()
    M32 = MFOperator(rules, coefs["mass"], "u_v", dtype=torch.float32)
    y32 = M32.apply(xd.float()).double().cpu().numpy()
    M.plan.check_status()
    M32.plan.check_status()
    ref = omf.mf_u_v(rules, coefs["mass"].cpu().numpy(), x)
    assert _rel(y64, ref) < 1e-12
    assert _rel(y32, ref) < 1e-5


@pytest.mark.parametrize("p", [2, 3, 4, 5])
def test_c3_refined_solve_oracle_residual(cuda, p):
    from igaops_b200 import GeometryOps, WeightedQuadrature, precompute_coefficients, unit_cube_ctrlpts
    from igaops_b200.refine import EllipticPatchSolver

    q = WeightedQuadrature(p, GeometryOps.make_open_knotvector(p, 96), "2")
    rl = [q, q, q]
    co = precompute_coefficients(rl, unit_cube_ctrlpts(rl, amplitude=0.1), mass=False)
    S = EllipticPatchSolver(rl, co["stiffness"], np.ones((1, 3, 2), dtype=bool))
    rng = np.random.default_rng(0)
    b = np.zeros(S.N)
    b[S.free] = rng.uniform(-1.0, 1.0, S.free.size)
    # the bench's setting: stop on the FP64 Arnoldi estimate (the reference
    # GMRES's rule), no confirming matvec inside the solve
    out = S.solve_mixed(b, tolerance=1e-10, residual="arnoldi")
    assert out.success and out.residual_kind == "arnoldi"
    C = co["stiffness"].cpu().numpy()
    free = S.free
    del co, S
    torch.cuda.empty_cache()
    x = np.asarray(out.solution)
    r = b - omf.mf_gradu_gradv(rl, C, x)
    res = np.linalg.norm(r[free]) / np.linalg.norm(b[free])
    assert res < 1e-10, res
    assert abs(res - out.true_residual) < 5e-12, (res, out.true_residual)
