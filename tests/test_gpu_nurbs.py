"""GPU parity of the rational (NURBS) operators and evaluations: against the
reference's own outputs (golden fixtures) and against the oracle
(oracle/nurbs.py) on larger seeded patches that take the fused kernels.

Tolerances (relative max-norm): FP64 1e-12 (evaluations 1e-11), FP32 1e-5.
"""
import numpy as np
import pytest
import torch

from oracle import nurbs as onu
from tests._golden import FixtureRule, load, rules as golden_rules
from tests._problems import coefficients, rel_err, rules

pytestmark = pytest.mark.gpu

OPS = ["u_v", "gradu_gradv", "gradu_v", "u_gradv"]


@pytest.mark.parametrize("name", ["2d", "3d", "3g", "st"])
@pytest.mark.parametrize("op", OPS)
def test_nurbs_matvec_matches_reference_golden(cuda, name, op):
    from igaops_b200.nurbs import NurbsOperations

    d = load("nurbs")
    ndim = 2 if name == "2d" else 3
    rl = golden_rules(d, name, ndim)
    td = tuple(int(t) for t in d[f"{name}_td"])
    td = None if td[0] < 0 else td
    fn = getattr(NurbsOperations, f"compute_mf_scalar_{op}")
    c, w = d[f"{name}_{op}_c"], d[f"{name}_w"]
    assert rel_err(fn(rl, c, d[f"{name}_x"], time_ders=td, nurbs_weights=w),
                   d[f"{name}_{op}_y"]) < 1e-12
    if op == "gradu_gradv" and f"{name}_X" in d:
        assert rel_err(fn(rl, c, d[f"{name}_X"], time_ders=td, nurbs_weights=w),
                       d[f"{name}_{op}_Y"]) < 1e-12


@pytest.mark.parametrize("name", ["2d", "3d", "3g"])
def test_nurbs_evaluations_match_reference_golden(cuda, name):
    from igaops_b200.nurbs import NurbsOperations

    d = load("nurbs")
    ndim = 2 if name == "2d" else 3
    basis = [FixtureRule(d, f"{name}_g{k}").basis for k in range(ndim)]
    u, w = d[f"{name}_u"], d[f"{name}_w"]
    assert rel_err(NurbsOperations.eval_interpolation(basis, u, nurbs_weights=w),
                   d[f"{name}_interp"]) < 1e-12
    assert rel_err(NurbsOperations.eval_jacobien(basis, u, nurbs_weights=w), d[f"{name}_jac"]) < 1e-11
    assert rel_err(NurbsOperations.eval_hessian(basis, u, nurbs_weights=w), d[f"{name}_hess"]) < 1e-11


@pytest.mark.parametrize("ndim,p,ne", [(2, 3, 20), (3, 3, 9), (3, 4, 7)])
@pytest.mark.parametrize("op", OPS)
def test_nurbs_operator_matches_oracle(cuda, ndim, p, ne, op):
    """Larger WQ type 2 patches: every term runs in the fused kernel."""
    from igaops_b200.nurbs import NurbsMFOperator

    rng = np.random.default_rng(17 * ndim + p + ne)
    rl = rules(ndim, p, ne)
    N = int(np.prod([q.nbctrlpts for q in rl]))
    w = 0.7 + 0.6 * rng.random(N)
    c = coefficients(op, rl, rng)
    x = rng.standard_normal(N)
    ref = onu.mf_nurbs(op, rl, c, x, w)
    oper = NurbsMFOperator(rl, c, w, op)
    assert all(t.fused for _, t in oper.terms)
    assert rel_err(oper.apply(x), ref) < 1e-12
    oper32 = NurbsMFOperator(rl, c, w, op, dtype=torch.float32)
    got = oper32.apply(torch.from_numpy(x).float().cuda()).double().cpu().numpy()
    assert rel_err(got, ref) < 1e-5


def test_nurbs_unit_weights_equal_bspline(cuda):
    """All weights 1: the rational operator is the B-spline one."""
    from igaops_b200 import BsplineOperations
    from igaops_b200.nurbs import NurbsOperations

    rng = np.random.default_rng(5)
    rl = rules(3, 2, 6)
    N = int(np.prod([q.nbctrlpts for q in rl]))
    c = coefficients("gradu_gradv", rl, rng)
    x = rng.standard_normal(N)
    a = NurbsOperations.compute_mf_scalar_gradu_gradv(rl, c, x, nurbs_weights=np.ones(N))
    b = BsplineOperations.compute_mf_scalar_gradu_gradv(rl, c, x)
    assert rel_err(a, b) < 1e-12


def test_nurbs_geometry_quarter_annulus(cuda):
    """Rational geometry: a quarter annulus (exact circle arcs, weights
    sqrt(2)/2 on the middle row) evaluated on the device equals the oracle's
    rational evaluation, and its det J is positive."""
    from igaops_b200.geometry import SingleSpline

    q2 = rules(1, 2, 1, kind="gauss")[0]
    q1 = rules(1, 2, 4, kind="gauss")[0]
    # direction 1 radial (p=2, 4 elements, 6 points r in [1, 2]); direction 2 angular arc
    r = np.linspace(1.0, 2.0, q1.nbctrlpts)
    arc = np.array([[1.0, 0.0], [1.0, 1.0], [0.0, 1.0]])
    wa = np.array([1.0, np.sqrt(0.5), 1.0])
    X = np.concatenate([r * a[0] for a in arc])
    Y = np.concatenate([r * a[1] for a in arc])
    w = np.repeat(wa, r.size)
    ctrl = np.stack([X, Y])
    spl = SingleSpline(ctrl, w, [q1, q2]).evaluate_spline()
    basis = [q1.basis, q2.basis]
    assert rel_err(spl.qp_phy, onu.eval_interpolation(basis, ctrl, w)) < 1e-12
    assert rel_err(spl.jac, onu.eval_jacobian(basis, ctrl, w)) < 1e-12
    rad = np.hypot(spl.qp_phy[0], spl.qp_phy[1])
    assert np.all(rad > 1.0 - 1e-12) and np.all(rad < 2.0 + 1e-12)
    assert np.all(spl.det_jac > 0)
