"""Full-size checks of the fused matvec at the benchmark configuration
(3D, degree 3, 128^3 elements: 2,248,091 DOFs, 58,863,869 quadrature points,
the perturbed cube of bench.py), where the oracle is too slow to run: the
size-independent properties of the operators and agreement with the
independent unfused device path (the reference's sequence of L-mode products
and pointwise scalings, itself checked against the oracle at small sizes).

Tolerances (relative max norm): FP64 1e-12 against the unfused path and for
linearity; FP32 1e-5 against FP64; K 1 = 0 (constants have zero gradient)
to 1e-12 of |K x| for a random x of unit entries.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max().clamp_min(1e-300))


@pytest.fixture(scope="module")
def c2(cuda):
    from igaops_b200 import GeometryOps, WeightedQuadrature, precompute_coefficients, unit_cube_ctrlpts

    q = WeightedQuadrature(3, GeometryOps.make_open_knotvector(3, 128), "2")
    rules = [q, q, q]
    coefs = precompute_coefficients(rules, unit_cube_ctrlpts(rules, amplitude=0.1))
    return rules, coefs


def test_fullsize_stiffness_properties(c2):
    from igaops_b200 import MFOperator

    rules, coefs = c2
    K = MFOperator(rules, coefs["stiffness"], "gradu_gradv", dtype=torch.float64)
    assert K.fused and K.N == 131 ** 3
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn(K.N, dtype=torch.float64, device="cuda", generator=g)
    z = torch.randn(K.N, dtype=torch.float64, device="cuda", generator=g)
    Kx, Kz = K.apply(x), K.apply(z)
    # linearity
    assert _rel(K.apply(2.0 * x - 3.0 * z), 2.0 * Kx - 3.0 * Kz) < 1e-12
    # constants are in the kernel of the stiffness operator
    one = torch.ones(K.N, dtype=torch.float64, device="cuda")
    assert float(K.apply(one).abs().max() / Kx.abs().max()) < 1e-12
    # the independent unfused device path
    G = MFOperator(rules, coefs["stiffness"], "gradu_gradv", dtype=torch.float64,
                   force_generic=True)
    assert not G.fused
    assert _rel(Kx, G.apply(x)) < 1e-12
    del G
    # FP32 operator against FP64
    K32 = MFOperator(rules, coefs["stiffness"], "gradu_gradv", dtype=torch.float32)
    assert _rel(K32.apply(x.float()).double(), Kx) < 1e-5
    # every launch shape of the autotuner gives the same product
    for nseg in (1, 3, 8):
        Kn = MFOperator(rules, coefs["stiffness"], "gradu_gradv", dtype=torch.float64, nseg=nseg)
        assert _rel(Kn.apply(x), Kx) < 1e-12
    K.plan.check_status()


def test_fullsize_mass_properties(c2):
    from igaops_b200 import MFOperator

    rules, coefs = c2
    M = MFOperator(rules, coefs["mass"], "u_v", dtype=torch.float64)
    assert M.fused
    g = torch.Generator(device="cuda").manual_seed(1)
    x = torch.randn(M.N, dtype=torch.float64, device="cuda", generator=g)
    Mx = M.apply(x)
    G = MFOperator(rules, coefs["mass"], "u_v", dtype=torch.float64, force_generic=True)
    assert _rel(Mx, G.apply(x)) < 1e-12
    # the mass of the constant function: M 1 = W0 (x) W0 (x) W0 c (the basis
    # is a partition of unity), the generic path's product of the weights alone
    one = torch.ones(M.N, dtype=torch.float64, device="cuda")
    assert _rel(M.apply(one), G.apply(one)) < 1e-12
    assert bool(torch.all(M.apply(one) > 0))
    M32 = MFOperator(rules, coefs["mass"], "u_v", dtype=torch.float32)
    assert _rel(M32.apply(x.float()).double(), Mx) < 1e-5
    M.plan.check_status()
