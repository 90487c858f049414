"""The device Gram kernel (iga_gram: G = A^H B over row sets, FP64
accumulation, two-stage fixed-order reduction) against a plain torch FP64
product, over the shapes the Krylov solvers use: the single-vector forms of
the Gram-Schmidt projections and norms (m x 1 and 1 x m, every accumulator
bucket up to 32 rows, FP64 and FP32 rows, a row stride larger than n), and
the general m1 x m2 real and complex forms.

Tolerance: relative max norm 1e-12 for FP64 rows; FP32 rows are summed in
FP64, so the reference is the FP64 product of the same FP32 values (1e-12).
"""
import pytest
import torch

from igaops_b200 import krylov_ops

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max().clamp_min(1e-300))


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("m,n", [(1, 1), (1, 2047), (3, 100_003), (5, 4096), (8, 777_777),
                                 (12, 65_537), (17, 300_001), (31, 250_000), (32, 131_072)])
def test_gram_single_vector_forms(cuda, dtype, m, n):
    g = torch.Generator(device="cuda").manual_seed(m * 1000 + n % 1000)
    ld = n + 5  # rows of a larger basis: stride > n
    Vb = torch.randn(m, ld, dtype=dtype, device="cuda", generator=g)
    V = Vb[:, :n]
    w = torch.randn(n, dtype=dtype, device="cuda", generator=g)
    ref = V.double() @ w.double()
    ws = krylov_ops.Workspace(torch.device("cuda"))
    G = krylov_ops.gram(ws, V, w)  # m x 1
    assert G.shape == (m, 1) and _rel(G[:, 0], ref) < TOL
    H = krylov_ops.gram(ws, w, V)  # 1 x m
    assert H.shape == (1, m) and _rel(H[0], ref) < TOL
    # repeated calls give the same bits (fixed reduction order)
    assert torch.equal(krylov_ops.gram(ws, V, w), G)


@pytest.mark.parametrize("m1,m2,n", [(12, 9, 4096), (2, 3, 1_000_003), (40, 1, 50_000),
                                     (64, 64, 20_000)])
def test_gram_general_forms(cuda, m1, m2, n):
    g = torch.Generator(device="cuda").manual_seed(m1 * 100 + m2)
    A = torch.randn(m1, n, dtype=torch.float64, device="cuda", generator=g)
    B = torch.randn(m2, n, dtype=torch.float64, device="cuda", generator=g)
    ws = krylov_ops.Workspace(torch.device("cuda"))
    assert _rel(krylov_ops.gram(ws, A, B), A @ B.T) < TOL


@pytest.mark.parametrize("m1,m2,n", [(1, 1, 100_000), (6, 1, 70_001), (5, 4, 4096)])
def test_gram_complex_forms(cuda, m1, m2, n):
    g = torch.Generator(device="cuda").manual_seed(7 + m1)
    A = torch.randn(m1, n, dtype=torch.complex128, device="cuda", generator=g)
    B = torch.randn(m2, n, dtype=torch.complex128, device="cuda", generator=g)
    ws = krylov_ops.Workspace(torch.device("cuda"))
    ref = A.conj() @ B.T
    assert _rel(krylov_ops.gram(ws, A, B), ref) < TOL
