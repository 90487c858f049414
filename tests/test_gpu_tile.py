"""The tensor-core tile kernel (csrc/mf_tile.cu) against the oracle: FP64
stiffness (symmetric coefficients) and mass, 1e-12 relative max norm, over
degrees 2..4, uneven extents, partial tiles and several right-hand sides;
two applies in a row give the same product.  The tile kernel runs when
asked for (kernel="tile") or when the autotuner (kernel="auto" with
nseg="auto") times it faster than the pencil kernel for the shape."""
import numpy as np
import pytest
import torch

from oracle import mf as omf
from tests._problems import coefficients, rel_err, rules

pytestmark = pytest.mark.gpu

CASES = [(3, 7), (2, 5), (4, 4), (3, 20), (3, [5, 9, 17]), (2, [33, 6, 11]), (4, [3, 12, 7]),
         (3, 1)]


@pytest.mark.parametrize("p,ne", CASES)
@pytest.mark.parametrize("op", ["gradu_gradv", "u_v"])
def test_tile_kernel_matches_oracle(cuda, p, ne, op):
    from igaops_b200 import MFOperator

    rl = rules(3, p, ne)
    rng = np.random.default_rng(11)
    N = int(np.prod([q.nbctrlpts for q in rl]))
    x = rng.standard_normal(N)
    c = coefficients(op, rl, rng)
    oper = MFOperator(rl, c, op, kernel="tile")
    assert oper.fused and oper.tiled
    ref = omf.OPS[op](rl, c, x)
    xd = torch.from_numpy(x).cuda()
    y1 = oper.apply(xd).cpu().numpy()
    y2 = oper.apply(xd).cpu().numpy()
    oper.plan.check_status()
    assert rel_err(y1, ref) < 1e-12, rel_err(y1, ref)
    assert rel_err(y2, ref) < 1e-12


def test_tile_kernel_several_columns(cuda):
    from igaops_b200 import MFOperator

    rl = rules(3, 3, [6, 10, 8])
    rng = np.random.default_rng(12)
    N = int(np.prod([q.nbctrlpts for q in rl]))
    X = rng.standard_normal((N, 3))
    c = coefficients("gradu_gradv", rl, rng)
    oper = MFOperator(rl, c, "gradu_gradv", kernel="tile")
    assert oper.tiled
    got = oper.apply(X)
    assert rel_err(got, omf.mf_gradu_gradv(rl, c, X)) < 1e-12


def test_tile_and_pencil_kernels_agree(cuda):
    from igaops_b200 import MFOperator

    rl = rules(3, 3, 24)
    rng = np.random.default_rng(13)
    N = int(np.prod([q.nbctrlpts for q in rl]))
    c = coefficients("gradu_gradv", rl, rng)
    x = torch.from_numpy(rng.standard_normal(N)).cuda()
    T = MFOperator(rl, c, "gradu_gradv", kernel="tile")
    P = MFOperator(rl, c, "gradu_gradv", kernel="pencil")
    assert T.tiled and not P.tiled
    a, b = T.apply(x), P.apply(x)
    assert float((a - b).abs().max() / b.abs().max()) < 1e-12


def test_tile_kernel_refuses_what_it_does_not_cover(cuda):
    from igaops_b200 import MFOperator

    rl = rules(3, 3, 5)
    rng = np.random.default_rng(14)
    c = coefficients("gradu_gradv", rl, rng, symmetric=False)
    with pytest.raises(NotImplementedError):
        MFOperator(rl, c, "gradu_gradv", kernel="tile")
    assert not MFOperator(rl, c, "gradu_gradv").tiled
    rl5 = rules(3, 5, 4)
    c5 = coefficients("gradu_gradv", rl5, rng)
    with pytest.raises(NotImplementedError):
        MFOperator(rl5, c5, "gradu_gradv", kernel="tile")


@pytest.mark.parametrize("op", ["gradu_gradv", "u_v"])
def test_autotuner_times_both_tilings_and_keeps_the_faster(cuda, op):
    """kernel="auto" with nseg="auto": the autotuner times the pencil
    kernel (at its tuned segment count) against the tile kernel on the
    operator's own data, keeps the faster, and records both timings; the
    chosen kernel gives the oracle's product; a second operator of the
    same shape reuses the cached choice without timing again."""
    from igaops_b200 import MFOperator, tune

    rl = rules(3, 3, 18)
    rng = np.random.default_rng(5)
    N = int(np.prod([q.nbctrlpts for q in rl]))
    x = rng.standard_normal(N)
    c = coefficients(op, rl, rng)
    pencil = MFOperator(rl, c, op, nseg="auto", kernel="pencil")
    key = tune.shape_key(pencil.plan)
    tune._CACHE.pop("kernel|" + key, None)
    tune._TIMES.pop("kernel|" + key, None)
    A = MFOperator(rl, c, op, nseg="auto")
    dec = tune.decisions()[key]
    assert dec["kernel"] == ("tile" if A.tiled else "pencil")
    assert dec["pencil_ms"] > 0 and dec["tile_ms"] > 0
    assert A.tiled == (dec["tile_ms"] < dec["pencil_ms"])
    ref = omf.OPS[op](rl, c, x)
    got = A.apply(torch.from_numpy(x).cuda()).cpu().numpy()
    A.plan.check_status()
    assert rel_err(got, ref) < 1e-12
    tune._TIMES["kernel|" + key]["marker"] = 1.0
    B = MFOperator(rl, c, op, nseg="auto")
    assert B.tiled == A.tiled and tune.decisions()[key].get("marker") == 1.0
