"""GPU parity of the space-time (arrowhead) fast-diagonalisation preconditioner
against the reference's outputs (golden fixtures) and the oracle.

Tolerances (relative max-norm): FP64 1e-11 (golden 1e-12), FP32 1e-5."""
import numpy as np
import pytest
import torch

from oracle import fd as ofd
from tests._golden import FixtureRule, load
from tests._problems import rel_err, rules

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag,adv", [("a1", None), ("a07", 0.7)])
def test_sptime_fd_matches_reference_golden(cuda, tag, adv):
    from igaops_b200.fastdiag import SingleFD

    d = load("sptime")
    qs, qt = FixtureRule(d, "space"), FixtureRule(d, "time")
    fd = SingleFD("spacetime")
    fd.compute_space_eigendecomposition([qs, qs], d["table"])
    fd.compute_time_schurdecomposition(qt)
    fd.update_space_eigenvalues(scalar_coefs=(0.25, 1.0))
    if adv is not None:
        fd.add_scalar_space_time_correctors(advection_corrector=[adv])
    assert np.array_equal(np.asarray(fd.sptm_preconditioner.sptm_free_nodes[0]), d["free"])
    assert rel_err(fd.apply(d[f"{tag}_v"]), d[f"{tag}_Pv"]) < 1e-12
    assert rel_err(fd.apply(d[f"{tag}_V"]), d[f"{tag}_PV"]) < 1e-12
    assert rel_err(fd.apply_transpose(d[f"{tag}_v"]), d[f"{tag}_PTv"]) < 1e-12
    v32 = torch.from_numpy(d[f"{tag}_v"]).float().cuda()
    assert rel_err(fd.apply(v32).double().cpu().numpy(), d[f"{tag}_Pv"]) < 1e-5


@pytest.mark.parametrize("sdim,p,ne,nt_el", [(2, 3, 12, 9), (3, 2, 6, 7), (1, 4, 20, 16)])
def test_sptime_fd_matches_oracle(cuda, sdim, p, ne, nt_el):
    from igaops_b200.fastdiag import SingleFD, rewrite_quadrature

    space = rules(sdim, p, ne)
    qt = rules(1, p, nt_el)[0]
    table = np.ones((1, sdim, 2), dtype=bool)
    table[0, 0, 1] = False
    fd = SingleFD("spacetime")
    fd.compute_space_eigendecomposition(space, table)
    fd.compute_time_schurdecomposition(qt)
    fd.update_space_eigenvalues(scalar_coefs=(0.1, 1.0))
    fd.add_scalar_space_time_correctors(advection_corrector=[1.3])
    ofdd = ofd.sptime_setup(rewrite_quadrature(space), table, rewrite_quadrature([qt])[0],
                            scalar_coefs=(0.1, 1.0), adv_corr=1.3)
    rng = np.random.default_rng(sdim * 100 + ne)
    N = int(np.prod([q.nbctrlpts for q in space])) * qt.nbctrlpts
    x = rng.standard_normal(N)
    assert rel_err(fd.apply(x), ofd.sptime_apply(ofdd, x)) < 1e-11
    assert rel_err(fd.apply_transpose(x), ofd.sptime_apply(ofdd, x, transpose=True)) < 1e-11


@pytest.mark.parametrize("tag,adv", [("l1", None), ("l07", 0.7)])
def test_sptime_qz_fd_matches_reference_golden(cuda, tag, adv):
    """The QZ ("legacy") form, use_arrowhead=False (preconditioner.py:66-86)."""
    from igaops_b200.fastdiag import SingleFD, SpaceTimeQZFD

    d = load("sptime")
    qs, qt = FixtureRule(d, "space"), FixtureRule(d, "time")
    fd = SingleFD("spacetime")
    fd.compute_space_eigendecomposition([qs, qs], d["table"])
    fd.compute_time_schurdecomposition(qt, use_arrowhead=False)
    assert isinstance(fd.sptm_preconditioner, SpaceTimeQZFD)
    fd.update_space_eigenvalues(scalar_coefs=(0.25, 1.0))
    if adv is not None:
        fd.add_scalar_space_time_correctors(advection_corrector=[adv])
    assert rel_err(fd.apply(d[f"{tag}_v"]), d[f"{tag}_Pv"]) < 1e-12
    assert rel_err(fd.apply(d[f"{tag}_V"]), d[f"{tag}_PV"]) < 1e-12
    assert rel_err(fd.apply_transpose(d[f"{tag}_v"]), d[f"{tag}_PTv"]) < 1e-12
    v32 = torch.from_numpy(d[f"{tag}_v"]).float().cuda()
    assert rel_err(fd.apply(v32).double().cpu().numpy(), d[f"{tag}_Pv"]) < 1e-5


@pytest.mark.parametrize("sdim,p,ne,nt_el", [(2, 3, 12, 9), (3, 2, 6, 7), (1, 4, 20, 16)])
def test_sptime_qz_fd_matches_oracle(cuda, sdim, p, ne, nt_el):
    from igaops_b200.fastdiag import SingleFD, rewrite_quadrature

    space = rules(sdim, p, ne)
    qt = rules(1, p, nt_el)[0]
    table = np.ones((1, sdim, 2), dtype=bool)
    table[0, 0, 1] = False
    fd = SingleFD("spacetime")
    fd.compute_space_eigendecomposition(space, table)
    fd.compute_time_schurdecomposition(qt, use_arrowhead=False)
    fd.update_space_eigenvalues(scalar_coefs=(0.1, 1.0))
    fd.add_scalar_space_time_correctors(advection_corrector=[1.3])
    ofdd = ofd.sptime_qz_setup(rewrite_quadrature(space), table, rewrite_quadrature([qt])[0],
                               scalar_coefs=(0.1, 1.0), adv_corr=1.3)
    rng = np.random.default_rng(sdim * 100 + ne + 1)
    N = int(np.prod([q.nbctrlpts for q in space])) * qt.nbctrlpts
    x = rng.standard_normal(N)
    assert rel_err(fd.apply(x), ofd.sptime_qz_apply(ofdd, x)) < 1e-11
    assert rel_err(fd.apply_transpose(x), ofd.sptime_qz_apply(ofdd, x, transpose=True)) < 1e-11
    # the arrowhead and QZ forms are the same preconditioner
    fa = SingleFD("spacetime")
    fa.compute_space_eigendecomposition(space, table)
    fa.compute_time_schurdecomposition(qt)
    fa.update_space_eigenvalues(scalar_coefs=(0.1, 1.0))
    fa.add_scalar_space_time_correctors(advection_corrector=[1.3])
    assert rel_err(fd.apply(x), fa.apply(x)) < 1e-9
