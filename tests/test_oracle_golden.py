"""The oracle (oracle/) reproduces the reference's own outputs (golden
fixtures generated from the unmodified reference) -- this pins the checker
that the GPU parity tests use.  CPU only."""
import numpy as np
import pytest

from oracle import fd as ofd
from oracle import krylov as okr
from oracle import mf as omf
from tests._golden import FixtureRule, load, rules


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - b)) / max(np.max(np.abs(b)), 1e-300))


def test_lmode_matches_reference():
    d = load("matvec")
    mats = [d[f"lm_M{k}"] for k in range(3)]
    assert rel(omf.lmode_apply(mats, d["lm_v"]), d["lm_y"]) < 1e-14
    assert rel(omf.lmode_apply(mats, d["lm_vt"], transpose=True), d["lm_yt"]) < 1e-14


@pytest.mark.parametrize("name", ["2d_wq2", "3d_wq2", "3d_wq1", "3d_gauss", "st_01", "st_00", "st_10"])
@pytest.mark.parametrize("op", ["u_v", "gradu_gradv", "gradu_v", "u_gradv"])
def test_matvec_matches_reference(name, op):
    d = load("matvec")
    ndim = 2 if name.startswith("2d") else 3
    rl = rules(d, name, ndim)
    td = tuple(int(t) for t in d[f"{name}_td"])
    td = None if td[0] < 0 else td
    c = d[f"{name}_{op}_c"]
    got = omf.OPS[op](rl, c, d[f"{name}_x"], td)
    assert rel(got, d[f"{name}_{op}_y"]) < 1e-13
    if f"{name}_{op}_Y" in d:
        got = omf.OPS[op](rl, c, d[f"{name}_X"], td)
        assert rel(got, d[f"{name}_{op}_Y"]) < 1e-13


def test_fd_matches_reference():
    d = load("fastdiag")
    from tests._problems import rules as mk

    q = mk(1, 3, 4, kind="gauss")[0]
    fd = ofd.setup([q] * 3, d["table"], scalar_coefs=d["scalar_coefs"], stiff_corr=d["corr"])
    assert np.array_equal(fd.free, d["free"])
    for k in range(3):
        assert np.allclose(np.abs(fd.U[k]), np.abs(d[f"U{k}"]), atol=1e-12)
        assert rel(fd.lam[k], d[f"lam{k}"]) < 1e-12
    assert rel(fd.eig, d["eig"]) < 1e-12
    assert rel(ofd.apply(fd, d["v"]), d["Pv"]) < 1e-12
    assert rel(ofd.apply(fd, d["V"]), d["PV"]) < 1e-12


def test_fd_wq_input_is_rewritten_to_gauss():
    d = load("fastdiag")
    from igaops_b200.fastdiag import rewrite_quadrature

    w = FixtureRule(d, "wq_rule")
    g = rewrite_quadrature([w, w])
    fd = ofd.setup(g, np.ones((1, 2, 2), dtype=bool))
    assert rel(ofd.apply(fd, d["wq_v"]), d["wq_Pv"]) < 1e-12


def test_gmres_matches_reference():
    d = load("solvers")
    q = FixtureRule(d, "gm_rule")
    rl = [q, q]
    coefs, b, free = d["gm_coefs"], d["gm_b"], d["gm_free"]
    N = q.nbctrlpts ** 2
    from igaops_b200.fastdiag import rewrite_quadrature

    fd = ofd.setup(rewrite_quadrature(rl), np.ones((1, 2, 2), dtype=bool))

    def A(x):
        full = np.zeros(N)
        full[free] = x
        return omf.mf_gradu_gradv(rl, coefs, full)[free]

    def P(x):
        full = np.zeros(N)
        full[free] = x
        return ofd.apply(fd, full)[free]

    for tol in (1e-6, 1e-10):
        x, res, ok, _ = okr.gmres(A, b, P, tol=tol, maxiters=100)
        assert ok
        assert len(res) == len(d[f"gm_res_{tol:g}"])
        assert np.allclose(res, d[f"gm_res_{tol:g}"], rtol=1e-6, atol=1e-13)
        assert rel(x, d[f"gm_x_{tol:g}"]) < 1e-10
    x, res, ok, _ = okr.gmres(A, b, None, tol=1e-10, maxiters=200)
    assert len(res) == len(d["gm_res_noprec"])
    assert rel(x, d["gm_x_noprec"]) < 1e-8


def test_gmres_mask_and_x0_match_reference():
    d = load("solvers")
    T = d["tri_T"]
    x, res, ok, _ = okr.gmres(lambda v: T @ v, d["tri_b"], None, tol=1e-9, maxiters=100,
                              cleandod=list(d["tri_mask"]), x0=d["tri_x0"])
    assert len(res) == len(d["tri_res"])
    assert rel(x, d["tri_x"]) < 1e-10


def test_gcrodr_matches_reference():
    d = load("solvers")
    T = d["gc_T"]
    g = okr.GCRODR(1e-8, 2000, m=30, k=10)
    x1, r1, ok1 = g.solve(lambda v: T @ v, d["gc_rhs"])
    x2, r2, ok2 = g.solve(lambda v: T @ v, 0.5 * d["gc_rhs"] + 0.1)
    assert ok1 and ok2
    assert len(r1) == len(d["gc_res1"]) and len(r2) == len(d["gc_res2"])
    assert rel(x1, d["gc_x1"]) < 1e-8
    assert rel(x2, d["gc_x2"]) < 1e-8


def test_geometry_matches_reference():
    d = load("geometry")
    q = FixtureRule(d, "rule")
    basis = [q.basis] * 3
    J = omf.eval_jacobian(basis, d["ctrlpts"])
    assert rel(J, d["jac"]) < 1e-13
    G = np.einsum("li...,lj...->ij...", J, J)
    det = np.linalg.det(np.moveaxis(G, (0, 1), (-2, -1)))
    assert rel(np.sqrt(det), d["det_jac"]) < 1e-12
    qp = omf.eval_interpolation(basis, d["ctrlpts"])
    assert rel(qp, d["qp_phy"]) < 1e-14


@pytest.mark.parametrize("name", ["2d", "3d", "3g", "st"])
@pytest.mark.parametrize("op", ["u_v", "gradu_gradv", "gradu_v", "u_gradv"])
def test_nurbs_matvec_matches_reference(name, op):
    from oracle import nurbs as onu

    d = load("nurbs")
    ndim = 2 if name == "2d" else 3
    rl = rules(d, name, ndim)
    td = tuple(int(t) for t in d[f"{name}_td"])
    td = None if td[0] < 0 else td
    got = onu.mf_nurbs(op, rl, d[f"{name}_{op}_c"], d[f"{name}_x"], d[f"{name}_w"], td)
    assert rel(got, d[f"{name}_{op}_y"]) < 1e-13
    if op == "gradu_gradv" and f"{name}_X" in d:
        got = onu.mf_nurbs(op, rl, d[f"{name}_{op}_c"], d[f"{name}_X"], d[f"{name}_w"], td)
        assert rel(got, d[f"{name}_{op}_Y"]) < 1e-13


@pytest.mark.parametrize("name", ["2d", "3d", "3g"])
def test_nurbs_evaluations_match_reference(name):
    from oracle import nurbs as onu

    d = load("nurbs")
    ndim = 2 if name == "2d" else 3
    basis = [FixtureRule(d, f"{name}_g{k}").basis for k in range(ndim)]
    u, w = d[f"{name}_u"], d[f"{name}_w"]
    assert rel(onu.eval_interpolation(basis, u, w), d[f"{name}_interp"]) < 1e-13
    assert rel(onu.eval_jacobian(basis, u, w), d[f"{name}_jac"]) < 1e-12
    assert rel(onu.eval_hessian(basis, u, w), d[f"{name}_hess"]) < 1e-11


def test_sptime_fd_matches_reference():
    from igaops_b200.fastdiag import rewrite_quadrature

    d = load("sptime")
    qs = rewrite_quadrature([FixtureRule(d, "space")])[0]
    qt = rewrite_quadrature([FixtureRule(d, "time")])[0]
    for tag, adv in (("a1", 1.0), ("a07", 0.7)):
        fd = ofd.sptime_setup([qs, qs], d["table"], qt, scalar_coefs=(0.25, 1.0), adv_corr=adv)
        assert rel(ofd.sptime_apply(fd, d[f"{tag}_v"]), d[f"{tag}_Pv"]) < 1e-12
        assert rel(ofd.sptime_apply(fd, d[f"{tag}_v"], transpose=True), d[f"{tag}_PTv"]) < 1e-12
        V = d[f"{tag}_V"]
        got = np.stack([ofd.sptime_apply(fd, V[:, k]) for k in range(V.shape[1])], axis=1)
        assert rel(got, d[f"{tag}_PV"]) < 1e-12


def test_sptime_qz_fd_matches_reference():
    """The QZ ("legacy") space-time form (time_legacy.py:43-170)."""
    from igaops_b200.fastdiag import rewrite_quadrature

    d = load("sptime")
    qs = rewrite_quadrature([FixtureRule(d, "space")])[0]
    qt = rewrite_quadrature([FixtureRule(d, "time")])[0]
    for tag, adv in (("l1", 1.0), ("l07", 0.7)):
        fd = ofd.sptime_qz_setup([qs, qs], d["table"], qt, scalar_coefs=(0.25, 1.0), adv_corr=adv)
        assert rel(ofd.sptime_qz_apply(fd, d[f"{tag}_v"]), d[f"{tag}_Pv"]) < 1e-12
        assert rel(ofd.sptime_qz_apply(fd, d[f"{tag}_v"], transpose=True), d[f"{tag}_PTv"]) < 1e-12
        V = d[f"{tag}_V"]
        got = np.stack([ofd.sptime_qz_apply(fd, V[:, k]) for k in range(V.shape[1])], axis=1)
        assert rel(got, d[f"{tag}_PV"]) < 1e-12
