"""Generate the golden fixtures of tests/golden/ from the unmodified reference.

Run where the igaops reference source is available (it is not needed on the
GPU box, which only reads the committed .npz files):

    python tests/golden/make_golden.py <igaops source dir> [fixture ...]

The igaops source directory (the one holding ``src/igaops``) is the first
argument, or the ``IGAOPS_REFERENCE_SRC`` environment variable when no
argument is given.

The reference imports the third-party ``geomdl`` (not installable here); the
stand-in package ``oracle/geomdl_shim`` supplies the three helpers it calls.
Every input is seeded; the fixtures store inputs and reference outputs.
"""
from __future__ import annotations

import logging
import os
import sys
from pathlib import Path

import numpy as np
import scipy.sparse as sp

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
if len(sys.argv) > 1:
    REF = Path(sys.argv[1])
elif os.environ.get("IGAOPS_REFERENCE_SRC"):
    REF = Path(os.environ["IGAOPS_REFERENCE_SRC"])
else:
    sys.exit("usage: make_golden.py <igaops source dir> [fixture ...] "
             "(or set IGAOPS_REFERENCE_SRC)")
sys.path[:0] = [str(REPO / "oracle" / "geomdl_shim"), str(REF / "src")]
logging.disable(logging.WARNING)

from igaops.common import KronProduct, combine_arrays  # noqa: E402
from igaops.fastdiag import SingleFD  # noqa: E402
from igaops.geometry import GeometryOps  # noqa: E402
from igaops.geometry.mixin.template import SingleSpline  # noqa: E402
from igaops.operators import BsplineOperations, MatrixFree  # noqa: E402
from igaops.quadrature import StandardGauss, WeightedQuadrature  # noqa: E402
from igaops.solvers import GCRODR, LinearSolver  # noqa: E402


def pack_csr(prefix: str, M, out: dict):
    M = sp.csr_array(M)
    out[prefix + "_data"] = M.data
    out[prefix + "_indices"] = M.indices.astype(np.int32)
    out[prefix + "_indptr"] = M.indptr.astype(np.int32)
    out[prefix + "_shape"] = np.asarray(M.shape, dtype=np.int64)


def pack_rule(prefix: str, q, out: dict):
    out[prefix + "_degree"] = np.asarray(q.degree)
    out[prefix + "_knotvector"] = np.asarray(q.knotvector, dtype=float)
    out[prefix + "_quadpts"] = np.asarray(q.quadpts, dtype=float)
    for k, B in enumerate(q.basis):
        pack_csr(f"{prefix}_B{k}", B, out)
    for k, W in enumerate(q.weights):
        pack_csr(f"{prefix}_W{k}", W, out)


def make_rule(kind, p, ne, rule="endpoint"):
    kv = GeometryOps.make_open_knotvector(p, ne)
    if kind == "gauss":
        return StandardGauss(p, kv, "legendre")
    if kind == "lobatto":
        return StandardGauss(p, kv, "lobatto")
    return WeightedQuadrature(p, kv, kind[-1], rule)


def quadrature_fixtures():
    out = {}
    cases = []
    for kind in ("wq1", "wq2"):
        for rule in ("endpoint", "cellcenter"):
            for p, ne in ((2, 4), (3, 8), (4, 5), (5, 6), (1, 4), (3, 1)):
                cases.append((kind, p, ne, rule))
    for kind in ("gauss", "lobatto"):
        for p, ne in ((2, 3), (3, 4), (5, 2)):
            cases.append((kind, p, ne, "endpoint"))
    cases.append(("wq2", 3, 64, "endpoint"))
    names = []
    for i, (kind, p, ne, rule) in enumerate(cases):
        q = make_rule(kind, p, ne, rule)
        pack_rule(f"r{i}", q, out)
        names.append(f"{kind}:{p}:{ne}:{rule}")
    out["names"] = np.asarray(names)
    np.savez_compressed(HERE / "quadrature.npz", **out)


def coef_for(op, ndim, nq, rng):
    if op == "u_v":
        return 1.0 + 0.5 * rng.random(nq)
    if op == "gradu_gradv":
        c = 0.3 * rng.standard_normal((ndim, ndim, nq))
        for i in range(ndim):
            c[i, i] += 2.0
        return c
    return rng.standard_normal((ndim, nq))


def matvec_fixtures():
    out = {}
    cases = [
        ("2d_wq2", [("wq2", 3, 6)] * 2, None),
        ("3d_wq2", [("wq2", 2, 4)] * 3, None),
        ("3d_wq1", [("wq1", 3, 3)] * 3, None),
        ("3d_gauss", [("gauss", 3, 3)] * 3, None),
        ("st_01", [("wq2", 2, 3), ("wq2", 2, 3), ("wq2", 2, 2)], (0, 1)),
        ("st_00", [("wq2", 2, 3), ("wq2", 2, 3), ("wq2", 2, 2)], (0, 0)),
        ("st_10", [("wq2", 2, 3), ("wq2", 2, 3), ("wq2", 2, 2)], (1, 0)),
    ]
    names = []
    for ci, (name, spec, td) in enumerate(cases):
        rng = np.random.default_rng(100 + ci)
        rules = [make_rule(k, p, ne) for k, p, ne in spec]
        for d, q in enumerate(rules):
            pack_rule(f"{name}_r{d}", q, out)
        ndim = len(rules)
        N = int(np.prod([q.nbctrlpts for q in rules]))
        nq = int(np.prod([q.nbquadpts for q in rules]))
        x = rng.standard_normal(N)
        X = rng.standard_normal((N, 2))
        out[f"{name}_x"] = x
        out[f"{name}_X"] = X
        for op in ("u_v", "gradu_gradv", "gradu_v", "u_gradv"):
            c = coef_for(op, ndim, nq, rng)
            out[f"{name}_{op}_c"] = c
            fn = getattr(BsplineOperations, f"compute_mf_scalar_{op}")
            out[f"{name}_{op}_y"] = fn(rules, c, x, time_ders=td)
            if op in ("u_v", "gradu_gradv"):
                out[f"{name}_{op}_Y"] = fn(rules, c, X, time_ders=td)
        names.append(name)
        out[f"{name}_td"] = np.asarray(td if td is not None else (-1, -1))
    out["names"] = np.asarray(names)
    # L-mode products on random sparse/dense factors
    rng = np.random.default_rng(7)
    mats = [rng.standard_normal((4, 3)), sp.random(5, 6, density=0.5, random_state=1, format="csr"),
            rng.standard_normal((2, 5))]
    for k, M in enumerate(mats):
        out[f"lm_M{k}"] = M.toarray() if sp.issparse(M) else M
    v = rng.standard_normal(3 * 6 * 5)
    out["lm_v"] = v
    out["lm_y"] = MatrixFree.apply(mats, v)
    vt = rng.standard_normal((4 * 5 * 2, 2))
    out["lm_vt"] = vt
    out["lm_yt"] = MatrixFree.apply(mats, vt, is_transpose=True)
    np.savez_compressed(HERE / "matvec.npz", **out)


def fd_fixtures():
    out = {}
    q = make_rule("gauss", 3, 4)
    rules = [q] * 3
    table = np.zeros((1, 3, 2), dtype=bool)
    table[0, 0, 0] = True
    table[0, 2, 1] = True
    fd = SingleFD("spatial")
    fd.compute_space_eigendecomposition(rules, table)
    fd.add_scalar_space_time_correctors(stiffness_corrector=[np.array([3.0, 2.0, 5.0])])
    fd.update_space_eigenvalues(scalar_coefs=(0.5, 1.0))
    spfd = fd.space_preconditioner
    out["table"] = table
    out["corr"] = np.array([3.0, 2.0, 5.0])
    out["scalar_coefs"] = np.array([0.5, 1.0])
    for d in range(3):
        out[f"U{d}"] = spfd.eigenvec_by_dir_space[0][d]
        out[f"lam{d}"] = spfd.eigenval_by_dir_space[0][d]
    out["eig"] = spfd.space_eigenvalues[0]
    out["free"] = np.asarray(spfd.space_free_nodes[0])
    rng = np.random.default_rng(0)
    v = rng.random(spfd.sp_nnz)
    V = rng.random((spfd.sp_nnz, 2))
    out["v"], out["Pv"] = v, fd.apply(v)
    out["V"], out["PV"] = V, fd.apply(V)
    # WQ input rules are rewritten to Gauss by the FD setup
    w = make_rule("wq2", 3, 5)
    fd2 = SingleFD("spatial")
    table2 = np.ones((1, 2, 2), dtype=bool)
    fd2.compute_space_eigendecomposition([w, w], table2)
    v2 = rng.standard_normal(w.nbctrlpts ** 2)
    out["wq_v"], out["wq_Pv"] = v2, fd2.apply(v2)
    pack_rule("wq_rule", w, out)
    out["kron_idx"] = np.asarray(KronProduct.kron_nonzero_indices([[0, 2], [1, 3], [0, 1]], [4, 4, 3]))
    out["comb"] = combine_arrays([np.array([1.0, 2.0]), np.array([3.0, 4.0, 5.0])], np.array([2.0, 0.5]))
    np.savez_compressed(HERE / "fastdiag.npz", **out)


def solver_fixtures():
    out = {}
    # 2D Poisson on the unit square, WQ type 2, all sides Dirichlet, FD-GMRES
    q = make_rule("wq2", 3, 8)
    rules = [q, q]
    nq = q.nbquadpts ** 2
    coefs = np.zeros((2, 2, nq))
    coefs[0, 0] = coefs[1, 1] = 1.0
    rng = np.random.default_rng(0)
    coefs[0, 1] = coefs[1, 0] = 0.2 * rng.random(nq)
    fd = SingleFD("spatial")
    fd.compute_space_eigendecomposition(rules, np.ones((1, 2, 2), dtype=bool))
    free = np.asarray(fd.space_preconditioner.space_free_nodes[0])
    N = q.nbctrlpts ** 2

    def A(x):
        full = np.zeros(N)
        full[free] = x
        return BsplineOperations.compute_mf_scalar_gradu_gradv(rules, coefs, full)[free]

    def P(x):
        full = np.zeros(N)
        full[free] = x
        return fd.apply(full)[free]

    b = rng.uniform(-1, 1, len(free))
    for tol in (1e-6, 1e-10):
        ls = LinearSolver(tol, 100, linear_type="gmres", verbose=False)
        o = ls.solve(A, b, P)
        out[f"gm_x_{tol:g}"] = o.solution
        out[f"gm_res_{tol:g}"] = o.residual
    ls = LinearSolver(1e-10, 200, linear_type="gmres", verbose=False)
    o = ls.solve(A, b)
    out["gm_x_noprec"], out["gm_res_noprec"] = o.solution, o.residual
    pack_rule("gm_rule", q, out)
    out["gm_coefs"], out["gm_b"], out["gm_free"] = coefs, b, free
    # mask + x0 on a tridiagonal system
    n = 60
    T = np.diag(np.full(n, 2.05)) + np.diag(np.full(n - 1, -1.0), 1) + np.diag(np.full(n - 1, -1.0), -1)
    bt = rng.standard_normal(n)
    x0 = rng.standard_normal(n)
    mask = [0, 5, n - 1]
    ls = LinearSolver(1e-9, 100, cleandod=list(mask), linear_type="gmres", verbose=False)
    o = ls.solve(lambda v: T @ v, bt, x0=x0)
    out["tri_T"], out["tri_b"], out["tri_x0"], out["tri_mask"] = T, bt, x0, np.asarray(mask)
    out["tri_x"], out["tri_res"] = o.solution, o.residual
    # GCRO-DR, two recycled solves
    n = 300
    T = np.diag(np.full(n, 2.05)) + np.diag(np.full(n - 1, -1.0), 1) + np.diag(np.full(n - 1, -1.0), -1)
    e0 = np.zeros(n)
    e0[0] = 1.0
    rhs = T @ e0
    g = GCRODR(tolerance=1e-8, maxiters=2000, krylov_size=30, recycled_size=10, verbose=False)
    o1 = g.solve(lambda v: T @ v, rhs)
    o2 = g.solve(lambda v: T @ v, 0.5 * rhs + 0.1)
    out["gc_T"] = T
    out["gc_rhs"] = rhs
    out["gc_x1"], out["gc_res1"] = o1.solution, o1.residual
    out["gc_x2"], out["gc_res2"] = o2.solution, o2.residual
    np.savez_compressed(HERE / "solvers.npz", **out)


def geometry_fixtures():
    out = {}
    q = make_rule("wq2", 2, 3)
    rules = [q] * 3
    g = GeometryOps.evaluate_greville(q.degree, q.knotvector)
    G3, G2, G1 = np.meshgrid(g, g, g, indexing="ij")
    X = np.stack([G1.ravel(), G2.ravel(), G3.ravel()])
    disp = 0.1 / 3 * np.sin(2 * np.pi * X[0]) * np.sin(2 * np.pi * X[1]) * np.sin(2 * np.pi * X[2])
    ctrl = X + disp[None, :]
    spl = SingleSpline(ctrl, np.array([]), rules).evaluate_spline()
    out["ctrlpts"] = ctrl
    out["jac"], out["det_jac"], out["inv_jac"], out["qp_phy"] = spl.jac, spl.det_jac, spl.inv_jac, spl.qp_phy
    pack_rule("rule", q, out)
    np.savez_compressed(HERE / "geometry.npz", **out)


def nurbs_fixtures():
    """NurbsOperations (rational operators and evaluations) on random positive
    control weights."""
    from igaops.operators import NurbsOperations

    out = {}
    cases = [
        ("2d", [("wq2", 3, 5)] * 2, None),
        ("3d", [("wq2", 2, 3)] * 3, None),
        ("3g", [("gauss", 2, 3)] * 3, None),
        ("st", [("wq2", 2, 3), ("wq2", 2, 3), ("wq2", 2, 2)], (0, 1)),
    ]
    names = []
    for ci, (name, spec, td) in enumerate(cases):
        rng = np.random.default_rng(300 + ci)
        rules = [make_rule(k, p, ne) for k, p, ne in spec]
        for d, q in enumerate(rules):
            pack_rule(f"{name}_r{d}", q, out)
        ndim = len(rules)
        sp_ndim = ndim - 1 if td is not None else ndim
        N = int(np.prod([q.nbctrlpts for q in rules]))
        nq = int(np.prod([q.nbquadpts for q in rules]))
        w = 0.7 + 0.6 * rng.random(N)
        x = rng.standard_normal(N)
        out[f"{name}_w"] = w
        out[f"{name}_x"] = x
        for op in ("u_v", "gradu_gradv", "gradu_v", "u_gradv"):
            c = coef_for(op, sp_ndim, nq, rng)
            out[f"{name}_{op}_c"] = c
            fn = getattr(NurbsOperations, f"compute_mf_scalar_{op}")
            out[f"{name}_{op}_y"] = fn(rules, c, x, time_ders=td, nurbs_weights=w)
        if td is None:
            X = rng.standard_normal((N, 2))
            out[f"{name}_X"] = X
            out[f"{name}_gradu_gradv_Y"] = NurbsOperations.compute_mf_scalar_gradu_gradv(
                rules, out[f"{name}_gradu_gradv_c"], X, nurbs_weights=w)
            # evaluations on Gauss bases carrying second derivatives
            kvs = [q.knotvector for q in rules]
            g2 = [StandardGauss(q.degree, kv, "legendre", nders=2) for q, kv in zip(rules, kvs)]
            for d, q in enumerate(g2):
                pack_rule(f"{name}_g{d}", q, out)
            u = rng.standard_normal((2, N))
            basis = [q.basis for q in g2]
            out[f"{name}_u"] = u
            out[f"{name}_interp"] = NurbsOperations.eval_interpolation(basis, u, nurbs_weights=w)
            out[f"{name}_jac"] = NurbsOperations.eval_jacobien(basis, u, nurbs_weights=w)
            out[f"{name}_hess"] = NurbsOperations.eval_hessian(basis, u, nurbs_weights=w)
        out[f"{name}_td"] = np.asarray(td if td is not None else (-1, -1))
        names.append(name)
    out["names"] = np.asarray(names)
    np.savez_compressed(HERE / "nurbs.npz", **out)


def sptime_fixtures():
    """Space-time arrowhead FD (2D space + time) of the reference."""
    out = {}
    qs = make_rule("wq2", 2, 4)
    qt = make_rule("wq2", 2, 5)
    table = np.ones((1, 2, 2), dtype=bool)
    table[0, 1, 1] = False
    pack_rule("space", qs, out)
    pack_rule("time", qt, out)
    out["table"] = table
    rng = np.random.default_rng(11)
    N = qs.nbctrlpts ** 2 * qt.nbctrlpts
    for tag, adv in (("a1", None), ("a07", 0.7)):
        fd = SingleFD("spacetime")
        fd.compute_space_eigendecomposition([qs, qs], table)
        fd.compute_time_schurdecomposition(qt)
        fd.update_space_eigenvalues(scalar_coefs=(0.25, 1.0))
        if adv is not None:
            fd.add_scalar_space_time_correctors(advection_corrector=[adv])
        v = rng.standard_normal(N)
        V = rng.standard_normal((N, 2))
        out[f"{tag}_v"], out[f"{tag}_Pv"] = v, fd.apply(v)
        out[f"{tag}_V"], out[f"{tag}_PV"] = V, fd.apply(V)
        out[f"{tag}_PTv"] = fd.apply_transpose(v)
    out["free"] = np.asarray(fd.sptm_preconditioner.sptm_free_nodes[0])
    # the QZ ("legacy") form: compute_time_schurdecomposition(use_arrowhead=False)
    for tag, adv in (("l1", None), ("l07", 0.7)):
        fd = SingleFD("spacetime")
        fd.compute_space_eigendecomposition([qs, qs], table)
        fd.compute_time_schurdecomposition(qt, use_arrowhead=False)
        fd.update_space_eigenvalues(scalar_coefs=(0.25, 1.0))
        if adv is not None:
            fd.add_scalar_space_time_correctors(advection_corrector=[adv])
        v = rng.standard_normal(N)
        V = rng.standard_normal((N, 2))
        out[f"{tag}_v"], out[f"{tag}_Pv"] = v, fd.apply(v)
        out[f"{tag}_V"], out[f"{tag}_PV"] = V, fd.apply(V)
        out[f"{tag}_PTv"] = fd.apply_transpose(v)
    np.savez_compressed(HERE / "sptime.npz", **out)


def bench_rule_fixtures():
    """The 1D rule of the benchmark configuration (weighted quadrature type
    "2", endpoint points, degree 3, 128 elements) as the reference builds it:
    the CPU legs of bench.py run the oracle on these factors so that they
    never load this package."""
    out = {}
    pack_rule("wq2_p3_ne128", make_rule("wq2", 3, 128), out)
    np.savez_compressed(HERE / "bench_rule.npz", **out)


FIXTURES = {
    "quadrature": lambda: quadrature_fixtures(),
    "matvec": lambda: matvec_fixtures(),
    "fastdiag": lambda: fd_fixtures(),
    "solvers": lambda: solver_fixtures(),
    "geometry": lambda: geometry_fixtures(),
    "nurbs": lambda: nurbs_fixtures(),
    "sptime": lambda: sptime_fixtures(),
    "bench_rule": lambda: bench_rule_fixtures(),
}


if __name__ == "__main__":
    # python make_golden.py [reference_dir] [fixture ...]   (default: all)
    for name in (sys.argv[2:] or list(FIXTURES)):
        FIXTURES[name]()
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size)
