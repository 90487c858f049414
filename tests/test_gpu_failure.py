"""Failure handling on the GPU path, made on the host or by a test hook that
withholds a copy (no fault, trap or hang of the GPU):

* non-finite input: a NaN / Inf right-hand side, or an operator that starts
  returning NaN, ends a solve with NonFiniteError (IGA_ERR_NONFINITE), never
  a hang or a garbage solution;
* non-convergence is a result, not an exception (success=False and a
  warning, src/igaops/solvers/linear_solver.py:518-521,
  src/igaops/solvers/deflated/gcrodr.py:365-367);
* Arnoldi breakdown (norm_w == 0, linear_solver.py:494) finishes the solve;
* the serving loop refuses an over-budget or non-finite request at submit
  and drops a cancelled one (queued or active) while the others converge;
* a bounded device wait that runs out: the fused matvec's test hook
  withholds the first coefficient copy of every CTA, the launch reports
  IGA_ERR_TIMEOUT (DeviceTimeoutError) after draining the copies it issued,
  and the next normal launch gives the oracle's product.
"""
import warnings

import numpy as np
import pytest
import torch

from oracle import mf as omf
from tests._problems import coefficients, rel_err, rules

pytestmark = pytest.mark.gpu


def _tridiag(n=200):
    T = np.diag(np.full(n, 2.5)) + np.diag(np.full(n - 1, -1.0), 1) + np.diag(np.full(n - 1, -1.0), -1)
    Td = torch.as_tensor(T, device="cuda")
    return T, (lambda v: Td @ v)


@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_nonfinite_rhs_is_refused(cuda, bad):
    from igaops_b200._lib import NonFiniteError
    from igaops_b200.solvers import LinearSolver

    T, A = _tridiag()
    b = np.ones(T.shape[0])
    b[7] = bad
    for kind in ("gmres", "cg", "bicgstab"):
        with pytest.raises(NonFiniteError):
            LinearSolver(1e-10, 50, linear_type=kind, verbose=False).solve(A, b)


def test_operator_turning_nonfinite_is_refused(cuda):
    from igaops_b200._lib import NonFiniteError
    from igaops_b200.solvers import LinearSolver

    T, A = _tridiag()
    calls = {"n": 0}

    def A_bad(v):
        calls["n"] += 1
        y = A(v)
        if calls["n"] == 3:
            y[5] = float("nan")
        return y

    with pytest.raises(NonFiniteError):
        LinearSolver(1e-12, 50, verbose=False).solve(A_bad, np.ones(T.shape[0]))
    assert calls["n"] == 3  # stopped at the first non-finite iterate


def test_iteration_limit_gives_success_false(cuda):
    from igaops_b200.solvers import GCRODR, LinearSolver

    T, A = _tridiag(400)
    b = np.random.default_rng(0).standard_normal(T.shape[0])
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        out = LinearSolver(1e-12, 3, verbose=False).solve(A, b)
    assert not out.success and len(out.residual) == 4
    assert any("No convergence" in str(x.message) for x in w)
    g = GCRODR(1e-12, 2000, krylov_size=4, recycled_size=2, max_cycles=2, verbose=False)
    assert not g.solve(A, b).success


def test_arnoldi_breakdown_finishes_the_solve(cuda):
    from igaops_b200.solvers import LinearSolver

    n = 64
    b = np.zeros(n)
    b[5] = 3.0
    # P = A^-1 and b a coordinate vector: the first Arnoldi vector spans an
    # invariant space and the projected vector is exactly zero (norm_w = 0)
    out = LinearSolver(1e-10, 20, verbose=False).solve(lambda v: 2.0 * v, b, lambda v: 0.5 * v)
    assert out.success and len(out.residual) == 2
    assert np.all(np.isfinite(out.solution))
    assert rel_err(out.solution, 0.5 * b) < 1e-14


def test_refined_and_batched_solves_refuse_nonfinite_rhs(cuda):
    from igaops_b200 import precompute_coefficients, unit_cube_ctrlpts
    from igaops_b200._lib import NonFiniteError
    from igaops_b200.batch import BatchedFGMRES, PatchBatch
    from igaops_b200.refine import EllipticPatchSolver

    rl = rules(3, 2, 6)
    co = precompute_coefficients(rl, unit_cube_ctrlpts(rl, amplitude=0.05))
    S = EllipticPatchSolver(rl, co["stiffness"], np.ones((1, 3, 2), dtype=bool))
    b = np.zeros(S.N)
    b[S.free] = 1.0
    b[S.free[3]] = np.nan
    with pytest.raises(NonFiniteError):
        S.solve_mixed(b)
    with pytest.raises(NonFiniteError):
        S.solve_mixed(b, precond="fp")
    B = PatchBatch([(rl, co["stiffness"], np.ones((1, 3, 2), dtype=bool))])
    with pytest.raises(NonFiniteError):
        BatchedFGMRES(B, tolerance=1e-10).solve(B.join([b]))


def _server_requests(n=4):
    from igaops_b200 import precompute_coefficients, unit_cube_ctrlpts
    from igaops_b200.serve import SolveRequest

    reqs = []
    for rid in range(n):
        rl = rules(3, 2, 6 + rid)
        co = precompute_coefficients(rl, unit_cube_ctrlpts(rl, amplitude=0.05))
        N = int(np.prod([q.nbctrlpts for q in rl]))
        rhs = np.random.default_rng(rid).uniform(-1, 1, N)
        reqs.append(SolveRequest(rid, "3d", rl, co["stiffness"], np.ones((1, 3, 2), dtype=bool),
                                 rhs, 1e-10, 0.0))
    return reqs


def test_server_refuses_and_cancels(cuda):
    from igaops_b200._lib import NonFiniteError
    from igaops_b200.serve import SolveServer

    reqs = _server_requests(4)
    small = SolveServer(hbm_budget_bytes=1 << 20)
    with pytest.raises(ValueError, match="budget"):
        small.submit(reqs[0])
    srv = SolveServer(hbm_budget_bytes=4 << 30, max_active=8, restart=2)
    bad = _server_requests(1)[0]
    bad.rid = 99
    bad.rhs = bad.rhs.copy()
    bad.rhs[0] = np.inf
    with pytest.raises(NonFiniteError):
        srv.submit(bad)
    for r in reqs:
        srv.submit(r)
    srv.cancel(0)  # still queued

    state = {"sent": False}

    def on_round(s):
        # cancel request 2 once it is active and has run a cycle (3D
        # requests join the rounds when their set-up is complete)
        if not state["sent"] and any(a.req.rid == 2 and a.req.cycles >= 1 for a in s.active):
            s.cancel(2)
            state["sent"] = True

    done = srv.run(on_round=on_round)
    by = {r.rid: r for r in done}
    assert set(by) == {0, 1, 2, 3}
    assert by[0].cancelled and not by[0].success
    assert by[2].cancelled and not by[2].success and by[2].cycles >= 1
    assert srv.in_use == 0
    for rid in (1, 3):
        r = by[rid]
        assert r.success and not r.cancelled
        C = r.coefs.cpu().numpy()
        res = r.rhs - omf.mf_gradu_gradv(r.rules, C, r.solution)
        free = np.flatnonzero(r.solution != 0.0)
        assert np.linalg.norm(res[free]) / np.linalg.norm(r.rhs[free]) < 1e-9


def test_device_wait_timeout_is_reported_and_recovered(cuda):
    from igaops_b200 import MFOperator
    from igaops_b200._lib import DeviceTimeoutError

    rl = rules(3, 3, 6)
    rng = np.random.default_rng(5)
    c = coefficients("gradu_gradv", rl, rng)
    x = rng.standard_normal(int(np.prod([q.nbctrlpts for q in rl])))
    op = MFOperator(rl, c, "gradu_gradv")
    assert op.fused and not op.tiled
    xd = torch.from_numpy(x).cuda()
    op.plan.P.wait_test = 1
    op.apply(xd)
    torch.cuda.synchronize()
    with pytest.raises(DeviceTimeoutError):
        op.plan.check_status()
    op.plan.P.wait_test = 0
    got = op.apply(xd).cpu().numpy()
    op.plan.check_status()
    assert rel_err(got, omf.mf_gradu_gradv(rl, c, x)) < 1e-12
