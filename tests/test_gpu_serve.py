"""Continuous batching: requests of different sizes and kinds (3D, 2D,
space-time 2D+1) arriving over time are served with their state on the
device; every result reaches its tolerance (true relative residual, FP64 --
recomputed here with the oracle's operator for the 3D requests) and is the
same alone and in the mix."""
import numpy as np
import pytest
import torch

from oracle import mf as omf
from tests._problems import rules

pytestmark = pytest.mark.gpu


def _requests():
    from igaops_b200 import precompute_coefficients, unit_cube_ctrlpts
    from igaops_b200.serve import SolveRequest

    reqs = []
    specs = [("3d", 2, 7, 0.0), ("3d", 3, 9, 0.002), ("2d", 3, 24, 0.004), ("3d", 4, 6, 0.006),
             ("spacetime", 2, 8, 0.008), ("3d", 2, 12, 0.01)]
    for rid, (kind, p, ne, t) in enumerate(specs):
        rng = np.random.default_rng(rid)
        if kind == "spacetime":
            rl = rules(3, p, [ne, ne, ne - 2])
            Nq = int(np.prod([q.nbquadpts for q in rl]))
            C = np.zeros((2, 2, Nq))
            C[0, 0] = C[1, 1] = 1.0
            req = SolveRequest(rid, kind, rl, C, np.ones((1, 2, 2), dtype=bool), None, 1e-10, t,
                               mass_coefs=np.ones(Nq))
        else:
            d = 3 if kind == "3d" else 2
            rl = rules(d, p, ne)
            co = precompute_coefficients(rl, unit_cube_ctrlpts(rl, amplitude=0.08))
            req = SolveRequest(rid, kind, rl, co["stiffness"], np.ones((1, d, 2), dtype=bool),
                               None, 1e-10 if rid % 2 else 1e-9, t)
        N = int(np.prod([q.nbctrlpts for q in req.rules]))
        req.rhs = rng.uniform(-1.0, 1.0, N)
        reqs.append(req)
    return reqs


def _serve(reqs):
    from igaops_b200.serve import SolveServer

    srv = SolveServer(hbm_budget_bytes=8 << 30, max_active=8, restart=6)
    for r in reqs:
        srv.submit(r)
    return srv.run(), srv


def test_serving_converges_and_alone_equals_mix(cuda):
    import copy

    from igaops_b200.serve import SolveServer

    import sys

    reqs = _requests()
    before = sys.getswitchinterval()
    done, srv = _serve(reqs)
    # run() shortens the interpreter's switch interval only while it runs
    assert sys.getswitchinterval() == before
    st = SolveServer.stats(done)
    assert st["requests"] == len(reqs) and st["all_converged"], st
    by_id = {r.rid: r for r in done}
    for r in done:
        assert r.true_residual < r.tol
        if r.kind == "3d":
            C = r.coefs.cpu().numpy() if isinstance(r.coefs, torch.Tensor) else r.coefs
            b = r.rhs.copy()
            free = np.ones(b.size, dtype=bool)
            # Dirichlet rows: every face
            n = [q.nbctrlpts for q in r.rules]
            idx = np.indices(n[::-1]).reshape(3, -1)
            for d in range(3):
                free &= (idx[2 - d] > 0) & (idx[2 - d] < n[d] - 1)
            res = b - omf.mf_gradu_gradv(r.rules, C, r.solution)
            assert np.linalg.norm(res[free]) / np.linalg.norm(b[free]) < r.tol
            assert np.all(r.solution[~free] == 0.0)
    # each request alone
    for rid in (1, 2, 4):
        alone = copy.copy(reqs[rid])
        alone.arrival = 0.0
        alone.solution, alone.success, alone.cycles = None, False, 0
        d2, _ = _serve([alone])
        x_mix, x_alone = by_id[rid].solution, d2[0].solution
        assert np.linalg.norm(x_mix - x_alone) / np.linalg.norm(x_alone) < 1e-8


def test_warmup_leaves_no_trace(cuda):
    """warmup() runs one small request per kind and degree through the loop
    and resets it: nothing in done, no rounds counted, no memory booked;
    the stream served afterwards converges as usual."""
    from igaops_b200.serve import SolveServer

    srv = SolveServer(hbm_budget_bytes=8 << 30, max_active=8, restart=6)
    t = srv.warmup(degrees=(2, 3))
    assert t > 0 and srv.done == [] and srv.rounds == 0 and srv.in_use == 0
    assert not srv.queue and not srv.active
    reqs = _requests()
    for r in reqs:
        srv.submit(r)
    done = srv.run()
    st = SolveServer.stats(done)
    assert st["requests"] == len(reqs) and st["all_converged"], st


def test_graph_capture_beside_setup_threads(cuda):
    """The 3D rounds capture their Arnoldi steps as CUDA graphs while the
    set-up and 2D threads allocate and copy: the capture is thread-local,
    so those threads' calls do not invalidate it (with capture mode
    "global" they did). Two set-up threads and two passes over the request
    mix make the overlap likely; every request converges."""
    from igaops_b200.serve import SolveServer

    srv = SolveServer(hbm_budget_bytes=8 << 30, max_active=8, restart=2, use_graphs=True,
                      prep_threads=2)
    for rnd in range(2):
        reqs = _requests()
        for r in reqs:
            r.rid += 100 * rnd
            srv.submit(r)
        done = srv.run()
        st = SolveServer.stats(done)
        assert st["requests"] == len(reqs) * (rnd + 1) and st["all_converged"], st
