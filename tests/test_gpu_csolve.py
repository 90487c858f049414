"""iga_gmres_solve, the solve-level C entry point, called through the C ABI
(ctypes) with C callbacks built from the library's own fused matvec
(iga_mf_matvec) and FP64 fast-diagonalisation apply (iga_fd_apply), as a C
caller would: the solution reaches the tolerance by the oracle's operator,
its residual history equals the Python GMRES path's (same Gram-Schmidt
passes), and the status codes of non-convergence, non-finite input and a
failing callback come back as the header states."""
import ctypes

import numpy as np
import pytest
import torch

from oracle import mf as omf
from tests._problems import rules

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problem(cuda):
    from igaops_b200 import MFOperator, precompute_coefficients, unit_cube_ctrlpts
    from igaops_b200.fastdiag import SingleFD

    rl = rules(3, 3, 8)
    co = precompute_coefficients(rl, unit_cube_ctrlpts(rl, amplitude=0.08), mass=False)
    op = MFOperator(rl, co["stiffness"], "gradu_gradv")
    fd = SingleFD("spatial")
    fd.compute_space_eigendecomposition(rl, np.ones((1, 3, 2), dtype=bool))
    sp = fd.space_preconditioner
    free = np.asarray(sp.space_free_nodes[0], dtype=np.int64)
    mask = np.ones(op.N, dtype=bool)
    mask[free] = False
    dirichlet = np.flatnonzero(mask)
    rng = np.random.default_rng(3)
    b = np.zeros(op.N)
    b[free] = rng.uniform(-1.0, 1.0, free.size)
    return rl, co["stiffness"].cpu().numpy(), op, sp, free, dirichlet, b


def _callbacks(op, sp):
    from igaops_b200 import _lib

    U, inv = sp.device_data(torch.float64)[0]
    lo, mm = sp._boxes[0]
    n = [sp._nonzeros_by_dir[d] for d in sp._space_dirs]
    M = int(np.prod(mm))
    w0 = torch.empty(M, dtype=torch.float64, device="cuda")
    w1 = torch.empty(M, dtype=torch.float64, device="cuda")
    arr = ctypes.c_int32 * 3
    ptrs = (ctypes.c_void_p * 3)(*[u.data_ptr() for u in U])
    keep = [U, inv, w0, w1, ptrs]

    def A(user, x, y, stream):
        return _lib.LIB.iga_mf_matvec(ctypes.byref(op.plan.P), _lib.IGA_F64, op.packed.data_ptr(),
                                      1, x, y, stream)

    def P(user, x, y, stream):
        return _lib.LIB.iga_fd_apply(_lib.IGA_F64, 3, arr(*n), arr(*lo), arr(*mm), ptrs,
                                     inv.data_ptr(), 1, x, y, w0.data_ptr(), w1.data_ptr(), stream)

    return _lib.APPLY_FN(A), _lib.APPLY_FN(P), keep


def _solve(op, sp, dirichlet, b, tol=1e-10, maxiters=40, A=None, P=None):
    from igaops_b200 import _lib
    from igaops_b200._device import stream_handle

    cA, cP, keep = _callbacks(op, sp)
    A = A or cA
    P = P or cP
    n = b.size
    elems = ctypes.c_int64(0)
    assert _lib.LIB.iga_gmres_workspace(n, maxiters, ctypes.byref(elems)) == 0
    work = torch.empty(int(elems.value), dtype=torch.float64, device="cuda")
    bd = torch.from_numpy(b).cuda()
    xd = torch.empty_like(bd)
    di = torch.from_numpy(dirichlet).cuda()
    hist = np.zeros(maxiters + 1)
    its = ctypes.c_int(0)
    rc = _lib.LIB.iga_gmres_solve(n, bd.data_ptr(), xd.data_ptr(), tol, maxiters, A, P, None,
                                  di.data_ptr(), di.numel(), work.data_ptr(), work.numel(),
                                  hist.ctypes.data_as(ctypes.c_void_p), ctypes.byref(its),
                                  stream_handle())
    torch.cuda.synchronize()
    return rc, xd.cpu().numpy(), hist[: its.value + 1], its.value, keep


def test_c_gmres_reaches_tolerance_and_matches_python_path(problem):
    from igaops_b200.solvers import LinearSolver

    rl, C, op, sp, free, dirichlet, b = problem
    rc, x, hist, its, _ = _solve(op, sp, dirichlet, b)
    assert rc == 0 and its >= 1
    r = b - omf.mf_gradu_gradv(rl, C, x)
    assert np.linalg.norm(r[free]) / np.linalg.norm(b[free]) < 1e-10
    assert np.all(x[dirichlet] == 0.0)

    def A(v):
        y = torch.empty_like(v)
        op.apply_into(v, y)
        return y

    def P(v):
        y = torch.empty_like(v)
        sp.apply_device(v, y)
        return y

    out = LinearSolver(1e-10, 40, cleandod=[int(i) for i in dirichlet], verbose=False).solve(
        A, b, P)
    k = min(len(hist), len(out.residual))
    assert np.allclose(hist[:k], out.residual[:k], rtol=1e-6, atol=1e-13)
    assert np.linalg.norm(x - out.solution) / np.linalg.norm(out.solution) < 1e-8


def test_c_gmres_status_codes(problem):
    from igaops_b200 import _lib

    rl, C, op, sp, free, dirichlet, b = problem
    rc, x, hist, its, _ = _solve(op, sp, dirichlet, b, maxiters=2)
    assert rc == _lib.IGA_ERR_NOT_CONVERGED and its == 2 and np.all(np.isfinite(x))
    bad = b.copy()
    bad[free[0]] = np.nan
    rc, *_ = _solve(op, sp, dirichlet, bad)
    assert rc == _lib.IGA_ERR_NONFINITE

    def failing(user, x, y, stream):
        return _lib.IGA_ERR_INVALID_ARG

    rc, *_ = _solve(op, sp, dirichlet, b, A=_lib.APPLY_FN(failing))
    assert rc == _lib.IGA_ERR_INVALID_ARG
