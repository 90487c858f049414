"""Mixed-precision solves: an FP64 flexible GMRES (FGMRES) outer loop around
a low-precision inner solve.

The reference solves A x = b with right-preconditioned GMRES in FP64
(src/igaops/solvers/linear_solver.py:438-525, storing Z = P V, which is the
flexible form).  Here the preconditioner slot of that same outer iteration
holds an *inner solve* in FP32: ``inner_iters`` GMRES iterations on the FP32
operator with the fast-diagonalisation preconditioner applied by the BF16
tensor-core kernel (FP32 accumulation), or, with ``inner_iters = 0``, the
BF16/FP32 preconditioner alone.  FP64 is kept where accuracy is decided: the
outer Arnoldi basis and its two Gram-Schmidt passes, the Hessenberg least
squares, the outer matvec ``A z`` and the final true residual ``b - A x``
(or, with ``residual="arnoldi"``, the FP64 Arnoldi residual estimate the
reference's GMRES stops on).
Because the outer loop is flexible, the low-precision inner result only
changes the search directions, and the iteration converges to the FP64
tolerance (iterative refinement in its FGMRES form).

All vector work runs in libigab200 kernels (gram, combine, scale, convert);
inside an Arnoldi cycle nothing waits for the host: projections, norms and
the Hessenberg matrix stay on the device, and the host reads the small
Hessenberg once per outer iteration / inner solve.
"""
from __future__ import annotations

import math
import warnings
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np
import torch
from numpy.linalg import lstsq

from . import _lib
from . import krylov_ops as K
from .batch import RESIDUAL_KINDS
from .solvers import _require_finite
from ._device import iga_dtype, require_cuda, stream_handle, to_device

__all__ = ["MixedPrecisionFGMRES", "RefinedOutput", "EllipticPatchSolver"]


def _gram_into(ws: K.Workspace, A: torch.Tensor, B: torch.Tensor, out: torch.Tensor):
    """out[j1 * m2 + j2] = A_j1 . B_j2 (FP64, on the device, no host sync)."""
    if A.ndim == 1:
        A = A.unsqueeze(0)
    if B.ndim == 1:
        B = B.unsqueeze(0)
    m1, n = A.shape
    m2 = B.shape[0]
    nblk = ws.ensure(n, m1, m2, 0)
    _lib.check(_lib.LIB.iga_gram(iga_dtype(A.dtype), 0, n, m1, A.data_ptr(), A.stride(0), m2,
                                 B.data_ptr(), B.stride(0), out.data_ptr(), ws.partial.data_ptr(),
                                 nblk, stream_handle()))


def _normalize(x: torch.Tensor, sq: torch.Tensor):
    """x /= sqrt(sq[0]) with sq on the device."""
    _lib.check(_lib.LIB.iga_scale_dev(iga_dtype(x.dtype), 0, x.numel(), x.data_ptr(),
                                      sq.data_ptr(), 2, stream_handle()))


def _convert(src: torch.Tensor, dst: torch.Tensor):
    _lib.check(_lib.LIB.iga_convert(iga_dtype(src.dtype), iga_dtype(dst.dtype), src.numel(),
                                    src.data_ptr(), dst.data_ptr(), stream_handle()))


class _Arnoldi:
    """Arnoldi process with two classical Gram-Schmidt passes (the two
    projection passes of linear_solver.py:481-490) whose projections,
    norms and Hessenberg entries stay on the device."""

    def __init__(self, n: int, m: int, dtype: torch.dtype, device):
        self.n, self.m = n, m
        self.V = torch.empty((m + 1, n), dtype=dtype, device=device)
        self.Z = torch.empty((m, n), dtype=dtype, device=device)
        # row j: h[0..j] of column j, then the squared norm of the new vector
        self.H = torch.zeros((m, m + 1), dtype=torch.float64, device=device)
        self.h2 = torch.zeros(m + 1, dtype=torch.float64, device=device)
        self.beta2 = torch.zeros(1, dtype=torch.float64, device=device)
        self.ws = K.Workspace(device)
        self.ws.ensure(n, m + 1, 1, 0)

    def start(self, r: torch.Tensor):
        _gram_into(self.ws, r, r, self.beta2)
        K.copy(r, self.V[0])
        _normalize(self.V[0], self.beta2)

    def step(self, j: int, A_into: Callable, P_into: Callable):
        V, w = self.V, self.V[j + 1]
        P_into(V[j], self.Z[j])
        A_into(self.Z[j], w)
        hj = self.H[j, : j + 1]
        _gram_into(self.ws, V[: j + 1], w, hj)
        K.combine(V[: j + 1], hj.reshape(j + 1, 1), w, alpha=-1.0, beta=1.0)
        h2 = self.h2[: j + 1]
        _gram_into(self.ws, V[: j + 1], w, h2)
        K.combine(V[: j + 1], h2.reshape(j + 1, 1), w, alpha=-1.0, beta=1.0)
        _lib.check(_lib.LIB.iga_axpby(_lib.IGA_F64, j + 1, 1.0, h2.data_ptr(), 1.0, hj.data_ptr(),
                                      stream_handle()))
        _gram_into(self.ws, w, w, self.H[j, j + 1: j + 2])
        _normalize(w, self.H[j, j + 1: j + 2])

    def host(self, k: int):
        """(beta, Hessenberg (k+1, k)) on the host: one device->host copy."""
        Hh = torch.cat([self.beta2, self.H[:k].reshape(-1)]).cpu().numpy()
        beta = math.sqrt(max(Hh[0], 0.0))
        Hr = Hh[1:].reshape(k, self.m + 1)
        Hm = np.zeros((k + 1, k))
        for j in range(k):
            Hm[: j + 1, j] = Hr[j, : j + 1]
            Hm[j + 1, j] = math.sqrt(max(Hr[j, j + 1], 0.0))
        return beta, Hm


@dataclass
class RefinedOutput:
    """Result of a refined solve (OutputArgs of the reference plus counters).
    true_residual: relative residual of the returned solution, recomputed as
    ||b - A x|| / ||b|| in FP64 when residual_kind is "true", the FP64
    Arnoldi residual estimate when it is "arnoldi"."""

    solution: object
    residual: np.ndarray
    success: bool
    true_residual: float = float("nan")
    residual_kind: str = "true"
    outer_iterations: int = 0
    inner_iterations: int = 0
    fp64_matvecs: int = 0
    low_matvecs: int = 0
    precond_applies: int = 0
    history: list = field(default_factory=list)


class MixedPrecisionFGMRES:
    """FGMRES(m) in FP64 whose preconditioner is an FP32 inner solve.

    ``A64(x, y)``: y = A x in FP64 (device tensors, overwrite y).
    ``A_low(x, y)`` / ``P_low(x, y)``: the operator and the preconditioner in
    the inner precision (FP32 tensors; P_low may run BF16 tensor cores).
    ``cleandod``: indices of Dirichlet DOFs, zeroed in b and in every operator
    output (the masking of linear_solver.py:119-124,213-233).
    Stopping: outer relative residual estimate < tolerance, confirmed by the
    FP64 true residual ||b - A x|| / ||b|| < tolerance (else restart); with
    ``residual="arnoldi"`` a cycle whose FP64 Arnoldi estimate met the
    tolerance ends without the confirming matvec, the stopping rule of the
    reference's GMRES (linear_solver.py:507-521)."""

    def __init__(self, tolerance: float = 1e-10, maxiters: int = 60, restart: int = 30,
                 inner_iters: int = 4, inner_dtype: torch.dtype = torch.float32,
                 residual: str = "true"):
        if not (0 < tolerance < 1):
            raise ValueError("tolerance must lie in (0, 1)")
        if maxiters < 1 or restart < 1 or inner_iters < 0:
            raise ValueError("maxiters and restart must be >= 1, inner_iters >= 0")
        if residual not in RESIDUAL_KINDS:
            raise ValueError(f"residual must be one of {RESIDUAL_KINDS}, got {residual!r}")
        self.residual = residual
        self.tolerance = float(tolerance)
        self.maxiters = int(maxiters)
        self.restart = int(restart)
        self.inner_iters = int(inner_iters)
        self.inner_dtype = inner_dtype
        self._cache = {}

    def _bufs(self, n, device):
        key = (n, str(device))
        if key not in self._cache:
            self._cache = {key: dict(
                outer=_Arnoldi(n, self.restart, torch.float64, device),
                inner=_Arnoldi(n, max(self.inner_iters, 1), self.inner_dtype, device),
                r=torch.empty(n, dtype=torch.float64, device=device),
                v32=torch.empty(n, dtype=self.inner_dtype, device=device),
                z32=torch.empty(n, dtype=self.inner_dtype, device=device),
                nrm=torch.zeros(1, dtype=torch.float64, device=device),
            )}
        return self._cache[key]

    def solve(self, A64: Callable, b, A_low: Callable, P_low: Callable,
              cleandod: Optional[torch.Tensor] = None) -> RefinedOutput:
        dev = require_cuda()
        numpy_in = not isinstance(b, torch.Tensor)
        bd = to_device(b, torch.float64, dev).reshape(-1).clone()
        _require_finite(bd, "right-hand side")
        n = bd.numel()
        mask = None
        if cleandod is not None and len(cleandod) > 0:
            mask = torch.as_tensor(np.asarray(cleandod, dtype=np.int64) if not isinstance(
                cleandod, torch.Tensor) else cleandod, device=dev, dtype=torch.int64)
            K.mask(bd, mask)
        B = self._bufs(n, dev)
        outer, inner = B["outer"], B["inner"]
        out = RefinedOutput(solution=torch.zeros_like(bd), residual=np.array([1.0]), success=False)
        x = out.solution

        def a64(src, dst):
            A64(src, dst)
            out.fp64_matvecs += 1
            if mask is not None:
                K.mask(dst, mask)

        def a_low(src, dst):
            A_low(src, dst)
            out.low_matvecs += 1
            if mask is not None:
                K.mask(dst, mask)

        def p_low(src, dst):
            P_low(src, dst)
            out.precond_applies += 1
            if mask is not None:
                K.mask(dst, mask)

        def precond(v64, z64):
            """z = inner solve of A z = v in the low precision."""
            _convert(v64, B["v32"])
            if self.inner_iters == 0:
                p_low(B["v32"], B["z32"])
            else:
                k = self.inner_iters
                inner.start(B["v32"])
                for j in range(k):
                    inner.step(j, a_low, p_low)
                beta, Hm = inner.host(k)
                rhs = np.zeros(k + 1)
                rhs[0] = beta
                y = lstsq(Hm, rhs, rcond=None)[0]
                K.combine(inner.Z[:k], y.reshape(k, 1), B["z32"])
                out.inner_iterations += k
            _convert(B["z32"], z64)

        r = B["r"]
        K.copy(bd, r)
        _gram_into(outer.ws, bd, bd, B["nrm"])
        b_norm = math.sqrt(max(float(B["nrm"].item()), 0.0))
        if b_norm == 0.0:
            out.success, out.true_residual = True, 0.0
            out.solution = x.cpu().numpy() if numpy_in else x
            return out
        hist = [1.0]
        it = 0
        while it < self.maxiters:
            outer.start(r)
            k_done = 0
            beta, Hm, y = None, None, None
            est = float("inf")
            for j in range(min(self.restart, self.maxiters - it)):
                outer.step(j, a64, precond)
                it += 1
                k_done = j + 1
                beta, Hm = outer.host(k_done)
                rhs = np.zeros(k_done + 1)
                rhs[0] = beta
                y = lstsq(Hm, rhs, rcond=None)[0]
                est = float(np.linalg.norm(rhs - Hm @ y)) / b_norm
                hist.append(est)
                if est < self.tolerance:
                    break
            K.combine(outer.Z[:k_done], y.reshape(k_done, 1), x, alpha=1.0, beta=1.0)
            if self.residual == "arnoldi" and est < self.tolerance:
                out.history.append(est)
                out.residual_kind = "arnoldi"
                out.success = True
                break
            # true residual in FP64
            a64(x, r)
            K.axpby(1.0, bd, -1.0, r)
            _gram_into(outer.ws, r, r, B["nrm"])
            true_rel = math.sqrt(max(float(B["nrm"].item()), 0.0)) / b_norm
            out.history.append(true_rel)
            if true_rel < self.tolerance:
                out.success = True
                break
        out.outer_iterations = it
        out.true_residual = out.history[-1] if out.history else float("nan")
        out.residual = np.asarray(hist)
        if not out.success:
            warnings.warn(f"No convergence after {it} iterations "
                          f"(true relative residual {out.true_residual:.2e}).")
        out.solution = x.cpu().numpy() if numpy_in else x
        return out


class EllipticPatchSolver:
    """Device-resident elliptic problem on one 3D patch -- stiffness operator
    (plus an optional mass shift), homogeneous Dirichlet conditions from a
    boundary table and the fast-diagonalisation preconditioner -- with two
    solve paths on the same inputs:

    * ``solve_fp64``: the plain FP64 GPU path (the reference's FD-preconditioned
      GMRES, linear_solver.py:438-525, with FP64 matvec and FP64 FD apply);
    * ``solve_mixed``: FGMRES(FP64) around the FP32 / BF16 inner solve.
    """

    def __init__(self, quadrule_list, stiffness_coefs, table_dirichlet, mass_coefs=None,
                 mass_scale: float = 0.0, inner_iters: int = 0, restart: int = 30):
        from .fastdiag import SingleFD
        from .operators import MFOperator

        dev = require_cuda()
        rules = list(quadrule_list)
        self.rules = rules
        self.K64 = MFOperator(rules, stiffness_coefs, "gradu_gradv", dtype=torch.float64)
        self.K32 = MFOperator(rules, stiffness_coefs, "gradu_gradv", dtype=torch.float32,
                              symmetric=self.K64.symmetric)
        self.mass_scale = float(mass_scale)
        self.M64 = self.M32 = None
        if mass_coefs is not None and mass_scale != 0.0:
            self.M64 = MFOperator(rules, mass_coefs, "u_v", dtype=torch.float64)
            self.M32 = MFOperator(rules, mass_coefs, "u_v", dtype=torch.float32)
        self.N = self.K64.N
        table = np.asarray(table_dirichlet, dtype=bool)
        self.fd = SingleFD("spatial")
        self.fd.compute_space_eigendecomposition(rules, table)
        self.fd.update_space_eigenvalues([self.mass_scale, 1.0])
        sp = self.fd.space_preconditioner
        self.dirichlet = torch.as_tensor(sp.dirichlet_nodes(0), device=dev)
        self.free = sp.free_nodes(0)
        self._tmp = {}
        self.mixed = MixedPrecisionFGMRES(1e-10, 60, restart, inner_iters)

    def _t(self, dtype):
        t = self._tmp.get(dtype)
        if t is None:
            t = torch.empty(self.N, dtype=dtype, device=self.dirichlet.device)
            self._tmp[dtype] = t
        return t

    def apply(self, x: torch.Tensor, y: torch.Tensor):
        """y = (K + s M) x in the precision of x."""
        K_, M_ = (self.K64, self.M64) if x.dtype == torch.float64 else (self.K32, self.M32)
        K_.apply_into(x, y)
        if M_ is not None:
            t = self._t(x.dtype)
            M_.apply_into(x, t)
            K.axpby(self.mass_scale, t, 1.0, y)

    def precond_tc(self, x: torch.Tensor, y: torch.Tensor):
        self.fd.space_preconditioner.apply_device_tc(x, y)

    def precond_fp(self, x: torch.Tensor, y: torch.Tensor):
        self.fd.space_preconditioner.apply_device(x, y)

    def solve_mixed(self, b, tolerance: float = 1e-10, maxiters: int = 60,
                    precond: str = "tc", residual: str = "true") -> RefinedOutput:
        """Mixed-precision solve.  3D stiffness problems with the tensor-core
        preconditioner run on the batched engine with one patch (device
        Givens least squares, CUDA-graph-captured Arnoldi steps); the others
        on MixedPrecisionFGMRES.  residual: "true" confirms convergence with
        the FP64 residual b - A x (one more FP64 matvec), "arnoldi" stops on
        the FP64 Arnoldi estimate as the reference's GMRES does."""
        _require_finite(to_device(b, torch.float64, require_cuda()), "right-hand side")
        if residual not in RESIDUAL_KINDS:
            raise ValueError(f"residual must be one of {RESIDUAL_KINDS}, got {residual!r}")
        if (precond == "tc" and len(self.rules) == 3 and self.M64 is None and self.K64.fused
                and self.K32.fused):
            return self._solve_engine(b, tolerance, maxiters, residual)
        self.mixed.tolerance, self.mixed.maxiters = tolerance, maxiters
        self.mixed.residual = residual
        P = self.precond_tc if precond == "tc" else self.precond_fp
        out = self.mixed.solve(self.apply, b, self.apply, P, cleandod=self.dirichlet)
        if precond == "tc":
            self.fd.space_preconditioner.check_tc_status()
        return out

    def _solve_engine(self, b, tolerance: float, maxiters: int,
                      residual: str = "true") -> RefinedOutput:
        from .batch import BatchedFGMRES, PatchBatch, _Patch

        restart = min(self.mixed.restart, 31)
        key = (restart, self.mixed.inner_iters)
        if getattr(self, "_engine_key", None) != key:
            patch = _Patch(self.rules, self.N, self.K64.plan.W,
                           self.K64, self.K32, self.fd, self.free,
                           self.dirichlet.cpu().numpy())
            self._engine = BatchedFGMRES(PatchBatch([patch]), tolerance=tolerance,
                                         restart=restart,
                                         max_cycles=max(1, -(-maxiters // restart)),
                                         inner_iters=self.mixed.inner_iters, use_graphs=True)
            self._engine_key = key
        eng = self._engine
        eng.residual = residual
        eng.tol = float(tolerance)
        eng.max_cycles = max(1, -(-maxiters // restart))
        numpy_in = not isinstance(b, torch.Tensor)
        res = eng.solve(b)
        eng.b.check_status()
        x = res.solution.clone()
        out = RefinedOutput(
            solution=x.cpu().numpy() if numpy_in else x,
            residual=np.asarray([1.0] + [float(h[0]) for h in res.history]),
            success=bool(res.success.all()),
            true_residual=float(res.true_residual.max()),
            residual_kind=res.residual_kind,
            outer_iterations=res.outer_steps,
            inner_iterations=res.outer_steps * self.mixed.inner_iters,
            history=[float(h[0]) for h in res.history],
        )
        if not out.success:
            warnings.warn(f"No convergence (true relative residual {out.true_residual:.2e}).")
        return out

    def solve_fp64(self, b, tolerance: float = 1e-10, maxiters: int = 60):
        """The plain FP64 GPU path: LinearSolver GMRES with FP64 operator and
        FP64 FD apply, Dirichlet DOFs masked (cleandod)."""
        from .solvers import LinearSolver

        def A(x):
            y = torch.empty_like(x)
            self.apply(x, y)
            return y

        def P(x):
            y = torch.empty_like(x)
            self.precond_fp(x, y)
            return y

        ls = LinearSolver(tolerance, maxiters, cleandod=[int(i) for i in self.dirichlet.tolist()],
                          linear_type="gmres", verbose=False)
        return ls.solve(A, b, P)

    def true_residual(self, x, b) -> float:
        """||b - A x|| / ||b|| in FP64 on the free DOFs."""
        xd = to_device(x, torch.float64).reshape(-1).clone()
        bd = to_device(b, torch.float64).reshape(-1).clone()
        K.mask(xd, self.dirichlet)
        K.mask(bd, self.dirichlet)
        r = torch.empty_like(xd)
        self.apply(xd, r)
        K.mask(r, self.dirichlet)
        K.axpby(1.0, bd, -1.0, r)
        ws = K.Workspace(r.device)
        return K.norm(ws, r) / K.norm(ws, bd)
