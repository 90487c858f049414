"""Krylov solvers with device-resident vectors, behind the reference API.

* ``LinearSolver``        -- src/igaops/solvers/linear_solver.py:26-639
  (GMRES, CG, BiCGSTAB, block CG, GCRO-DR wrapper; direct solve on the host)
* ``GCRODR``              -- src/igaops/solvers/deflated/gcrodr.py:50-373 with
  the cycles / harmonic Ritz extraction of deflated/helpers.py:13-265
* ``ConvergenceManager``  -- src/igaops/solvers/utils/convergence_manager.py

Vectors and Krylov bases live on the GPU; every O(n) operation runs in a
libigab200 kernel (gram / combine / axpby / mask).  Only the small dense
problems of the reference -- the Hessenberg least squares, harmonic Ritz
eigenproblems and k x k factorizations -- run on the host in FP64, as they do
in the reference.  Gram-Schmidt is classical with a second pass (CGS2): the
same two projection passes as the reference's modified Gram-Schmidt, each
pass one gram + one combine kernel over the whole basis.

``Afun`` / ``Pfun`` receive torch CUDA float64 tensors (complex128 parts are
passed as two real calls, as the reference does) and may return torch or
numpy arrays.  Numpy right-hand sides give numpy solutions.
"""
from __future__ import annotations

import logging
import warnings
from dataclasses import dataclass
from time import time
from typing import Callable, Dict, List, Literal, Optional

import numpy as np
import scipy.linalg as sclin
import torch
from numpy.linalg import lstsq

from . import krylov_ops as K
from ._device import require_cuda, to_device
from .common import Constants, validate_entry

logger = logging.getLogger(__name__)


# ======================================================= configuration
@dataclass
class SolverArgs:
    tolerance: float
    maxiters: int

    def __post_init__(self):
        if self.tolerance < Constants.SAFEGUARD or self.tolerance >= 1:
            raise ValueError(f"Relative tolerance must be > 0 and < 1, got {self.tolerance}")
        if self.maxiters <= 0:
            raise ValueError(f"Max iterations must be > 0, got {self.maxiters}")


@dataclass
class GcrodrArgs(SolverArgs):
    krylov_size: int = 40
    recycled_size: int = 20
    max_cycles: int = 10

    def __post_init__(self):
        super().__post_init__()
        if self.krylov_size <= 0:
            raise ValueError("Krylov size should be positive")
        if self.recycled_size < 0:
            raise ValueError("Recycle size should be greater than or equal to 0")
        if self.max_cycles <= 0:
            raise ValueError("Max no. cycles should greater than 0")
        if self.krylov_size < self.recycled_size:
            raise ValueError("Not consistent with the method")


@dataclass
class OutputArgs:
    solution: object
    residual: np.ndarray
    success: bool = False


# ================================================== convergence manager
class ConvergenceManager:
    """Stops when ANY non-iteration criterion is below its reference; raises
    RuntimeError when the iteration count exceeds its reference
    (convergence_manager.py:13-350)."""

    class Parameter:
        kind = "base"

        def __init__(self, name: str = ""):
            self._name = name
            self._reference = 0.0
            self._current: Optional[float] = None

        name = property(lambda self: self._name)

        @property
        def reference(self) -> float:
            return self._reference

        @reference.setter
        def reference(self, value):
            if not isinstance(value, (int, float, np.floating)):
                raise TypeError(f"Reference must be numeric, got {type(value)}")
            if value < 0:
                raise ValueError(f"Reference must be non-negative, got {value}")
            self._reference = float(value)

        @property
        def current(self):
            return self._current

        @current.setter
        def current(self, value):
            if not isinstance(value, (int, float, np.floating)):
                raise TypeError(f"Current must be numeric, got {type(value)}")
            if value < 0:
                raise ValueError(f"Current must be non-negative, got {value}")
            self._current = float(value)

        def is_defined(self) -> bool:
            return self._current is not None

        def reset(self):
            self._current = None

        def has_converged(self) -> bool:
            if self._current is None:
                return False
            return self._current < max(self._reference, Constants.SAFEGUARD)

    class AbsoluteError(Parameter):
        kind = "absolute_error"

    class RelativeError(Parameter):
        kind = "relative_error"

    class Iteration(Parameter):
        kind = "iteration"

        def has_converged(self) -> bool:
            if self._current is None:
                return False
            if self._current > self._reference:
                raise RuntimeError(f"Maximum iterations ({int(self._reference)}) exceeded. "
                                   "Algorithm did not converge.")
            return False

    PARAMETER_TYPES = {
        "absolute_error": AbsoluteError,
        "relative_error": RelativeError,
        "iteration": Iteration,
    }

    def __init__(self, refe_relative: float, refe_iteration: int, refe_absolute: float = 0.0):
        if not (0 < refe_relative < 1):
            raise ValueError(f"Relative tolerance must be > 0 and < 1, got {refe_relative}")
        if refe_iteration <= 0:
            raise ValueError(f"Max iterations must be > 0, got {refe_iteration}")
        if refe_absolute < 0:
            raise ValueError(f"Absolute tolerance must be >= 0, got {refe_absolute}")
        self._parameters: Dict[str, ConvergenceManager.Parameter] = {
            "absolute_error": self.AbsoluteError("absolute_error"),
            "relative_error": self.RelativeError("relative_error"),
            "iteration": self.Iteration("iteration"),
        }
        self._parameters["absolute_error"].reference = max(refe_absolute, Constants.SAFEGUARD)
        self._parameters["relative_error"].reference = refe_relative
        self._parameters["iteration"].reference = refe_iteration

    parameters = property(lambda self: self._parameters)

    def add_criterion(self, name: str, criterion_type: str, reference: Optional[float] = None):
        if name in self._parameters:
            raise ValueError(f"Criterion '{name}' already exists")
        if criterion_type not in self.PARAMETER_TYPES:
            raise ValueError(f"Invalid criterion type '{criterion_type}'")
        p = self.PARAMETER_TYPES[criterion_type](name)
        p.reference = reference if reference is not None else self._parameters[criterion_type].reference
        self._parameters[name] = p

    def update(self, curr_absolute=None, curr_relative=None, curr_iteration=None, **kwargs):
        for name, v in (("absolute_error", curr_absolute), ("relative_error", curr_relative),
                        ("iteration", curr_iteration)):
            if v is not None:
                self._parameters[name].current = v
        for name, v in kwargs.items():
            if name in self._parameters and isinstance(v, (int, float, np.floating)) and v >= 0:
                self._parameters[name].current = v
            else:
                logger.warning(f"Skipping convergence parameter {name!r} = {v!r}")

    def clear(self):
        for p in self._parameters.values():
            p.reset()

    def has_converged(self) -> bool:
        defined = [p for p in self._parameters.values() if p.is_defined()]
        if not defined:
            raise AssertionError("No convergence parameters have been set.")
        for name, p in self._parameters.items():
            if not p.is_defined():
                continue
            if name == "iteration":
                p.has_converged()
                continue
            if p.has_converged():
                return True
        return False

    def get_status(self):
        return {n: {"reference": p.reference, "current": p.current,
                    "converged": p.has_converged() if p.is_defined() else None}
                for n, p in self._parameters.items()}


# ========================================================== helpers
def _require_finite(v: torch.Tensor, what: str):
    """NonFiniteError (IGA_ERR_NONFINITE) when v holds a NaN or Inf: the
    reference would carry them through every iteration into the solution."""
    if not bool(torch.isfinite(v).all()):
        from ._lib import IGA_ERR_NONFINITE, NonFiniteError

        raise NonFiniteError(IGA_ERR_NONFINITE, f"{what} holds non-finite values")


def _check_finite_host(vals, what: str):
    if not np.all(np.isfinite(vals)):
        from ._lib import IGA_ERR_NONFINITE, NonFiniteError

        raise NonFiniteError(IGA_ERR_NONFINITE, f"non-finite value in {what}")


def _as_vec(y, like: torch.Tensor) -> torch.Tensor:
    if isinstance(y, torch.Tensor):
        if y.device == like.device and y.dtype == like.dtype and y.is_contiguous():
            return y
        return y.to(device=like.device, dtype=like.dtype).contiguous()
    return torch.from_numpy(np.ascontiguousarray(np.asarray(y, dtype=np.float64))).to(
        like.device, like.dtype)


# ======================================================= linear solver
class LinearSolver:
    """Iterative solvers of the reference with device-resident vectors."""

    def __init__(self, tolerance: float, maxiters: int, cleandod: Optional[List[int]] = None,
                 linear_type: Literal["cg", "bicgstab", "gcrodr", "gmres", "block_cg"] = "gmres",
                 verbose: bool = True):
        self._config = SolverArgs(tolerance=tolerance, maxiters=maxiters)
        self.set_cleandod(cleandod)
        self._linear_type = validate_entry(linear_type, ["cg", "bicgstab", "gcrodr", "gmres",
                                                         "block_cg"])
        self._convergence_manager: Optional[ConvergenceManager] = None
        self._last_simulation: Optional[OutputArgs] = None
        self._verbose = verbose
        self._gcrodr_solver: Optional[GCRODR] = None

    config = property(lambda self: self._config)
    linear_type = property(lambda self: self._linear_type)
    verbose = property(lambda self: self._verbose)

    def set_cleandod(self, cleandod: Optional[List[int]]):
        if cleandod is not None and not isinstance(cleandod, list):
            raise TypeError("Cleandod should be list")
        self._cleandod = cleandod
        self._mask_dev = None

    @property
    def last_simulation(self) -> OutputArgs:
        if self._last_simulation is None:
            return OutputArgs(solution=np.array([]), residual=np.array([]), success=False)
        return self._last_simulation

    @property
    def convergence_manager(self) -> ConvergenceManager:
        if self._convergence_manager is None:
            cm = ConvergenceManager(self._config.tolerance, self._config.maxiters,
                                    Constants.SAFEGUARD)
            cm.add_criterion("curr_increment", "relative_error")
            self._convergence_manager = cm
        return self._convergence_manager

    def update(self, tolerance: Optional[float] = None, maxiters: Optional[int] = None):
        kw = dict(tolerance=self._config.tolerance, maxiters=self._config.maxiters)
        if tolerance is not None:
            kw["tolerance"] = tolerance
        if maxiters is not None:
            kw["maxiters"] = maxiters
        self._config = SolverArgs(**kw)
        self._convergence_manager = None

    def _mask(self, x: torch.Tensor):
        if self._cleandod is None:
            return
        if self._mask_dev is None or self._mask_dev.device != x.device:
            self._mask_dev = torch.as_tensor(np.asarray(self._cleandod, dtype=np.int64),
                                             device=x.device)
        if x.ndim == 1:
            K.mask(x, self._mask_dev)
        else:
            for k in range(x.shape[1]):
                col = x[:, k].contiguous()
                K.mask(col, self._mask_dev)
                x[:, k] = col

    def solve(self, Afun: Callable, b, Pfun: Optional[Callable] = None, x0=None, **mv_args) -> OutputArgs:
        def identity(x):
            return x

        self.convergence_manager.clear()
        Pfun = Pfun if callable(Pfun) else identity
        if not (callable(Afun) and callable(Pfun)):
            raise TypeError("Afun and Pfun should be callable")
        solver = {"cg": self._CG, "bicgstab": self._BICGSTAB, "gcrodr": self._gcrodr,
                  "gmres": self._GMRES, "block_cg": self._BLOCK_CG}[self._linear_type]
        solver_args = {}
        for ky in ("krylov_size", "recycled_size", "max_cycles"):
            if ky in mv_args:
                solver_args[ky] = mv_args[ky]
            mv_args.pop(ky, None)
        dev = require_cuda()
        numpy_in = not isinstance(b, torch.Tensor)

        def matvec(x: torch.Tensor) -> torch.Tensor:
            self._mask(x)
            y = _as_vec(Afun(x, **mv_args), x)
            if y is x:
                y = y.clone()
            self._mask(y)
            return y

        def precond(x: torch.Tensor) -> torch.Tensor:
            self._mask(x)
            y = _as_vec(Pfun(x), x)
            if y is x:
                y = y.clone()
            self._mask(y)
            return y

        start = time()
        bd = to_device(b, torch.float64, dev).clone()
        _require_finite(bd, "right-hand side")
        self._mask(bd)
        x0d = None
        if x0 is not None:
            x0d = to_device(x0, torch.float64, dev).clone()
            self._mask(x0d)
            K.axpby(-1.0, matvec(x0d.clone()), 1.0, bd)
        output = solver(matvec, bd, precond, **solver_args)
        if x0d is not None:
            sol = _as_vec(output.solution, x0d)
            K.axpby(1.0, x0d, 1.0, sol)
            output.solution = sol
        if numpy_in and isinstance(output.solution, torch.Tensor):
            output.solution = output.solution.cpu().numpy()
        self._last_simulation = output
        if self._verbose and self._linear_type != "gcrodr":
            st = self.convergence_manager.get_status()
            logger.info(f"LINEAR SOLVER: {st['iteration']['current']} iterations, "
                        f"rel residue {st['relative_error']['current']}, "
                        f"{time() - start:.2e} s")
        return output

    # ------------------------------------------------------------ GMRES
    def _GMRES(self, Afun, b: torch.Tensor, Pfun, **kw) -> OutputArgs:
        """Unrestarted GMRES, right preconditioned with the stored Z = P V
        (flexible form), two Gram-Schmidt passes, least squares on the
        Hessenberg matrix each iteration (linear_solver.py:438-525)."""
        cm = self.convergence_manager
        ws = K.Workspace(b.device)
        n = b.shape[0]
        x = torch.zeros_like(b)
        output = OutputArgs(solution=x, residual=np.array([1.0]), success=True)
        r0 = K.norm(ws, b)
        cm.update(curr_absolute=r0)
        if cm.has_converged():
            return output
        m = int(cm.parameters["iteration"].reference)
        H = np.zeros((m + 1, m))
        V = torch.empty((m + 1, n), dtype=b.dtype, device=b.device)
        Z = torch.empty((m, n), dtype=b.dtype, device=b.device)
        K.axpby(1.0 / r0, b, 0.0, V[0])
        w = torch.empty_like(b)
        xold = torch.empty_like(b)
        diff = torch.empty_like(b)
        res = [1.0]
        converged = False
        for it in range(1, m + 1):
            z = Pfun(V[it - 1].clone())
            K.copy(z, Z[it - 1])
            K.copy(Afun(Z[it - 1].clone()), w)
            # both projection passes and the new norm stay on the device
            # until one transfer (same host arithmetic as reading each)
            hs = []
            for _ in range(2):
                h = K.gram(ws, V[:it], w)[:, 0]
                K.combine(V[:it], h.reshape(it, 1), w, alpha=-1.0, beta=1.0)
                hs.append(h)
            hs.append(K.gram(ws, w, w)[0])
            hv = torch.cat(hs).cpu().numpy()
            _check_finite_host(hv, "the Arnoldi step (operator or preconditioner output)")
            H[:it, it - 1] += hv[:it]
            H[:it, it - 1] += hv[it:2 * it]
            nw = float(np.sqrt(max(float(np.real(hv[2 * it])), 0.0)))
            H[it, it - 1] = nw
            if nw != 0:
                K.axpby(1.0 / nw, w, 0.0, V[it])
            else:
                # breakdown (the Krylov space is invariant): the reference keeps
                # a zero basis vector and lets the least squares finish
                V[it].zero_()
            mat = H[: it + 1, :it]
            rhs = np.zeros(it + 1)
            rhs[0] = r0
            y = lstsq(mat, rhs, rcond=None)[0]
            K.copy(x, xold)
            K.combine(Z[: len(y)], y.reshape(-1, 1), x)
            K.copy(x, diff)
            K.axpby(-1.0, xold, 1.0, diff)
            nd = torch.cat([K.gram(ws, diff, diff)[0], K.gram(ws, x, x)[0]]).cpu().numpy()
            incr = (float(np.sqrt(max(float(np.real(nd[0])), 0.0)))
                    / (float(np.sqrt(max(float(np.real(nd[1])), 0.0))) + Constants.SAFEGUARD))
            r1 = float(np.linalg.norm(rhs - mat @ y))
            res.append(r1 / r0)
            cm.update(curr_iteration=it, curr_absolute=r1, curr_relative=res[-1],
                      curr_increment=float(incr))
            if cm.has_converged():
                converged = True
                break
        if not converged:
            output.success = False
            warnings.warn(f"No convergence after {m} iterations.")
        output.solution = x
        output.residual = np.asarray(res)
        return output

    # --------------------------------------------------------------- CG
    def _CG(self, Afun, b: torch.Tensor, Pfun, **kw) -> OutputArgs:
        """Preconditioned CG (linear_solver.py:259-319)."""
        cm = self.convergence_manager
        ws = K.Workspace(b.device)
        x = torch.zeros_like(b)
        r = b.clone()
        output = OutputArgs(solution=x, residual=np.array([1.0]), success=True)
        n0 = K.norm(ws, r)
        cm.update(curr_absolute=n0)
        if cm.has_converged():
            return output
        pt = Pfun(r.clone())
        p = pt.clone()
        rs_old = float(K.dot(ws, r, pt))
        res = [1.0]
        m = int(cm.parameters["iteration"].reference)
        converged = False
        for it in range(1, m + 1):
            Ap = Afun(p.clone())
            alpha = rs_old / float(K.dot(ws, Ap, p))
            K.axpby(-alpha, Ap, 1.0, r)
            K.axpby(alpha, p, 1.0, x)
            incr = abs(alpha) * K.norm(ws, p) / (K.norm(ws, x) + Constants.SAFEGUARD)
            n1 = K.norm(ws, r)
            res.append(n1 / n0)
            cm.update(curr_iteration=it, curr_absolute=n1, curr_relative=res[-1],
                      curr_increment=float(incr))
            if cm.has_converged():
                converged = True
                break
            pt = Pfun(r.clone())
            rs_new = float(K.dot(ws, pt, r))
            K.axpby(1.0, pt, rs_new / rs_old, p)
            rs_old = rs_new
        if not converged:
            output.success = False
            warnings.warn(f"No convergence after {m} iterations.")
        output.solution = x
        output.residual = np.asarray(res)
        return output

    # --------------------------------------------------------- BiCGSTAB
    def _BICGSTAB(self, Afun, b: torch.Tensor, Pfun, **kw) -> OutputArgs:
        """Preconditioned BiCGSTAB (linear_solver.py:321-406)."""
        cm = self.convergence_manager
        ws = K.Workspace(b.device)
        x = torch.zeros_like(b)
        r = b.clone()
        output = OutputArgs(solution=x, residual=np.array([1.0]), success=True)
        n0 = K.norm(ws, r)
        cm.update(curr_absolute=n0)
        if cm.has_converged():
            return output
        rhat = r.clone()
        p = r.clone()
        rs_old = float(K.dot(ws, r, rhat))
        res = [1.0]
        m = int(cm.parameters["iteration"].reference)
        converged = False
        s = torch.empty_like(b)
        for it in range(1, m + 1):
            pt = Pfun(p.clone())
            Apt = Afun(pt.clone())
            alpha = rs_old / float(K.dot(ws, Apt, rhat))
            K.copy(r, s)
            K.axpby(-alpha, Apt, 1.0, s)
            K.axpby(alpha, pt, 1.0, x)
            incr = abs(alpha) * K.norm(ws, pt) / (K.norm(ws, x) + Constants.SAFEGUARD)
            n1 = K.norm(ws, s)
            res.append(n1 / n0)
            cm.update(curr_iteration=it, curr_absolute=n1, curr_relative=res[-1],
                      curr_increment=float(incr))
            if cm.has_converged():
                converged = True
                break
            st = Pfun(s.clone())
            Ast = Afun(st.clone())
            omega = float(K.dot(ws, Ast, s)) / float(K.dot(ws, Ast, Ast))
            K.copy(s, r)
            K.axpby(-omega, Ast, 1.0, r)
            K.axpby(omega, st, 1.0, x)
            n1 = K.norm(ws, r)
            res.append(n1 / n0)
            cm.update(curr_iteration=it, curr_absolute=n1, curr_relative=res[-1])
            if cm.has_converged():
                converged = True
                break
            rs_new = float(K.dot(ws, rhat, r))
            beta = (alpha / omega) * (rs_new / rs_old)
            # p = r + beta (p - omega Apt)
            K.axpby(-omega, Apt, 1.0, p)
            K.axpby(1.0, r, beta, p)
            rs_old = rs_new
        if not converged:
            output.success = False
            warnings.warn(f"No convergence after {m} iterations.")
        output.solution = x
        output.residual = np.asarray(res)
        return output

    # --------------------------------------------------------- block CG
    def _BLOCK_CG(self, Afun, b: torch.Tensor, Pfun, **kw) -> OutputArgs:
        """Block CG for b of shape (n, k) (linear_solver.py:527-593)."""
        if b.ndim != 2:
            raise ValueError("Expected 2D array.")
        cm = self.convergence_manager
        ws = K.Workspace(b.device)
        # rows = right-hand sides
        R = b.t().contiguous()
        X = torch.zeros_like(R)
        output = OutputArgs(solution=X.t(), residual=np.array([1.0]), success=True)

        def fro(A):
            return float(np.sqrt(max(np.trace(K.gram_host(ws, A, A)).real, 0.0)))

        n0 = fro(R)
        cm.update(curr_absolute=n0)
        if cm.has_converged():
            return output

        def apply_cols(fn, Rows):
            out = _as_vec(fn(Rows.t().contiguous()), Rows)
            return out.reshape(Rows.shape[1], Rows.shape[0]).t().contiguous() if out.ndim == 2 else out

        Zr = apply_cols(Pfun, R)
        P = Zr.clone()
        rtz_old = K.gram_host(ws, R, Zr)
        res = [1.0]
        m = int(cm.parameters["iteration"].reference)
        converged = False
        for it in range(1, m + 1):
            AP = apply_cols(Afun, P)
            PtAP = K.gram_host(ws, P, AP)
            PtR = K.gram_host(ws, P, R)
            gamma = lstsq(PtAP, PtR, rcond=None)[0]
            K.combine(AP, gamma, R, alpha=-1.0, beta=1.0)
            incr_rows = torch.zeros_like(X)
            K.combine(P, gamma, incr_rows)
            K.axpby(1.0, incr_rows, 1.0, X)
            incr = fro(incr_rows) / (fro(X) + Constants.SAFEGUARD)
            n1 = fro(R)
            res.append(n1 / n0)
            cm.update(curr_iteration=it, curr_absolute=n1, curr_relative=res[-1],
                      curr_increment=float(incr))
            if cm.has_converged():
                converged = True
                break
            Zr = apply_cols(Pfun, R)
            rtz_new = K.gram_host(ws, R, Zr)
            delta = lstsq(rtz_old, rtz_new, rcond=None)[0]
            Pn = Zr.clone()
            K.combine(P, delta, Pn, alpha=1.0, beta=1.0)
            P = Pn
            rtz_old = rtz_new
        if not converged:
            output.success = False
            warnings.warn(f"No convergence after {m} iterations.")
        output.solution = X.t().contiguous()
        output.residual = np.asarray(res)
        return output

    # ----------------------------------------------------------- GCRODR
    def _gcrodr(self, Afun, b, Pfun, **kw) -> OutputArgs:
        if self._gcrodr_solver is None:
            self._gcrodr_solver = GCRODR(self._config.tolerance, self._config.maxiters,
                                         krylov_size=kw.get("krylov_size", 40),
                                         recycled_size=kw.get("recycled_size", 20),
                                         max_cycles=kw.get("max_cycles", 10), verbose=self._verbose)
        o = self._gcrodr_solver.solve(Afun, b, Pfun)
        return OutputArgs(solution=o.solution, residual=o.residual, success=o.success)

    @staticmethod
    def direct(A, b, verbose: bool = True) -> OutputArgs:
        """Sparse LU solve (host, scipy) -- a verification tool, as in the
        reference (linear_solver.py:595-630)."""
        from scipy import sparse as sp
        from scipy.sparse.linalg import LinearOperator, spsolve

        if isinstance(A, LinearOperator):
            A = np.asarray(A @ np.eye(A.shape[1]))
        if isinstance(A, np.ndarray):
            A = sp.csr_array(A)
            A.eliminate_zeros()
        x = spsolve(A, np.asarray(b))
        return OutputArgs(solution=np.asarray(x), residual=np.array([]), success=True)


# ================================================================ GCRODR
class GCRODR:
    """GCRO with deflated restarting (Parks et al. 2006), left preconditioned,
    complex128 vectors on the device, recycled subspace kept per key."""

    def __init__(self, tolerance: float, maxiters: int, krylov_size: int = 40,
                 recycled_size: int = 20, max_cycles: int = 10, verbose: bool = True):
        self._verbose = verbose
        self._U_persist: Dict[str, torch.Tensor] = {}
        self._config = GcrodrArgs(tolerance=tolerance, maxiters=maxiters, krylov_size=krylov_size,
                                  recycled_size=recycled_size, max_cycles=max_cycles)
        self._convergence_manager: Optional[ConvergenceManager] = None

    config = property(lambda self: self._config)
    verbose = property(lambda self: self._verbose)

    @property
    def convergence_manager(self) -> ConvergenceManager:
        if self._convergence_manager is None:
            cm = ConvergenceManager(self._config.tolerance, self._config.maxiters,
                                    Constants.SAFEGUARD)
            cm.add_criterion("curr_increment", "relative_error")
            self._convergence_manager = cm
        return self._convergence_manager

    def update(self, tolerance: Optional[float] = None, maxiters: Optional[float] = None):
        kw = dict(self._config.__dict__)
        if tolerance is not None and np.isscalar(tolerance):
            kw["tolerance"] = float(np.abs(tolerance))
        if maxiters is not None and np.isscalar(maxiters):
            kw["maxiters"] = int(np.abs(maxiters))
        self._config = GcrodrArgs(**kw)
        self._convergence_manager = None

    def reset(self, reuse_name: str = "default"):
        self._U_persist.pop(reuse_name, None)

    # -- real operators on complex vectors, part by part
    def _op(self, fn, v: torch.Tensor, out: torch.Tensor):
        re, im = K.split_complex(v)
        yr = _as_vec(fn(re), re)
        yi = _as_vec(fn(im), im)
        K.merge_complex(yr, yi, out)
        return out

    def _MA(self, v: torch.Tensor, out: torch.Tensor):
        tmp = torch.empty_like(v)
        self._op(self.A, v, tmp)
        return self._op(self.M, tmp, out)

    def _cycle(self, ws, r: torch.Tensor, m: int, tol: float, C: Optional[torch.Tensor]):
        """Up to m (deflated) Arnoldi steps of M A from r (helpers.py:13-146)."""
        n = r.shape[0]
        dev = r.device
        V = torch.zeros((m + 1, n), dtype=torch.complex128, device=dev)
        H = np.zeros((m + 1, m), dtype=complex)
        Bc = None if C is None else np.zeros((C.shape[0], m), dtype=complex)
        resv = np.zeros(m)
        beta = K.norm(ws, r)
        k = 1
        y = np.zeros(1, dtype=complex)
        res = np.array([beta], dtype=complex)
        if beta <= Constants.SAFEGUARD:
            return V, H, Bc, k, resv[:k], y, res
        K.axpby(1.0 / beta, r, 0.0, V[0])
        w = torch.empty(n, dtype=torch.complex128, device=dev)
        for k in range(1, m + 1):
            self._MA(V[k - 1], w)
            if C is not None:
                bc = K.gram(ws, C, w)[:, 0]
                K.combine(C, bc.reshape(-1, 1), w, alpha=-1.0, beta=1.0)
                Bc[:, k - 1] = bc.cpu().numpy()
            for _ in range(2):
                h = K.gram(ws, V[:k], w)[:, 0]
                K.combine(V[:k], h.reshape(k, 1), w, alpha=-1.0, beta=1.0)
                H[:k, k - 1] += h.cpu().numpy()
            nw = K.norm(ws, w)
            H[k, k - 1] = nw
            if nw > 0.0:
                K.axpby(1.0 / nw, w, 0.0, V[k])
            mat = H[: k + 1, :k]
            rhs = np.zeros(k + 1, dtype=complex)
            rhs[0] = beta
            y = np.linalg.lstsq(mat, rhs, rcond=None)[0]
            res = rhs - mat @ y
            resv[k - 1] = np.linalg.norm(res)
            if resv[k - 1] < tol:
                break
        return V, H, Bc, k, resv[:k], y, res

    @staticmethod
    def _harm1(m, k, H):
        Hm = H[:m, :m]
        em = np.zeros(m, dtype=complex)
        em[-1] = 1.0
        f = np.linalg.solve(Hm.conj().T, em)
        G = Hm + (abs(H[m, m - 1]) ** 2) * np.outer(f, em.conj())
        vals, vecs = sclin.eig(G)
        good = np.isfinite(vals)
        vals, vecs = vals[good], vecs[:, good]
        return vecs[:, np.argsort(np.abs(vals))[:k]]

    @staticmethod
    def _harm2(k, G, Phi):
        vals, vecs = sclin.eig(G.conj().T @ G, G.conj().T @ Phi)
        good = np.isfinite(vals)
        vals, vecs = vals[good], vecs[:, good]
        return vecs[:, np.argsort(np.abs(vals))[:k]]

    @staticmethod
    def _rinv(R):
        return sclin.solve_triangular(R, np.eye(R.shape[0], dtype=R.dtype), lower=False)

    def _cholqr(self, ws, Cm: torch.Tensor):
        """Orthonormal C and R with Cm = C R (Cholesky QR, two passes)."""
        kk = Cm.shape[0]
        Rtot = np.eye(kk, dtype=complex)
        C = Cm
        for _ in range(2):
            G = K.gram_host(ws, C, C)
            G = 0.5 * (G + G.conj().T)
            R = np.linalg.cholesky(G).conj().T
            Cn = torch.empty_like(C)
            K.combine(C, self._rinv(R), Cn)
            C = Cn
            Rtot = R @ Rtot
        return C, Rtot

    def solve(self, Afun: Callable, b, Pfun: Optional[Callable] = None,
              reuse_name: str = "default") -> OutputArgs:
        if not callable(Afun):
            raise TypeError("Afun should be a function.")
        Pfun = Pfun if Pfun is not None else (lambda x: x)
        if not callable(Pfun):
            raise TypeError("Pfun should be a function.")
        cm = self.convergence_manager
        cm.clear()
        self.A, self.M = Afun, Pfun
        dev = require_cuda()
        numpy_in = not isinstance(b, torch.Tensor)
        ws = K.Workspace(dev)
        m, k = self._config.krylov_size, self._config.recycled_size
        tol, max_cycles = self._config.tolerance, self._config.max_cycles
        bd = to_device(b, torch.float64, dev)
        n = bd.shape[0]
        bc = K.merge_complex(bd, torch.zeros_like(bd))
        x = torch.zeros(n, dtype=torch.complex128, device=dev)
        r = torch.empty_like(x)
        self._op(self.M, bc, r)
        norm0 = K.norm(ws, r)
        resvec = [norm0]

        def finish(success):
            xr = K.split_complex(x)[0]
            sol = xr.cpu().numpy() if numpy_in else xr
            v = np.abs(np.asarray(resvec))
            return OutputArgs(solution=sol, residual=v / max(v[0], Constants.SAFEGUARD),
                              success=success)

        cm.update(curr_absolute=norm0, curr_iteration=0)
        if cm.has_converged():
            return finish(True)
        nmv = 0
        U = C = None
        if reuse_name in self._U_persist:
            Y = self._U_persist[reuse_name]
            Cm = torch.empty_like(Y)
            for i in range(Y.shape[0]):
                self._MA(Y[i], Cm[i])
            C, R = self._cholqr(ws, Cm)
            U = torch.empty_like(Y)
            K.combine(Y, self._rinv(R), U)
            cr = K.gram(ws, C, r)[:, 0]
            K.combine(U, cr.reshape(-1, 1), x, alpha=1.0, beta=1.0)
            K.combine(C, cr.reshape(-1, 1), r, alpha=-1.0, beta=1.0)
            resvec.append(K.norm(ws, r))
            p = np.inf
        else:
            V, H, _, p, rv, y, res = self._cycle(ws, r, m, tol * norm0, None)
            K.combine(V[:p], y.reshape(-1, 1), x, alpha=1.0, beta=1.0)
            r = torch.zeros_like(x)
            K.combine(V[: p + 1], res.reshape(-1, 1), r)
            resvec.extend(rv.tolist())
            nmv += p
            if p >= k:
                Pk = self._harm1(p, k, H)
                Y = torch.empty((k, n), dtype=torch.complex128, device=dev)
                K.combine(V[:p], Pk, Y)
                Q, R = np.linalg.qr(H[: p + 1, :p] @ Pk, mode="reduced")
                C = torch.empty((k, n), dtype=torch.complex128, device=dev)
                K.combine(V[: p + 1], Q, C)
                U = torch.empty_like(Y)
                K.combine(Y, self._rinv(R), U)
        rn = K.norm(ws, r)
        cm.update(curr_absolute=rn, curr_relative=rn / norm0, curr_iteration=nmv)
        if cm.has_converged() or p < m:
            if U is not None:
                self._U_persist[reuse_name] = U
            return finish(True)
        if U is None or C is None:
            raise RuntimeError("U and/or C are not initialized.")
        success = False
        for _cycle in range(max_cycles):
            V, H, Bc, p, rv, _, _ = self._cycle(ws, r, m - k, tol * norm0, C)
            resvec.extend(rv.tolist())
            nmv += p
            dvals = np.real(np.diag(K.gram_host(ws, U, U)))
            D = np.diag(1.0 / np.sqrt(dvals))
            Ut = torch.empty_like(U)
            K.combine(U, D, Ut)
            G = np.block([[D, Bc[:, :p]], [np.zeros((p + 1, k), dtype=complex), H[: p + 1, :p]]])
            rhs = np.concatenate([K.gram_host(ws, C, r)[:, 0], K.gram_host(ws, V[: p + 1], r)[:, 0]])
            yv = np.linalg.lstsq(G, rhs, rcond=None)[0]
            K.combine(Ut, yv[:k].reshape(-1, 1), x, alpha=1.0, beta=1.0)
            K.combine(V[:p], yv[k:].reshape(-1, 1), x, alpha=1.0, beta=1.0)
            gz = G @ yv
            K.combine(C, gz[:k].reshape(-1, 1), r, alpha=-1.0, beta=1.0)
            K.combine(V[: p + 1], gz[k:].reshape(-1, 1), r, alpha=-1.0, beta=1.0)
            rn = K.norm(ws, r)
            cm.update(curr_absolute=rn, curr_relative=rn / norm0, curr_iteration=nmv)
            if cm.has_converged() or p < m - k:
                success = True
                break
            # Phi = W^H Vhat with W = [C; V_{p+1}], Vhat = [Ut; V_p]
            Phi = np.block([[K.gram_host(ws, C, Ut), K.gram_host(ws, C, V[:p])],
                            [K.gram_host(ws, V[: p + 1], Ut), K.gram_host(ws, V[: p + 1], V[:p])]])
            Pk = self._harm2(k, G, Phi)
            Y = torch.zeros((k, n), dtype=torch.complex128, device=dev)
            K.combine(Ut, Pk[:k], Y)
            K.combine(V[:p], Pk[k:], Y, alpha=1.0, beta=1.0)
            Q, R = np.linalg.qr(G @ Pk, mode="reduced")
            Cn = torch.zeros_like(Y)
            K.combine(C, Q[:k], Cn)
            K.combine(V[: p + 1], Q[k:], Cn, alpha=1.0, beta=1.0)
            C = Cn
            U = torch.empty_like(Y)
            K.combine(Y, self._rinv(R), U)
        else:
            warnings.warn(f"No convergence after {max_cycles} cycles.")
        self._U_persist[reuse_name] = U
        return finish(success)
