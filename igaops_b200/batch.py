"""Many independent patches solved together on one GPU.

The reference solves one patch per call (a GMRES loop around user callables,
src/igaops/solvers/linear_solver.py:438-525).  Small and medium patches leave
a B200 mostly idle in that form: every iteration is a handful of short
kernels and host round trips.  ``PatchBatch`` keeps all patches resident and
runs each step of the iteration for all of them at once:

* one fused matvec launch per band width over every patch of that width
  (``iga_mf_batch_matvec``; FP64 for the outer iteration, FP32 inside);
* one set of six tensor-core launches for the fast-diagonalisation apply of
  every patch (``iga_fd_tc_batch_apply``, BF16 products, FP32 accumulation);
* segmented Gram / combine / scale kernels for the per-patch Arnoldi vectors
  and a per-patch Givens update of the Hessenberg least squares on the device
  (``iga_seg_*``), so an Arnoldi step needs no host round trip;
* each Arnoldi step, matvec and preconditioner included, is captured once in
  a CUDA graph and replayed; the host reads the per-patch convergence flags
  every few steps.

``BatchedFGMRES`` is the mixed-precision solver of
``igaops_b200.refine.MixedPrecisionFGMRES`` in this batched form: FP64
flexible GMRES outside (FP64 matvec, Arnoldi, residual check), an FP32 GMRES
of ``inner_iters`` steps with the BF16 tensor-core preconditioner inside (or
the preconditioner alone for ``inner_iters = 0``).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from . import krylov_ops as K
from ._device import iga_dtype, require_cuda, stream_handle, to_device

__all__ = ["PatchBatch", "BatchedFGMRES", "BatchResult"]


def _ptr(t: torch.Tensor, elem_offset: int = 0) -> int:
    return t.data_ptr() + elem_offset * t.element_size()


class _Seg:
    """Segmentation of a flat multi-patch vector (see iga_seg_*)."""

    def __init__(self, sizes: Sequence[int], device):
        chunk = int(_lib.LIB.iga_seg_chunk())
        self.np = len(sizes)
        offs = np.zeros(self.np + 1, dtype=np.int64)
        offs[1:] = np.cumsum(sizes)
        nb = [max(1, -(-int(s) // chunk)) for s in sizes]
        blk0 = np.zeros(self.np + 1, dtype=np.int32)
        blk0[1:] = np.cumsum(nb)
        self.offs_host = offs
        self.ntot = int(offs[-1])
        self.nblk = int(blk0[-1])
        self.offs = torch.from_numpy(offs).to(device)
        self.blk0 = torch.from_numpy(blk0).to(device)
        self.partial = torch.empty(self.nblk * 32, dtype=torch.float64, device=device)

    def gram(self, A: torch.Tensor, m: int, x: torch.Tensor, out_ptr: int, ldo: int):
        _lib.check(_lib.LIB.iga_seg_gram(iga_dtype(A.dtype), self.np, self.offs.data_ptr(),
                                         self.blk0.data_ptr(), self.nblk, m, A.data_ptr(),
                                         A.stride(0) if A.ndim == 2 else A.numel(), x.data_ptr(),
                                         self.partial.data_ptr(), out_ptr, ldo, stream_handle()))

    def combine(self, A: torch.Tensor, m: int, coef_ptr: int, ldc: int, alpha: float,
                beta: float, out: torch.Tensor):
        _lib.check(_lib.LIB.iga_seg_combine(iga_dtype(out.dtype), self.np, self.offs.data_ptr(),
                                            self.blk0.data_ptr(), self.nblk, m, A.data_ptr(),
                                            A.stride(0) if A.ndim == 2 else A.numel(), coef_ptr,
                                            ldc, float(alpha), float(beta), out.data_ptr(),
                                            stream_handle()))

    def scale(self, x: torch.Tensor, s_ptr: int, lds: int, mode: int):
        _lib.check(_lib.LIB.iga_seg_scale(iga_dtype(x.dtype), self.np, self.offs.data_ptr(),
                                          self.blk0.data_ptr(), self.nblk, x.data_ptr(), s_ptr,
                                          lds, mode, stream_handle()))


class _BatchArnoldi:
    """Per-patch Arnoldi with two classical Gram-Schmidt passes and the
    Givens least squares, all patches at once, no host round trip."""

    def __init__(self, seg: _Seg, m: int, dtype: torch.dtype, device):
        if m > 31:
            raise ValueError("at most 31 Arnoldi steps per cycle")
        self.seg, self.m, self.dtype = seg, m, dtype
        P, n = seg.np, seg.ntot
        f64 = dict(dtype=torch.float64, device=device)
        self.V = torch.zeros((m + 1, n), dtype=dtype, device=device)
        self.Z = torch.zeros((m, n), dtype=dtype, device=device)
        self.H = torch.zeros((P, m, m + 1), **f64)
        self.h2 = torch.zeros((P, m + 1), **f64)
        self.cs = torch.zeros((P, m), **f64)
        self.sn = torch.zeros((P, m), **f64)
        self.g = torch.zeros((P, m + 1), **f64)
        self.y = torch.zeros((P, m), **f64)
        self.beta2 = torch.zeros(P, **f64)
        self.ref = torch.ones(P, **f64)
        self.resid = torch.zeros(P, **f64)
        self.conv = torch.full((P,), -1, dtype=torch.int32, device=device)
        self.tol = 0.0

    def start(self, r: torch.Tensor):
        s, m = self.seg, self.m
        s.gram(r, 1, r, self.beta2.data_ptr(), 1)
        K.copy(r, self.V[0])
        s.scale(self.V[0], self.beta2.data_ptr(), 1, 2)
        _lib.check(_lib.LIB.iga_seg_givens_init(s.np, m, self.beta2.data_ptr(), self.g.data_ptr(),
                                                self.conv.data_ptr(), self.resid.data_ptr(),
                                                stream_handle()))

    def step(self, j: int, A_into: Callable, P_into: Callable):
        s, m = self.seg, self.m
        V, w = self.V, self.V[j + 1]
        P_into(V[j], self.Z[j])
        A_into(self.Z[j], w)
        ldH = m * (m + 1)
        colj = _ptr(self.H, j * (m + 1))
        s.gram(V, j + 1, w, colj, ldH)
        s.combine(V, j + 1, colj, ldH, -1.0, 1.0, w)
        s.gram(V, j + 1, w, self.h2.data_ptr(), m + 1)
        s.combine(V, j + 1, self.h2.data_ptr(), m + 1, -1.0, 1.0, w)
        nrm = _ptr(self.H, j * (m + 1) + j + 1)
        s.gram(w, 1, w, nrm, ldH)
        s.scale(w, nrm, ldH, 2)
        _lib.check(_lib.LIB.iga_seg_givens_step(
            s.np, m, j, self.H.data_ptr(), self.h2.data_ptr(), m + 1, self.cs.data_ptr(),
            self.sn.data_ptr(), self.g.data_ptr(), self.ref.data_ptr(), float(self.tol),
            self.conv.data_ptr(), self.resid.data_ptr(), stream_handle()))

    def update(self, k: int, x: torch.Tensor, beta: float = 1.0):
        """x = beta*x + Z[:k] y_p per patch (y from the triangular solve)."""
        s, m = self.seg, self.m
        _lib.check(_lib.LIB.iga_seg_trisolve(s.np, m, k, self.H.data_ptr(), self.g.data_ptr(),
                                             self.conv.data_ptr(), self.y.data_ptr(),
                                             stream_handle()))
        s.combine(self.Z, k, self.y.data_ptr(), m, 1.0, beta, x)


@dataclass
class _Patch:
    rules: list
    N: int
    W: int
    K64: object
    K32: object
    fd: object
    free: np.ndarray
    dirichlet: np.ndarray


class PatchBatch:
    """Independent 3D patches -- stiffness operator, homogeneous Dirichlet
    boundary from a table, fast-diagonalisation preconditioner each -- held
    on the device with the multi-patch launch tables.

    patches: sequence of (quadrule_list, stiffness_coefficients, table_dirichlet).
    """

    @staticmethod
    def make_patch(rules, coefs, table, nseg=None) -> _Patch:
        """Device data of one patch: FP64 and FP32 packed operators, FD
        eigendata (tensor-core images built on first use), Dirichlet sets."""
        from .fastdiag import SingleFD
        from .operators import MFOperator

        rules = list(rules)
        if len(rules) != 3:
            raise ValueError("batched patches are 3D")
        # segment count of each operator: autotuned per patch shape (cached)
        # by default; "heuristic" takes the plan's rule of thumb (no timing)
        ns = "auto" if nseg is None else (None if nseg == "heuristic" else nseg)
        # one host -> device copy of the coefficients serves both operators
        coefs = to_device(coefs, torch.float64)
        # the batched launches run the pencil kernel's multi-patch form
        K64 = MFOperator(rules, coefs, "gradu_gradv", dtype=torch.float64, nseg=ns, kernel="pencil")
        K32 = MFOperator(rules, coefs, "gradu_gradv", dtype=torch.float32, nseg=ns, kernel="pencil",
                         symmetric=K64.symmetric)
        if not (K64.fused and K32.fused):
            raise NotImplementedError("batched patches need fused-kernel rules (WQ type 2 or Gauss)")
        fd = SingleFD("spatial")
        # scalar coefficients (0, 1), the default: Lambda is formed where an
        # apply needs it (the tensor-core data forms 1/Lambda on the device)
        fd.compute_space_eigendecomposition(rules, np.asarray(table, dtype=bool))
        sp = fd.space_preconditioner
        return _Patch(rules, K64.N, K64.plan.W, K64, K32, fd, sp.free_nodes(0),
                      sp.dirichlet_nodes(0))

    def __init__(self, patches: Sequence, nseg=None):
        dev = require_cuda()
        self.device = dev
        self.patches: List[_Patch] = [
            p if isinstance(p, _Patch) else PatchBatch.make_patch(*p, nseg=nseg) for p in patches]
        self.np = len(self.patches)
        self.seg = _Seg([p.N for p in self.patches], dev)
        offs = self.seg.offs_host
        self.dirichlet = torch.from_numpy(
            np.concatenate([p.dirichlet + offs[i] for i, p in enumerate(self.patches)])).to(dev)
        self.ntot = self.seg.ntot
        self._mv = {torch.float64: self._matvec_tables(torch.float64),
                    torch.float32: self._matvec_tables(torch.float32)}
        self._fd = {}  # tensor-core FD tables, built on first use per I/O precision

    # -------------------------------------------------------------- tables
    def _matvec_tables(self, dtype):
        dt = iga_dtype(dtype)
        groups = {}
        for i, p in enumerate(self.patches):
            groups.setdefault(p.W, []).append(i)
        out = []
        for W, idx in sorted(groups.items()):
            ops = [self.patches[i].K64 if dtype == torch.float64 else self.patches[i].K32
                   for i in idx]
            plans = (_lib.iga_mf_plan * len(idx))(*[o.plan.P for o in ops])
            packed = (ctypes.c_void_p * len(idx))(*[o.packed.data_ptr() for o in ops])
            offs = (ctypes.c_int64 * len(idx))(*[int(self.seg.offs_host[i]) for i in idx])
            nbytes = ctypes.c_int64(0)
            _lib.check(_lib.LIB.iga_mf_batch_table_bytes(dt, len(idx), ctypes.byref(nbytes)))
            table = torch.empty(int(nbytes.value) + 256, dtype=torch.uint8, device=self.device)
            base = (table.data_ptr() + 255) // 256 * 256
            ctas = ctypes.c_int32(0)
            smem = ctypes.c_int64(0)
            _lib.check(_lib.LIB.iga_mf_batch_prepare(plans, len(idx), dt, packed, offs, base,
                                                     ctypes.byref(ctas), ctypes.byref(smem)))
            # the kernel reads the skip flag of its group-local patch index:
            # each group gathers the flags of its patches (global indices)
            gidx = torch.tensor(idx, dtype=torch.int64, device=self.device)
            contiguous = idx == list(range(len(idx)))
            out.append(dict(plan0=plans[0], plans=plans, n=len(idx), table=table, base=base,
                            ctas=int(ctas.value), smem=int(smem.value), ops=ops, gidx=gidx,
                            identity=contiguous,
                            skipbuf=torch.empty(len(idx), dtype=torch.int32, device=self.device)))
        return out

    def _fd_table(self, io_dtype):
        P = self.np
        i32 = ctypes.c_int32 * (3 * P)
        n, lo, m = i32(), i32(), i32()
        Bf = (ctypes.c_void_p * (3 * P))()
        Bb = (ctypes.c_void_p * (3 * P))()
        inv = (ctypes.c_void_p * P)()
        w0 = (ctypes.c_void_p * P)()
        w1 = (ctypes.c_void_p * P)()
        offs = (ctypes.c_int64 * P)()
        keep = []
        status = torch.zeros(1, dtype=torch.int32, device=self.device)
        for i, p in enumerate(self.patches):
            sp = p.fd.space_preconditioner
            fwd, bwd, invl, work, _ = sp.tc_data(0)
            keep.append((fwd, bwd, invl, work))
            lo_i, mm = sp._boxes[0]
            nn = [sp._nonzeros_by_dir[d] for d in sp._space_dirs]
            for d in range(3):
                n[3 * i + d], lo[3 * i + d], m[3 * i + d] = int(nn[d]), int(lo_i[d]), int(mm[d])
                Bf[3 * i + d] = fwd[d].data_ptr()
                Bb[3 * i + d] = bwd[d].data_ptr()
            inv[i] = invl.data_ptr()
            w0[i] = work[0].data_ptr()
            w1[i] = work[1].data_ptr()
            offs[i] = int(self.seg.offs_host[i])
        nbytes = ctypes.c_int64(0)
        _lib.check(_lib.LIB.iga_fd_tc_batch_table_bytes(P, ctypes.byref(nbytes)))
        table = torch.empty(int(nbytes.value) + 256, dtype=torch.uint8, device=self.device)
        base = (table.data_ptr() + 255) // 256 * 256
        grid = (ctypes.c_int32 * 6)()
        smem = ctypes.c_int64(0)
        _lib.check(_lib.LIB.iga_fd_tc_batch_prepare(P, n, lo, m, Bf, Bb, inv, w0, w1, offs,
                                                    iga_dtype(io_dtype), status.data_ptr(), base,
                                                    grid, ctypes.byref(smem)))
        return dict(table=table, base=base, grid=grid, smem=int(smem.value), keep=keep,
                    status=status)

    # ---------------------------------------------------------- operators
    def matvec(self, x: torch.Tensor, y: torch.Tensor, skip: Optional[torch.Tensor] = None):
        """y = K_p x_p for every patch (one launch per band width), Dirichlet
        rows zeroed; patches with skip[p] >= 0 are left at zero."""
        if self.np == 1:
            # one patch: its own operator's launch (arguments as kernel
            # parameters, 5-7 % faster than the multi-patch kernel).  skip is
            # not needed: a step after convergence only fills Arnoldi columns
            # beyond the converged one, which the triangular solve ignores.
            p = self.patches[0]
            (p.K64 if x.dtype == torch.float64 else p.K32).apply_into(x, y)
            K.mask(y, self.dirichlet)
            return
        dt = iga_dtype(x.dtype)
        for gi, g in enumerate(self._mv[x.dtype]):
            if skip is None:
                sk = None
            elif g["identity"]:
                sk = skip.data_ptr()
            else:
                torch.index_select(skip, 0, g["gidx"], out=g["skipbuf"])
                sk = g["skipbuf"].data_ptr()
            _lib.check(_lib.LIB.iga_mf_batch_matvec(
                ctypes.byref(g["plan0"]), dt, g["n"], g["base"], g["ctas"], g["smem"],
                x.data_ptr(), y.data_ptr(), self.ntot, 1 if gi == 0 else 0, sk, stream_handle()))
        K.mask(y, self.dirichlet)

    def precond(self, x: torch.Tensor, y: torch.Tensor, skip: Optional[torch.Tensor] = None):
        """y = P_p^{-1} x_p for every patch: BF16 tensor-core FD apply."""
        f = self._fd.get(x.dtype)
        if f is None:
            f = self._fd[x.dtype] = self._fd_table(x.dtype)
        _lib.check(_lib.LIB.iga_fd_tc_batch_apply(iga_dtype(x.dtype), self.np, f["base"],
                                                  f["grid"], f["smem"], x.data_ptr(),
                                                  y.data_ptr(), self.ntot,
                                                  None if skip is None else skip.data_ptr(),
                                                  stream_handle()))

    def precond_fp64(self, x: torch.Tensor, y: torch.Tensor):
        """y = P_p^{-1} x_p for every patch with the FP64 fast-diagonalisation
        apply (the reference's SpaceFD.apply arithmetic in FP64, SIMT mode
        products): one apply per patch."""
        o = self.seg.offs_host
        if not hasattr(self, "_fd64_work"):
            self._fd64_work = []
            for p in self.patches:
                sp = p.fd.space_preconditioner
                M = int(np.prod(sp._boxes[0][1]))
                self._fd64_work.append((torch.empty(M, dtype=torch.float64, device=self.device),
                                        torch.empty(M, dtype=torch.float64, device=self.device)))
        for i, p in enumerate(self.patches):
            p.fd.space_preconditioner.apply_device(x[o[i]:o[i + 1]], y[o[i]:o[i + 1]],
                                                   work=self._fd64_work[i])
        # the apply writes the free box only: the Dirichlet entries are zero
        K.mask(y, self.dirichlet)

    def check_status(self):
        for f in self._fd.values():
            st = int(f["status"].item())
            if st:
                f["status"].zero_()
                _lib.check(st)
        for p in self.patches:
            p.K64.plan.check_status()
            p.K32.plan.check_status()

    def split(self, flat) -> List[np.ndarray]:
        """Per-patch pieces of a flat vector (host)."""
        a = flat.detach().cpu().numpy() if isinstance(flat, torch.Tensor) else np.asarray(flat)
        o = self.seg.offs_host
        return [a[o[i]:o[i + 1]] for i in range(self.np)]

    def join(self, parts) -> torch.Tensor:
        return to_device(np.concatenate([np.asarray(p, dtype=np.float64) for p in parts]),
                         torch.float64, self.device)

    # ------------------------------------------------------ plain FP64 path
    def solve_fp64_sequential(self, b_flat, tolerance: float = 1e-10, maxiters: int = 60):
        """The plain FP64 GPU path on the same inputs: one patch after the
        other, the reference's FD-preconditioned GMRES
        (linear_solver.py:438-525) with the FP64 fused matvec and the FP64
        FD apply of that patch."""
        from .solvers import LinearSolver

        bs = [torch.from_numpy(np.ascontiguousarray(p)).to(self.device) for p in self.split(b_flat)]
        sols, iters = [], []
        for p, b in zip(self.patches, bs):
            def A(x, p=p):
                y = torch.empty_like(x)
                p.K64.apply_into(x, y)
                return y

            def P(x, p=p):
                y = torch.empty_like(x)
                p.fd.space_preconditioner.apply_device(x, y)
                return y

            ls = LinearSolver(tolerance, maxiters, cleandod=[int(i) for i in p.dirichlet],
                              linear_type="gmres", verbose=False)
            out = ls.solve(A, b, P)
            sols.append(out.solution)
            iters.append(len(out.residual) - 1)
        return sols, iters


@dataclass
class BatchResult:
    """true_residual: per-patch relative residual of the returned solution,
    ||b - A x|| / ||b|| recomputed in FP64 when residual_kind is "true", the
    FP64 Arnoldi (Givens) estimate when it is "arnoldi"."""

    solution: torch.Tensor
    success: np.ndarray
    true_residual: np.ndarray
    cycles: int = 0
    outer_steps: int = 0
    history: list = field(default_factory=list)
    residual_kind: str = "true"


RESIDUAL_KINDS = ("true", "arnoldi")


class BatchedFGMRES:
    """FGMRES(restart) in FP64 over all patches of a ``PatchBatch`` with a
    low-precision inner solve (see the module docstring).

    precision="fp64": the same engine (batched FP64 matvec, segmented
    Arnoldi, device Givens, graph-captured steps) with the FP64 FD apply of
    every patch as the preconditioner and no low-precision work -- the
    baseline that isolates what the mixed precision buys.

    residual="true": every cycle ends with the FP64 residual b - A x (one
    more matvec), which decides success and starts the next cycle;
    "arnoldi": a cycle in which every patch met its tolerance by the FP64
    Arnoldi (Givens) residual estimate ends there, the stopping rule of the
    reference's GMRES (linear_solver.py:507-521); cycles that restart still
    take the true residual."""

    def __init__(self, batch: PatchBatch, tolerance: float = 1e-10, restart: int = 12,
                 max_cycles: int = 6, inner_iters: int = 0, check_every: int = 1,
                 use_graphs: bool = True, precision: str = "mixed", residual: str = "true"):
        if precision not in ("mixed", "fp64"):
            raise ValueError(f"precision must be 'mixed' or 'fp64', got {precision!r}")
        if residual not in RESIDUAL_KINDS:
            raise ValueError(f"residual must be one of {RESIDUAL_KINDS}, got {residual!r}")
        self.precision = precision
        self.residual = residual
        self.b = batch
        self.tol = float(tolerance)
        self.restart = int(restart)
        self.max_cycles = int(max_cycles)
        self.inner_iters = int(inner_iters)
        self.check_every = max(1, int(check_every))
        self.use_graphs = use_graphs
        dev = batch.device
        seg = batch.seg
        self.outer = _BatchArnoldi(seg, self.restart, torch.float64, dev)
        self.outer.tol = self.tol
        self.inner = _BatchArnoldi(seg, max(1, self.inner_iters), torch.float32, dev)
        self.inner.tol = 0.0
        n = seg.ntot
        self.v32 = torch.zeros(n, dtype=torch.float32, device=dev)
        self.z32 = torch.zeros(n, dtype=torch.float32, device=dev)
        self.r = torch.zeros(n, dtype=torch.float64, device=dev)
        self.x = torch.zeros(n, dtype=torch.float64, device=dev)
        self.bd = torch.zeros(n, dtype=torch.float64, device=dev)
        self.rr = torch.zeros(seg.np, dtype=torch.float64, device=dev)
        self._graphs = {}

    def _convert(self, src, dst):
        _lib.check(_lib.LIB.iga_convert(iga_dtype(src.dtype), iga_dtype(dst.dtype), src.numel(),
                                        src.data_ptr(), dst.data_ptr(), stream_handle()))

    def _precond(self, v64: torch.Tensor, z64: torch.Tensor):
        B = self.b
        if self.precision == "fp64":
            B.precond_fp64(v64, z64)
            return
        sk = self.outer.conv  # patches that converged in this cycle do no more work
        self._convert(v64, self.v32)
        if self.inner_iters == 0:
            B.precond(self.v32, self.z32, sk)
        else:
            inn = self.inner
            inn.start(self.v32)
            for j in range(self.inner_iters):
                inn.step(j, lambda a, b: B.matvec(a, b, sk), lambda a, b: B.precond(a, b, sk))
            inn.update(self.inner_iters, self.z32, beta=0.0)
        self._convert(self.z32, z64)

    def _step(self, j: int):
        self.outer.step(j, lambda a, b: self.b.matvec(a, b, self.outer.conv), self._precond)

    def _run_step(self, j: int):
        if not self.use_graphs:
            self._step(j)
            return
        g = self._graphs.get(j)
        if g is None:
            # the first use runs the step eagerly on a side stream (the first
            # launch configures the kernels) and then captures it; capture
            # records without executing, and the eager run was this step, so
            # it is not replayed now: the Givens update of g is not
            # idempotent, and a second run would scale the residual estimate
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                self._step(j)
            torch.cuda.current_stream().wait_stream(s)
            g = torch.cuda.CUDAGraph()
            # thread-local capture: other threads of the process (a serving
            # loop's set-up and 2D threads) keep allocating and copying while
            # this thread captures; only this thread's calls are restricted
            with torch.cuda.graph(g, capture_error_mode="thread_local"):
                self._step(j)
            self._graphs[j] = g
            return
        g.replay()

    def _norms(self, v: torch.Tensor) -> np.ndarray:
        self.b.seg.gram(v, 1, v, self.rr.data_ptr(), 1)
        return np.sqrt(np.maximum(self.rr.cpu().numpy(), 0.0))

    def set_problem(self, b_flat, x0=None, tolerances=None):
        """Load b (and an initial guess) for a sequence of cycle() calls;
        tolerances: per-patch relative tolerances (default: the solver's)."""
        B = self.b
        K.copy(to_device(b_flat, torch.float64, B.device).reshape(-1), self.bd)
        K.mask(self.bd, B.dirichlet)
        self.bnorm = self._norms(self.bd)
        if not np.all(np.isfinite(self.bnorm)):
            from ._lib import IGA_ERR_NONFINITE, NonFiniteError

            bad = [int(i) for i in np.flatnonzero(~np.isfinite(self.bnorm))]
            raise NonFiniteError(IGA_ERR_NONFINITE,
                                 f"right-hand sides of patches {bad} hold non-finite values")
        self.safe = np.where(self.bnorm > 0, self.bnorm, 1.0)
        tols = np.full(B.np, self.tol) if tolerances is None else np.asarray(tolerances, float)
        self.tols = tols
        # a patch's Arnoldi cycle stops at ||r|| < tol_p ||b_p|| (tol folded into ref)
        self.outer.tol = 1.0
        self.outer.ref.copy_(torch.from_numpy(tols * self.bnorm))
        if x0 is None:
            self.x.zero_()
            K.copy(self.bd, self.r)
        else:
            K.copy(to_device(x0, torch.float64, B.device).reshape(-1), self.x)
            K.mask(self.x, B.dirichlet)
            B.matvec(self.x, self.r)
            K.axpby(1.0, self.bd, -1.0, self.r)

    def cycle(self, res: BatchResult):
        """One restart cycle of FGMRES for every patch; updates x, the
        residual (see ``residual``) and the per-patch success flags."""
        B = self.b
        self.outer.start(self.r)
        k = 0
        all_conv = False
        for j in range(self.restart):
            self._run_step(j)
            k = j + 1
            res.outer_steps += 1
            if k % self.check_every == 0 or k == self.restart:
                all_conv = bool((self.outer.conv >= 0).all().item())
                if all_conv:
                    break
        self.outer.update(k, self.x, beta=1.0)
        if all_conv and self.residual == "arnoldi":
            # each patch's estimate at the step the back substitution used
            tr = self.outer.resid.cpu().numpy() / self.safe
            res.residual_kind = "arnoldi"
        else:
            B.matvec(self.x, self.r)
            K.axpby(1.0, self.bd, -1.0, self.r)
            tr = self._norms(self.r) / self.safe
            res.residual_kind = "true"
        res.history.append(tr.copy())
        res.cycles += 1
        res.true_residual = tr
        res.success = tr < self.tols

    def solve(self, b_flat, tolerances=None) -> BatchResult:
        B = self.b
        self.set_problem(b_flat, tolerances=tolerances)
        res = BatchResult(solution=self.x, success=np.zeros(B.np, dtype=bool),
                          true_residual=np.ones(B.np))
        for _ in range(self.max_cycles):
            self.cycle(res)
            if res.success.all():
                break
        return res
