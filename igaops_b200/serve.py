"""Continuous batching of elliptic solve requests on one GPU.

Requests arrive over time (each: a patch -- quadrature rules and operator
coefficients, or a callable that computes the coefficients on the device --,
a Dirichlet table, a right-hand side and a tolerance).  The server keeps a
set of *active* requests whose whole state (packed operators, preconditioner
data, current iterate x and right-hand side) stays on the device, and runs
scheduling rounds:

1. admit queued requests in arrival order while their estimated device
   memory fits the HBM budget (and the active set is below ``max_active``);
   an admitted request's operator set-up (coefficients computed on the
   device when given as a callable, packing, fast-diagonalisation set-up)
   happens here, inside its latency;
2. run one restart cycle of the batched mixed-precision FGMRES
   (``igaops_b200.batch``) over every active 3D request at once -- the
   iterate of each request carries over from its previous cycles, so a
   request that joins later simply starts at its own first cycle; while the
   active 3D set stays the same, the cycle's Arnoldi steps run as captured
   CUDA graphs;
3. 2D and space-time (2D+1) requests are solved by a worker thread on its
   own CUDA stream (mixed-precision FGMRES, ``igaops_b200.refine``), so
   their device work overlaps the 3D rounds instead of holding them up;
4. retire requests whose FP64 true residual is below their tolerance
   (their latency is measured from arrival) and free their memory.

A request's result does not depend on the company it keeps: every
per-request quantity (Arnoldi basis, Hessenberg, rotations, tolerance) is
segmented per patch, and the kernels of the batch compute each patch's
values from that patch's data only.
"""
from __future__ import annotations

import math
import queue
import sys
import threading
import time
from dataclasses import dataclass
from typing import List, Optional

import numpy as np
import torch

from . import krylov_ops as K
from ._device import require_cuda, to_device
from .batch import BatchedFGMRES, BatchResult, PatchBatch

__all__ = ["SolveRequest", "SolveServer"]


@dataclass
class SolveRequest:
    """One solve: kind "3d" (stiffness, batched path), "2d" (stiffness) or
    "spacetime" (u_v(time_ders=(0,1)) + gradu_gradv(time_ders=(0,0)), 2D+1)."""

    rid: int
    kind: str
    rules: list
    coefs: object            # stiffness coefficients (device tensor or numpy), or a
                             # callable computing them (called at admission)
    table: np.ndarray        # Dirichlet table of the space directions
    rhs: np.ndarray
    tol: float = 1e-10
    arrival: float = 0.0     # seconds on the server clock
    mass_coefs: object = None  # space-time only: coefficients of the u_v term
    # filled by the server
    solution: Optional[np.ndarray] = None
    success: bool = False
    true_residual: float = float("nan")
    t_admit: float = float("nan")
    t_done: float = float("nan")
    cycles: int = 0
    cancelled: bool = False

    @property
    def latency(self) -> float:
        return self.t_done - self.arrival

    def estimate_bytes(self) -> int:
        """Peak device memory of the request: packed FP64 + FP32 operators,
        the reference-layout coefficients while they are packed, Krylov
        state."""
        N = math.prod(int(q.nbctrlpts) for q in self.rules)
        Nq = math.prod(int(q.nbquadpts) for q in self.rules)
        d = len(self.rules) if self.kind != "spacetime" else len(self.rules) - 1
        per_q = 6 * (8 + 4) if self.kind != "spacetime" else (3 + 1) * (8 + 4)
        per_q += d * d * 8 + 8
        return int(per_q * Nq + 40 * 8 * N + (1 << 20))


class _Active:
    def __init__(self, req: SolveRequest, device):
        self.req = req
        self.x = None
        self.b = None
        self.patch = None
        self.device = device
        self.finished = False    # worker requests: set by the worker thread
        self.ready = False       # 3D requests: patch set up by the preparation thread
        self.error = None


def _materialise(req: SolveRequest) -> bool:
    """Coefficients given as callables are computed now (on the device);
    returns whether any were, so that the caller can drop them once the
    operators are packed."""
    made = False
    if callable(req.coefs):
        req.coefs = req.coefs()
        made = True
    if callable(req.mass_coefs):
        req.mass_coefs = req.mass_coefs()
        made = True
    return made


class SolveServer:
    """Continuous-batching solve loop (see the module docstring)."""

    def __init__(self, hbm_budget_bytes: int, max_active: int = 64, restart: int = 8,
                 inner_iters: int = 0, use_graphs: bool = True,
                 switch_interval: Optional[float] = 2e-4, prep_threads: int = 1):
        self.dev = require_cuda()
        # The 3D loop and the 2D / space-time worker share the interpreter
        # lock.  Each stream synchronisation of one thread hands the lock to
        # the other, and getting it back waits for the other thread's switch
        # interval (5 ms by default): a short interval bounds that wait while
        # run() is active (None keeps the interpreter's setting).
        self.switch_interval = switch_interval
        self.budget = int(hbm_budget_bytes)
        self.max_active = int(max_active)
        self.restart = int(restart)
        self.inner_iters = int(inner_iters)
        self.use_graphs = bool(use_graphs)
        self.queue: List[SolveRequest] = []
        self.active: List[_Active] = []
        self.done: List[SolveRequest] = []
        self.in_use = 0
        self.t0 = None
        self.rounds = 0
        self._batch_key = None   # active 3D set of the cached batch and solver
        self._batch = None
        self._solver = None
        self._batch_rounds = 0   # consecutive rounds the cached batch has served
        self._cancel = set()     # request ids to drop at the next round
        self._lock = threading.Lock()
        self._work: "queue.Queue[Optional[_Active]]" = queue.Queue()
        self._worker = None
        self._prep_q: "queue.Queue[Optional[_Active]]" = queue.Queue()
        # 3D set-up threads (each with its own stream); one overlaps the
        # rounds, a second measured no faster
        self.prep_threads = max(1, int(prep_threads))
        self._prep: List[threading.Thread] = []

    def now(self) -> float:
        return time.perf_counter() - self.t0

    def submit(self, req: SolveRequest):
        """Queue a request.  Refused (the exceptions of the reference's
        argument checks): an unknown kind or a request whose estimated device
        memory exceeds the whole budget (ValueError), a right-hand side with
        NaN / Inf entries (NonFiniteError)."""
        if req.kind not in ("3d", "2d", "spacetime"):
            raise ValueError(f"unknown request kind {req.kind!r}")
        if req.estimate_bytes() > self.budget:
            raise ValueError(f"request {req.rid} needs more than the HBM budget")
        rhs = req.rhs.detach().cpu().numpy() if isinstance(req.rhs, torch.Tensor) else req.rhs
        if not np.all(np.isfinite(np.asarray(rhs, dtype=np.float64))):
            from ._lib import IGA_ERR_NONFINITE, NonFiniteError

            raise NonFiniteError(IGA_ERR_NONFINITE,
                                 f"request {req.rid}: right-hand side holds non-finite values")
        with self._lock:
            self.queue.append(req)

    def cancel(self, rid: int):
        """Drop request `rid`: a queued request leaves the queue, an active one
        leaves the device at the start of the next round (its memory returns
        to the budget).  Either way it is reported done with cancelled=True
        and success=False.  Safe to call from another thread while run()
        serves."""
        with self._lock:
            self._cancel.add(rid)

    def _apply_cancels(self):
        with self._lock:
            ids, self._cancel = self._cancel, set()
        if not ids:
            return
        now = self.now() if self.t0 is not None else 0.0
        keepq = []
        for req in self.queue:
            if req.rid in ids:
                req.cancelled, req.success, req.t_done = True, False, now
                self.done.append(req)
            else:
                keepq.append(req)
        self.queue = keepq
        keep = []
        for a in self.active:
            if a.req.rid in ids:
                a.req.cancelled, a.req.success, a.req.t_done = True, False, now
                self.in_use -= a.req.estimate_bytes()
                self.done.append(a.req)
            else:
                keep.append(a)
        self.active = keep

    # ------------------------------------------------------------ admission
    def _admit(self):
        now = self.now()
        while self.queue and len(self.active) < self.max_active:
            req = self.queue[0]
            if req.arrival > now:
                break
            need = req.estimate_bytes()
            if self.in_use + need > self.budget:
                break
            self.queue.pop(0)
            a = _Active(req, self.dev)
            req.t_admit = self.now()
            self.in_use += need
            self.active.append(a)
            if req.kind == "3d":
                # set up on the preparation thread (its own stream), while
                # the rounds of the requests already set up go on here
                self._ensure_prep()
                self._prep_q.put(a)
            else:
                self._ensure_worker()
                self._work.put(a)

    def _ensure_prep(self):
        self._prep = [t for t in self._prep if t.is_alive()]
        while len(self._prep) < self.prep_threads:
            t = threading.Thread(target=self._prep_loop, daemon=True)
            t.start()
            self._prep.append(t)

    def _prep_loop(self):
        """Sets 3D requests up one after the other (coefficients computed,
        operators packed, FD set up) on a CUDA stream of its own; a request
        joins the 3D rounds once its stream work is complete."""
        torch.cuda.set_device(self.dev)
        stream = torch.cuda.Stream()
        while True:
            a = self._prep_q.get()
            if a is None:
                return
            try:
                if not a.req.cancelled:
                    with torch.cuda.stream(stream):
                        self._prepare_3d(a)
                    stream.synchronize()
            except Exception as e:  # reported by the main loop
                a.error = e
            a.ready = True

    def _prepare_3d(self, a: _Active):
        req = a.req
        made = _materialise(req)
        b = to_device(req.rhs, torch.float64, self.dev).reshape(-1).clone()
        # fixed launch shape: timing every new request shape would add its
        # tuning to the request latency
        patch = PatchBatch.make_patch(req.rules, req.coefs, req.table, nseg=2)
        if made:
            req.coefs = None  # computed here, packed now: free them
        K.mask(b, torch.as_tensor(patch.dirichlet, device=self.dev))
        a.x = torch.zeros_like(b)
        a.b = b
        a.patch = patch

    # ---------------------------------------------------------- 3D batched
    def _round_3d(self, act: List[_Active]):
        # the launch tables and Krylov buffers are rebuilt only when the
        # active set changes (an admission or a retirement); a set that
        # stays for a second round runs its Arnoldi steps as CUDA graphs
        key = tuple(a.req.rid for a in act)
        if key != self._batch_key:
            self._batch = PatchBatch([a.patch for a in act])
            self._solver = None
            self._batch_key = key
            self._batch_rounds = 0
        self._batch_rounds += 1
        if self._solver is None or (self.use_graphs and self._batch_rounds == 2
                                    and not self._solver.use_graphs):
            self._solver = BatchedFGMRES(self._batch, tolerance=1e-10, restart=self.restart,
                                         max_cycles=1, inner_iters=self.inner_iters,
                                         use_graphs=self.use_graphs and self._batch_rounds >= 2)
        B, S = self._batch, self._solver
        off = B.seg.offs_host
        bflat = torch.empty(B.ntot, dtype=torch.float64, device=self.dev)
        xflat = torch.empty(B.ntot, dtype=torch.float64, device=self.dev)
        for i, a in enumerate(act):
            K.copy(a.b, bflat[off[i]:off[i + 1]])
            K.copy(a.x, xflat[off[i]:off[i + 1]])
        S.set_problem(bflat, x0=xflat, tolerances=[a.req.tol for a in act])
        res = BatchResult(solution=S.x, success=np.zeros(B.np, dtype=bool),
                          true_residual=np.ones(B.np))
        S.cycle(res)
        B.check_status()
        for i, a in enumerate(act):
            K.copy(S.x[off[i]:off[i + 1]], a.x)
            a.req.true_residual = float(res.true_residual[i])
            a.req.success = bool(res.success[i])
            a.req.cycles += 1

    # ------------------------------------------- 2D and space-time (worker)
    def _ensure_worker(self):
        if self._worker is None or not self._worker.is_alive():
            self._worker = threading.Thread(target=self._worker_loop, daemon=True)
            self._worker.start()

    def _worker_loop(self):
        """Solves 2D and space-time requests one after the other on a CUDA
        stream of its own, so that their kernels overlap the 3D rounds."""
        torch.cuda.set_device(self.dev)
        stream = torch.cuda.Stream()
        while True:
            a = self._work.get()
            if a is None:
                return
            try:
                if not a.req.cancelled:
                    with torch.cuda.stream(stream):
                        self._solve_single(a)
                    stream.synchronize()
            except Exception as e:  # reported by the main loop
                a.error = e
            a.finished = True

    def _solve_single(self, a: _Active):
        from .refine import EllipticPatchSolver

        req = a.req
        made = _materialise(req)
        b = to_device(req.rhs, torch.float64, self.dev).reshape(-1).clone()
        if req.kind == "2d":
            S = EllipticPatchSolver(req.rules, req.coefs, req.table)
            if made:
                req.coefs = None
            out = S.solve_mixed(b, tolerance=req.tol, precond="fp")
            del S
        else:
            out = _spacetime_solve(req, b)
            if made:
                req.coefs = req.mass_coefs = None
        a.x = to_device(out.solution, torch.float64, self.dev).reshape(-1).cpu()
        req.true_residual = float(out.true_residual)
        req.success = bool(out.success)
        req.cycles += 1

    # ----------------------------------------------------------------- loop
    def run(self, idle_sleep: float = 1e-4, on_round=None) -> List[SolveRequest]:
        """Serve every submitted request (arrival times are relative to the
        start of this call); returns the finished requests (cancelled ones
        included, flagged).  on_round(server), if given, is called before
        each scheduling round."""
        self.queue.sort(key=lambda r: r.arrival)
        self.t0 = time.perf_counter()
        saved_interval = sys.getswitchinterval()
        if self.switch_interval is not None:
            sys.setswitchinterval(self.switch_interval)
        try:
            while True:
                if on_round is not None:
                    on_round(self)
                self._apply_cancels()
                if not (self.queue or self.active):
                    break
                self._admit()
                act3 = [a for a in self.active
                        if a.req.kind == "3d" and a.ready and a.error is None]
                if not act3 and not any(a.finished or (a.ready and a.error is not None)
                                        for a in self.active):
                    time.sleep(idle_sleep)
                    continue
                if act3:
                    self.rounds += 1
                    self._round_3d(act3)
                    torch.cuda.current_stream().synchronize()
                self._retire()
        finally:
            if self._worker is not None and self._worker.is_alive():
                self._work.put(None)
                self._worker.join()
                self._worker = None
            live = [t for t in self._prep if t.is_alive()]
            for _ in live:
                self._prep_q.put(None)
            for t in live:
                t.join()
            self._prep = []
            sys.setswitchinterval(saved_interval)
        return self.done

    def warmup(self, degrees=(2, 3, 4, 5), kinds=("3d", "2d", "spacetime"),
               reserve: bool = True) -> float:
        """Prepares the server before traffic arrives: with ``reserve``, one
        device allocation of the HBM budget (at most 90 % of the free
        memory), released at once into torch's caching allocator, so that
        the requests' large buffers are carved from it instead of each
        calling cudaMalloc (tens of milliseconds for the multi-GB operators
        of a 128^3 patch); then one small request per kind and degree
        through the loop, so that the kernels a stream launches are loaded
        (a kernel's first launch loads its module).  The results are
        discarded and the loop's counters reset.  Returns the seconds it
        took."""
        from .geometry import GeometryOps, precompute_coefficients, unit_cube_ctrlpts
        from .quadrature import WeightedQuadrature

        if self.queue or self.active:
            raise RuntimeError("warmup() runs before the stream: the server has work")
        t0 = time.perf_counter()
        if reserve:
            free, _ = torch.cuda.mem_get_info(self.dev)
            nbytes = min(self.budget, int(0.9 * free))
            while nbytes >= (1 << 30):
                try:
                    block = torch.empty(nbytes, dtype=torch.uint8, device=self.dev)
                    del block
                    break
                except torch.cuda.OutOfMemoryError:
                    nbytes //= 2
        rng = np.random.default_rng(0)
        reqs = []
        for p in degrees:
            q = WeightedQuadrature(p, GeometryOps.make_open_knotvector(p, 6), "2")
            for kind in kinds:
                rid = -(len(reqs) + 1)
                if kind == "spacetime":
                    qt = WeightedQuadrature(p, GeometryOps.make_open_knotvector(p, 4), "2")
                    rl = [q, q, qt]
                    Nq = int(np.prod([r.nbquadpts for r in rl]))
                    C = np.zeros((2, 2, Nq))
                    C[0, 0] = C[1, 1] = 1.0
                    req = SolveRequest(rid, kind, rl, C, np.ones((1, 2, 2), bool), None, 1e-8,
                                       0.0, mass_coefs=np.ones(Nq))
                else:
                    rl = [q] * (3 if kind == "3d" else 2)
                    C = precompute_coefficients(rl, unit_cube_ctrlpts(rl, amplitude=0.05),
                                                mass=False)["stiffness"]
                    req = SolveRequest(rid, kind, rl, C,
                                       np.ones((1, len(rl), 2), bool), None, 1e-8, 0.0)
                N = int(np.prod([r.nbctrlpts for r in rl]))
                req.rhs = rng.uniform(-1.0, 1.0, N)
                reqs.append(req)
        for r in reqs:
            self.submit(r)
        self.run()
        self.done = []
        self.rounds = 0
        self._batch_key = self._batch = self._solver = None
        self._batch_rounds = 0
        torch.cuda.synchronize()
        return time.perf_counter() - t0

    def _retire(self):
        keep = []
        for a in self.active:
            r = a.req
            if r.kind == "3d":
                if a.ready and a.error is not None:
                    raise a.error
                fin = r.success or r.cycles >= 60
            else:
                fin = a.finished
                if fin and a.error is not None:
                    raise a.error
            if fin:
                r.t_done = self.now()
                r.solution = a.x.cpu().numpy() if a.x is not None else None
                self.in_use -= r.estimate_bytes()
                self.done.append(r)
                a.patch = a.x = a.b = None
            else:
                keep.append(a)
        self.active = keep

    @staticmethod
    def stats(done: List[SolveRequest]) -> dict:
        done = [r for r in done if not r.cancelled]
        lat = np.array([r.latency for r in done]) * 1e3
        span = max(r.t_done for r in done) - min(r.arrival for r in done)
        return {
            "requests": len(done),
            "all_converged": bool(all(r.success for r in done)),
            "max_true_residual": float(max(r.true_residual for r in done)),
            "latency_p50_ms": float(np.percentile(lat, 50)),
            "latency_p99_ms": float(np.percentile(lat, 99)),
            "solves_per_s": len(done) / span if span > 0 else float("inf"),
        }


def _spacetime_solve(req: SolveRequest, b: torch.Tensor):
    """Mixed-precision FGMRES on the space-time operator
    u_v(time_ders=(0,1)) + gradu_gradv(time_ders=(0,0)) (the reference's
    examples/performance_matvec_sptm.py:42-57) with the arrowhead space-time
    FD preconditioner (SingleFD("spacetime"))."""
    from .fastdiag import SingleFD
    from .operators import MFOperator
    from .refine import MixedPrecisionFGMRES

    rules = list(req.rules)
    ops = {}
    for dt in (torch.float64, torch.float32):
        ops[dt] = (MFOperator(rules, req.mass_coefs, "u_v", (0, 1), dtype=dt),
                   MFOperator(rules, req.coefs, "gradu_gradv", (0, 0), dtype=dt))
    tmp = {}

    def apply(x, y):
        M, Kst = ops[x.dtype]
        M.apply_into(x, y)
        t = tmp.get(x.dtype)
        if t is None:
            t = tmp[x.dtype] = torch.empty_like(x)
        Kst.apply_into(x, t)
        K.axpby(1.0, t, 1.0, y)

    fd = SingleFD("spacetime")
    fd.compute_space_eigendecomposition(rules[:-1], req.table)
    fd.compute_time_schurdecomposition(rules[-1])
    fd.update_space_eigenvalues([0.0, 1.0])
    stfd = fd.sptm_preconditioner

    def prec(x, y):
        stfd.apply_device(x, y)

    N = b.numel()
    free = np.asarray(stfd.sptm_free_nodes[0], dtype=np.int64)
    mask = np.ones(N, dtype=bool)
    mask[free] = False
    dirichlet = torch.as_tensor(np.nonzero(mask)[0], device=b.device)
    solver = MixedPrecisionFGMRES(req.tol, maxiters=80, restart=40, inner_iters=0)
    return solver.solve(apply, b, apply, prec, cleandod=dirichlet)
