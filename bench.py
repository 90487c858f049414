"""Benchmark of the matrix-free weighted-quadrature hot path on B200.

Workload (one GPU): 3D, degree 3, 128^3 elements (131^3 = 2,248,091 DOFs,
389^3 = 58,863,869 quadrature points), weighted quadrature type "2",
unit-cube control net with every control point displaced by
0.1*h*sin(2 pi x) sin(2 pi y) sin(2 pi z), isotropic coefficient 1
(stiffness coefficients det J * J^+ J^+T and mass coefficient det J computed on
the device), seeded random input vectors.

One step = one FP64 stiffness matvec + one FP64 mass matvec (the plain
method, same precision as the reference) on an input vector from a ring of
eight.  metric: matvec throughput in GDOF/s = DOFs / step time.  The launch
shape (segments of the streamed direction) is picked by the autotuner before
timing, and so is the kernel (the pencil kernel or the FP64 tensor-core
tile kernel, whichever the autotuner measures faster).  "e2e": the same steps through the operator API with the input
copied in from pinned host memory and both results copied out every step;
the copies run on two copy streams, overlapping the neighbouring steps'
matvecs.  At one GPU the line also carries solve-level numbers ("solves"):
96^3 single-patch solves per degree (mixed precision vs plain FP64), 512
batched patches in memory waves and a degree-3 batch of 128 (batched mixed
precision, FP64 on the same batched engine, and the plain FP64 path one patch
after the other) and a 1000-request Poisson-arrival serving sample per rate.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl {b200,reference}]
Multi-GPU (torchrun): every rank runs the same patch (independent replicas,
weak scaling, no collective on the data path); time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

DEGREE = 3
NBEL = 128
WORKLOAD = "mf_matvec_3d_p3_ne{ne}_perturbed_cube"
METRIC = "MF matvec GDOF/s (FP64 stiffness+mass per step)"


def _peaks():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic_per_launch():
    """DRAM bytes (read+write) per stiffness launch from the committed ncu
    summary, if present (see profiles/)."""
    f = ROOT / "profiles" / "mf_stiffness_f64_ne128_traffic.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith("bytes_per_launch_full_size:"):
            return float(line.split(":", 1)[1])
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons during the timed region."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"iga_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        # nvidia-smi takes a while to start: wait (bounded) for its first two
        # samples so that the timed region that follows is covered
        t_end = time.time() + 10.0
        while time.time() < t_end and self.proc.poll() is None:
            try:
                if self.path.read_text().count("\n") >= 2:
                    break
            except OSError:
                pass
            time.sleep(0.05)

    def stop(self, t0: float | None = None, t1: float | None = None):
        """Median SM clock and active throttle reasons over the samples taken
        between host wall times t0 and t1 (all samples when not given)."""
        import datetime as _dt

        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                ts = _dt.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                f_sm, f_max = float(parts[2]), float(parts[3])
            except ValueError:
                continue
            if t0 is not None and not (t0 <= ts <= t1):
                continue
            sm.append(f_sm)
            smax.append(f_max)
            for nm, v in zip(names, parts[6:10]):
                if v.lower() == "active":
                    reasons.add(nm)
        self.path.unlink(missing_ok=True)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(smax) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


def build_problem(ne=NBEL, p=DEGREE):
    import torch

    from igaops_b200 import GeometryOps, WeightedQuadrature, precompute_coefficients, unit_cube_ctrlpts

    kv = GeometryOps.make_open_knotvector(p, ne)
    q = WeightedQuadrature(p, kv, "2")
    rules = [q, q, q]
    ctrl = unit_cube_ctrlpts(rules, amplitude=0.1)
    coefs = precompute_coefficients(rules, ctrl)
    torch.cuda.synchronize()
    return rules, coefs


# ---------------------------------------------------------------- CPU legs
# The oracle (numpy restatement of the reference path) on the reference's own
# 1D factors of the benchmark rule (tests/golden/bench_rule.npz, written by
# tests/golden/make_golden.py from the unmodified reference).  Neither leg
# imports igaops_b200 or loads its library.  Coefficients: the reference's
# full (3, 3, Nq) stiffness layout and (Nq,) mass, synthetic values of the
# perturbed cube's magnitude (identity plus a small seeded perturbation,
# symmetric), input vector N(0, 1) from seed 0.
def _cpu_coefs(npts: int, seed: int):
    rng = np.random.default_rng(1000 + seed)
    C = np.empty((3, 3, npts))
    for i in range(3):
        C[i, i] = 1.0 + 0.005 * rng.standard_normal(npts)
        for j in range(i):
            C[i, j] = 0.001 * rng.standard_normal(npts)
            C[j, i] = C[i, j]
    m = 1.0 + 0.005 * rng.standard_normal(npts)
    return C, m


def _cpu_slab(nslab: int, slab: int):
    """Rules, coefficients and input of slab `slab` of `nslab` (contiguous
    ranges of quadrature points of the slowest direction), and the range of
    control planes of that direction its product touches."""
    from oracle.rules import bench_rule, slab_rule

    q = bench_rule()
    nq = q.nbquadpts
    cuts = np.linspace(0, nq, nslab + 1).astype(int)
    q0, q1 = int(cuts[slab]), int(cuts[slab + 1])
    rl = [q, q, slab_rule(q, q0, q1)]
    rows = np.unique(np.concatenate([W.tocsc().indices for W in rl[2].weights]))
    p0, p1 = int(rows.min()), int(rows.max()) + 1
    C, m = _cpu_coefs(nq * nq * (q1 - q0), slab)
    x = np.random.default_rng(0).standard_normal(q.nbctrlpts ** 3)
    return rl, C, m, x, (p0, p1), q.nbctrlpts


def _cpu_pair(rl, C, m, x):
    from oracle import mf as omf

    return omf.mf_gradu_gradv(rl, C, x), omf.mf_u_v(rl, m, x)


def _ref_worker(conn, nslab: int, slab: int):
    """Reference-arm worker: owns one slab, computes its stiffness and mass
    products on request and returns the touched control planes."""
    rl, C, m, x, (p0, p1), n = _cpu_slab(nslab, slab)
    plane = n * n
    conn.send(("ready", p0, p1))
    while True:
        msg = conn.recv()
        if msg is None:
            break
        ys, ym = _cpu_pair(rl, C, m, x)
        conn.send_bytes(np.ascontiguousarray(ys[p0 * plane:p1 * plane]).tobytes())
        conn.send_bytes(np.ascontiguousarray(ym[p0 * plane:p1 * plane]).tobytes())
    conn.close()


def cpu_sample(nslab: int = 16, reps: int = 3):
    """The bench line's cpu_baseline: one host process runs the oracle's
    stiffness + mass pair on slab 0 of `nslab` of the 128^3 workload (1/nslab
    of its quadrature points), at numpy's default threading and again limited
    to one thread; DOF/s counted as N x (slab points / all points)."""
    from threadpoolctl import threadpool_limits

    rl, C, m, x, _, n = _cpu_slab(nslab, 0)
    N = n ** 3
    frac = rl[2].nbquadpts / rl[0].nbquadpts
    _cpu_pair(rl, C, m, x)  # warm-up
    out = {}
    for mode in ("default", "single"):
        if mode == "single":
            lim = threadpool_limits(1)
        t0 = time.perf_counter()
        for _ in range(reps):
            _cpu_pair(rl, C, m, x)
        dt = (time.perf_counter() - t0) / reps
        if mode == "single":
            lim.unregister()
        out[mode] = (N * frac / dt, dt)
    return out, N, frac


def run_reference(args):
    """--impl reference: the reference algorithm (the oracle's numpy
    restatement on the reference's own 1D factors; the reference package
    itself imports geomdl, which cannot be installed here) on the full
    benchmark configuration (3D p3 128^3) using every host core: one
    single-threaded worker process per core, each owning a slab of the
    quadrature points of the slowest direction; a step is one full stiffness
    + mass matvec pair -- every worker's slab product, and the parent's sum
    of the slabs' control planes into the two result vectors.
    value = DOFs / step time."""
    import multiprocessing as mp

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cores = len(os.sched_getaffinity(0))
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[k] = "1"
    ctx = mp.get_context("spawn")
    pipes, procs, ranges = [], [], []
    t_setup = time.perf_counter()
    for s in range(cores):
        a, b = ctx.Pipe()
        pr = ctx.Process(target=_ref_worker, args=(b, cores, s), daemon=True)
        pr.start()
        pipes.append(a)
        procs.append(pr)
    for a in pipes:
        _, p0, p1 = a.recv()
        ranges.append((p0, p1))
    t_setup = time.perf_counter() - t_setup
    from oracle.rules import bench_rule

    n = bench_rule().nbctrlpts
    N, plane = n ** 3, n * n
    ys = np.zeros(N)
    ym = np.zeros(N)

    def step():
        for a in pipes:
            a.send(1)
        ys[:] = 0.0
        ym[:] = 0.0
        for a, (p0, p1) in zip(pipes, ranges):
            ys[p0 * plane:p1 * plane] += np.frombuffer(a.recv_bytes(), dtype=np.float64)
            ym[p0 * plane:p1 * plane] += np.frombuffer(a.recv_bytes(), dtype=np.float64)

    for _ in range(args.warmup):
        step()
    steps = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s0 = time.perf_counter()
        step()
        steps.append(time.perf_counter() - s0)
    total = time.perf_counter() - t0
    for a in pipes:
        a.send(None)
    for pr in procs:
        pr.join(timeout=30)
    mean_dt = sum(steps) / len(steps)
    value = N / mean_dt / 1e9
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "GDOF/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": mean_dt * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD.format(ne=NBEL), "dofs": N,
                   "quadrature_points": bench_rule().nbquadpts ** 3,
                   "sample": f"full workload every step, split over {cores} worker processes "
                             f"by slabs of quadrature points"},
        "cpu_baseline": {"value": value, "unit": "GDOF/s", "cores": cores, "kind": "port",
                         "sample": f"oracle stiffness+mass matvec pair on the full 128^3 p3 "
                                   f"configuration ({N} DOFs), {cores} single-threaded worker "
                                   f"processes (one slab of quadrature points each, results "
                                   f"summed by the parent), {args.steps} steps in {total:.1f} s, "
                                   f"set-up {t_setup:.1f} s"},
        "e2e": {"value": value, "unit": "GDOF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def _best_ms(fn, reps=3):
    import torch

    fn()
    torch.cuda.synchronize()
    best, out = float("inf"), None
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        best = min(best, (time.perf_counter() - t0) * 1e3)
    return best, out


def solve_single(ne: int = 96, degrees=(2, 3, 4, 5)):
    """One elliptic solve per degree on the perturbed cube (all faces
    Dirichlet, RHS U(-1,1) seed 0): the mixed-precision FGMRES (FP32/BF16
    inner, FP64 outer) against the plain FP64 GPU path (FD-preconditioned
    GMRES, FP64 matvec and FD), both to 1e-10 and both stopping on their
    FP64 Arnoldi residual estimate (the reference GMRES's rule); wall time
    of a whole solve, best of 3 after one warm-up; both true residuals are
    recomputed in FP64 after the timed solves."""
    import torch

    from igaops_b200 import GeometryOps, WeightedQuadrature, precompute_coefficients, unit_cube_ctrlpts
    from igaops_b200.refine import EllipticPatchSolver

    out = {}
    for p in degrees:
        q = WeightedQuadrature(p, GeometryOps.make_open_knotvector(p, ne), "2")
        rl = [q, q, q]
        co = precompute_coefficients(rl, unit_cube_ctrlpts(rl, amplitude=0.1))
        S = EllipticPatchSolver(rl, co["stiffness"], np.ones((1, 3, 2), dtype=bool))
        del co
        rng = np.random.default_rng(0)
        b = np.zeros(S.N)
        b[S.free] = rng.uniform(-1.0, 1.0, S.free.size)
        bd = torch.from_numpy(b).cuda()
        t64, r64 = _best_ms(lambda: S.solve_fp64(bd))
        tmx, rmx = _best_ms(lambda: S.solve_mixed(bd, residual="arnoldi"))
        x64 = r64.solution
        xmx = rmx.solution
        err = float(torch.linalg.vector_norm(xmx - x64) / torch.linalg.vector_norm(x64))
        out[f"p{p}"] = {
            "dofs": S.N,
            "fp64_ms": round(t64, 3), "fp64_iterations": len(r64.residual) - 1,
            "fp64_true_residual": S.true_residual(x64, bd),
            "mixed_ms": round(tmx, 3), "mixed_iterations": rmx.outer_iterations,
            "mixed_true_residual": S.true_residual(xmx, bd),
            "mixed_arnoldi_residual": rmx.true_residual,
            "mixed_vs_fp64_solution_rel_diff": err,
            "speedup": round(t64 / tmx, 3),
        }
        del S
        torch.cuda.empty_cache()
    return out


def _patch_spec(i: int, degrees=(2, 3, 4)):
    """Patch i of the batched configuration: elements per direction U{16..96},
    degree uniform over `degrees`, displacement amplitude and right-hand side
    seeded by i."""
    r = np.random.default_rng(i)
    ne, p = int(r.integers(16, 97)), int(degrees[int(r.integers(0, len(degrees)))])
    amp = 0.05 + 0.1 * r.random()
    return ne, p, amp


def solve_batched(npatch: int = 512, degrees=(2, 3, 4), budget_gb: float = 100.0):
    """Independent 3D patches (elements per direction U{16..96}, degree
    uniform over `degrees`, own displacement amplitude and RHS, seeded per
    patch) solved to 1e-10 in waves that fit `budget_gb` of device memory
    (the packed FP64 + FP32 operators of 512 patches need about 285 GB):

    * mixed: batched mixed-precision FGMRES (FP64 outer, BF16 tensor-core FD
      preconditioner; one launch per operator for all patches of a wave,
      graph-captured Arnoldi steps);
    * fp64_batched: the same engine in FP64 (FP64 FD apply per patch);
    * fp64_sequential: the plain FP64 GPU path (the reference's GMRES with
      FP64 matvec and FD, host least squares) one patch after the other.

    Wall times of each wave's solve after one untimed solve of the same wave
    (graph capture), summed over the waves."""
    import torch

    from igaops_b200 import GeometryOps, WeightedQuadrature, precompute_coefficients, unit_cube_ctrlpts
    from igaops_b200.batch import BatchedFGMRES, BatchResult, PatchBatch
    from igaops_b200.solvers import LinearSolver

    rule_cache = {}

    def rule(p, ne):
        if (p, ne) not in rule_cache:
            rule_cache[(p, ne)] = WeightedQuadrature(p, GeometryOps.make_open_knotvector(p, ne), "2")
        return rule_cache[(p, ne)]

    specs = [_patch_spec(i, degrees) for i in range(npatch)]
    waves, cur, cur_b = [], [], 0.0
    for i, (ne, p, amp) in enumerate(specs):
        est = 72.0 * (3 * ne + p + 1) ** 3 + 200.0 * (ne + p) ** 3
        if cur and cur_b + est > budget_gb * 1e9:
            waves.append(cur)
            cur, cur_b = [], 0.0
        cur.append(i)
        cur_b += est
    waves.append(cur)
    t_setup = 0.0
    tot = {"mixed": 0.0, "fp64_batched": 0.0, "fp64_sequential": 0.0}
    lat, max_res, max_diff, steps, dofs = [], 0.0, 0.0, {"mixed": 0, "fp64_batched": 0}, 0
    ok = {"mixed": True, "fp64_batched": True, "fp64_sequential": True}
    for wave in waves:
        s0 = time.perf_counter()
        pats = []
        for i in wave:
            ne, p, amp = specs[i]
            q = rule(p, ne)
            rl = [q, q, q]
            co = precompute_coefficients(rl, unit_cube_ctrlpts(rl, amplitude=amp), mass=False)
            pats.append(PatchBatch.make_patch(rl, co["stiffness"], np.ones((1, 3, 2), dtype=bool),
                                              nseg="heuristic"))
            del co
        B = PatchBatch(pats)
        del pats
        parts = []
        for k, pt in enumerate(B.patches):
            r = np.random.default_rng(1000 + wave[k])
            b = np.zeros(pt.N)
            b[pt.free] = r.uniform(-1.0, 1.0, pt.free.size)
            parts.append(b)
        bflat = B.join(parts)
        torch.cuda.synchronize()
        t_setup += time.perf_counter() - s0
        dofs += B.ntot
        sols = {}
        for arm in ("mixed", "fp64_batched"):
            S = BatchedFGMRES(B, tolerance=1e-10, restart=12, inner_iters=0,
                              precision="mixed" if arm == "mixed" else "fp64")
            S.solve(bflat)  # graph capture
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res = S.solve(bflat)
            torch.cuda.synchronize()
            tot[arm] += time.perf_counter() - t0
            B.check_status()
            ok[arm] &= bool(res.success.all())
            max_res = max(max_res, float(res.true_residual.max()))
            steps[arm] += res.outer_steps
            sols[arm] = B.split(res.solution)
            del S
        # plain FP64 path, one patch after the other, per-patch latencies
        bs = B.split(bflat)
        torch.cuda.synchronize()
        for pt, bp, xm in zip(B.patches, bs, sols["mixed"]):
            s1 = time.perf_counter()
            bd = torch.from_numpy(np.ascontiguousarray(bp)).cuda()

            def A(x, pt=pt):
                y = torch.empty_like(x)
                pt.K64.apply_into(x, y)
                return y

            def P(x, pt=pt):
                y = torch.empty_like(x)
                pt.fd.space_preconditioner.apply_device(x, y)
                return y

            ls = LinearSolver(1e-10, 60, cleandod=[int(i) for i in pt.dirichlet],
                              linear_type="gmres", verbose=False)
            out = ls.solve(A, bd, P)
            torch.cuda.synchronize()
            lat.append((time.perf_counter() - s1) * 1e3)
            ok["fp64_sequential"] &= bool(out.success)
            xs = out.solution.cpu().numpy()
            max_diff = max(max_diff, float(np.linalg.norm(xm - xs) / np.linalg.norm(xs)))
        tot["fp64_sequential"] += sum(lat[-len(wave):]) * 1e-3
        del B, bflat
        torch.cuda.empty_cache()
    return {
        "patches": npatch, "degrees": list(degrees), "dofs_total": dofs, "waves": len(waves),
        "wave_budget_gb": budget_gb, "setup_s": round(t_setup, 2),
        "mixed_s": round(tot["mixed"], 4), "mixed_solves_per_s": npatch / tot["mixed"],
        "fp64_batched_s": round(tot["fp64_batched"], 4),
        "fp64_batched_solves_per_s": npatch / tot["fp64_batched"],
        "fp64_sequential_s": round(tot["fp64_sequential"], 4),
        "fp64_sequential_solves_per_s": npatch / tot["fp64_sequential"],
        "speedup_vs_fp64_sequential": round(tot["fp64_sequential"] / tot["mixed"], 3),
        "speedup_vs_fp64_batched": round(tot["fp64_batched"] / tot["mixed"], 3),
        "outer_steps": steps, "all_converged": ok,
        "max_true_residual": max_res,
        "max_solution_rel_diff_mixed_vs_fp64": max_diff,
        "fp64_sequential_latency_p50_ms": float(np.percentile(lat, 50)),
        "fp64_sequential_latency_p99_ms": float(np.percentile(lat, 99)),
        "mixed_wave_latency_ms": round(1e3 * tot["mixed"] / len(waves), 2),
    }


NE_GRID = (8, 10, 12, 14, 16, 20, 24, 28, 32, 40, 48, 56, 64, 80, 96, 128)


def serve_sample(nreq: int = 1000, rates=(50.0, 200.0), seed: int = 0, keep_requests=None,
                 server_kwargs=None):
    """Poisson-arrival stream of solve requests through the continuous-
    batching server, per mean arrival rate: p50/p99 latency from arrival to
    result and solves/s.  Mix: 60 % 3D (elements per direction log-uniform
    on a grid of 16 values in 8..128), 25 % 2D (same grid), 15 % space-time
    2D+1 (8..24 in space); degree 2..5, tolerance log-uniform in
    [1e-10, 1e-8].  The operators' coefficients are computed on the device
    when a request is admitted (inside its latency); the 1D quadrature
    rules are built once per (degree, elements) before the stream starts
    (host set-up, excluded from the latencies)."""
    import torch

    from igaops_b200 import GeometryOps, WeightedQuadrature, precompute_coefficients
    from igaops_b200.fastdiag import clear_pencil_cache
    from igaops_b200.serve import SolveRequest, SolveServer

    cache = {}

    def rule(p, ne):
        if (p, ne) not in cache:
            cache[(p, ne)] = WeightedQuadrature(p, GeometryOps.make_open_knotvector(p, ne), "2")
        return cache[(p, ne)]

    def net_device(rl, amp):
        # the displaced Greville net of unit_cube_ctrlpts, built on the device
        g = [torch.from_numpy(GeometryOps.evaluate_greville(q.degree, q.knotvector)).cuda()
             for q in rl]
        grids = torch.meshgrid(*g[::-1], indexing="ij")[::-1]
        coords = [gk.reshape(-1) for gk in grids]
        h = 1.0 / (len(rl[0].unique_kv) - 1)
        disp = torch.sin(2 * np.pi * coords[0])
        for c in coords[1:]:
            disp = disp * torch.sin(2 * np.pi * c)
        disp = disp * (amp * h)
        return torch.stack([c + disp for c in coords])

    def coef_fn(rl, amp):
        return lambda: precompute_coefficients(rl, net_device(rl, amp), mass=False)["stiffness"]

    def log_grid(rng, lo, hi):
        grid = [g for g in NE_GRID if lo <= g <= hi]
        return int(grid[int(rng.integers(0, len(grid)))])

    t_rules = time.perf_counter()
    streams = {}
    for rate in rates:
        rng = np.random.default_rng(seed)
        t = 0.0
        reqs = []
        for rid in range(nreq):
            t += rng.exponential(1.0 / rate)
            u = rng.random()
            p = int(rng.integers(2, 6))
            tol = float(10 ** rng.uniform(-10, -8))
            if u < 0.6:
                ne = log_grid(rng, 8, 128)
                q = rule(p, ne)
                rl = [q, q, q]
                req = SolveRequest(rid, "3d", rl, coef_fn(rl, 0.1 * rng.random()),
                                   np.ones((1, 3, 2), bool), None, tol, t)
            elif u < 0.85:
                ne = log_grid(rng, 8, 128)
                q = rule(p, ne)
                rl = [q, q]
                req = SolveRequest(rid, "2d", rl, coef_fn(rl, 0.1 * rng.random()),
                                   np.ones((1, 2, 2), bool), None, tol, t)
            else:
                ne = log_grid(rng, 8, 24)
                qs, qt = rule(p, ne), rule(p, max(4, ne // 2))
                rl = [qs, qs, qt]
                Nq = int(np.prod([q.nbquadpts for q in rl]))
                C = np.zeros((2, 2, Nq))
                C[0, 0] = C[1, 1] = 1.0
                req = SolveRequest(rid, "spacetime", rl, C, np.ones((1, 2, 2), bool), None, tol, t,
                                   mass_coefs=np.ones(Nq))
            N = int(np.prod([q.nbctrlpts for q in req.rules]))
            req.rhs = rng.uniform(-1.0, 1.0, N)
            reqs.append(req)
        streams[rate] = reqs
    t_rules = time.perf_counter() - t_rules
    out = {}
    for rate, reqs in streams.items():
        torch.cuda.synchronize()
        # every rate replays the same kind of stream: start each from an
        # empty preconditioner set-up cache so that no rate profits from
        # the requests of another
        clear_pencil_cache()
        srv = SolveServer(hbm_budget_bytes=96 << 30, max_active=48, restart=8,
                          **(server_kwargs or {}))
        # one small request per kind and degree before the stream (kernel
        # modules load on first launch), outside the latencies
        t_warm = srv.warmup()
        clear_pencil_cache()
        for r in reqs:
            srv.submit(r)
        done = srv.run()
        if keep_requests is not None:
            keep_requests[rate] = done  # the finished requests, for analysis
        st = SolveServer.stats(done)
        st["rounds_3d"] = srv.rounds
        st["warmup_s"] = round(t_warm, 3)
        st["kinds"] = {k: sum(1 for r in done if r.kind == k) for k in ("3d", "2d", "spacetime")}
        st["max_3d_elements"] = max(int(r.rules[0].nbctrlpts) - int(r.rules[0].degree)
                                    for r in done if r.kind == "3d")
        out[f"rate_{rate:g}_per_s"] = st
        del srv, done
        torch.cuda.empty_cache()
    out["note"] = (f"{nreq} requests per rate; 3D and 2D elements per direction log-uniform on "
                   f"{list(NE_GRID)}, space-time 8..24 in space; coefficients computed on the "
                   f"device at admission (in the latency); the 1D rules of all (degree, "
                   f"elements) pairs were built beforehand in {t_rules:.1f} s of host time "
                   f"(not in the latency); before each rate the server is warmed up with "
                   f"one small request per kind and degree (first kernel launches; not in "
                   f"the latencies) and the preconditioner set-up cache is then emptied")
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-solves", action="store_true")
    ap.add_argument("--batch-patches", type=int, default=512)
    ap.add_argument("--ne", type=int, default=NBEL)
    ap.add_argument("--solves-only", action="store_true",
                    help="run only the single-patch solves (for profiling) and print them")
    ap.add_argument("--solve-degrees", default="2,3,4,5")
    ap.add_argument("--batched-only", action="store_true",
                    help="run only the batched-patch solves and print them")
    ap.add_argument("--serving-only", action="store_true",
                    help="run only the serving sample and print it")
    ap.add_argument("--serve-requests", type=int, default=1000)
    ap.add_argument("--solve-ne", type=int, default=96)
    ap.add_argument("--kernel", choices=["auto", "pencil", "tile"], default="auto",
                    help="matvec kernel of the timed steps: chosen per operator by the "
                         "autotuner (default), the pencil kernel, or the FP64 tensor-core "
                         "tile kernel")
    ap.add_argument("--nseg", default="auto",
                    help="segment counts of the pencil kernel: 'auto' (timed by the "
                         "autotuner) or 'S,M' for the stiffness and mass operators (no "
                         "timing launches, so a profiler sees the steps' launches first)")
    args = ap.parse_args(argv)
    if args.nseg != "auto":
        try:
            args.nseg = tuple(int(v) for v in args.nseg.split(","))
        except ValueError:
            ap.error("--nseg must be 'auto' or 'S,M'")
        if len(args.nseg) != 2 or min(args.nseg) < 1:
            ap.error("--nseg must be 'auto' or 'S,M' with counts >= 1")
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)
    if args.serving_only:
        print(json.dumps({"serving": serve_sample(args.serve_requests)}))
        return 0
    if args.batched_only:
        print(json.dumps({"batched": solve_batched(args.batch_patches)}))
        return 0
    if args.solves_only:
        degs = tuple(int(d) for d in args.solve_degrees.split(","))
        print(json.dumps({f"single_patch_{args.solve_ne}": solve_single(args.solve_ne, degs)}))
        return 0

    import torch

    from igaops_b200 import MFOperator
    from igaops_b200.replicas import finish, init_group, job_throughput, max_over_ranks, rank_env

    info = rank_env()
    world, rank, local = info.world, info.rank, info.local
    torch.cuda.set_device(local)
    dist = init_group(info, "nccl", timeout_s=120.0)

    rules, coefs = build_problem(args.ne)
    # kernel (pencil or tile) and launch shape (segments of the streamed
    # direction) chosen by the autotuner, timed on these operators
    nseg_k, nseg_m = ("auto", "auto") if args.nseg == "auto" else args.nseg
    stiff = MFOperator(rules, coefs["stiffness"], "gradu_gradv", dtype=torch.float64,
                       nseg=nseg_k, kernel=args.kernel)
    mass = MFOperator(rules, coefs["mass"], "u_v", dtype=torch.float64, nseg=nseg_m,
                      kernel=args.kernel)
    del coefs
    from igaops_b200 import tune

    tune_decisions = tune.decisions()
    N = stiff.N
    Nq = stiff.Nq
    K, W = args.steps, args.warmup
    gen = torch.Generator(device="cuda").manual_seed(1234 + rank)
    RING = 8
    xs = torch.randn((RING, N), dtype=torch.float64, device="cuda", generator=gen)
    ys = torch.empty((2, N), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()

    def step(i):
        stiff.apply_into(xs[i % RING], ys[0])
        mass.apply_into(xs[i % RING], ys[1])

    for i in range(W):
        step(i)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(K)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    w0 = time.time()
    t_start.record(stream)
    for i in range(K):
        ev[i][0].record(stream)
        stiff.apply_into(xs[(W + i) % RING], ys[0])
        ev[i][1].record(stream)
        mass.apply_into(xs[(W + i) % RING], ys[1])
    t_end.record(stream)
    torch.cuda.synchronize()
    w1 = time.time()
    # a short timed region (20 steps take about 30 ms) holds one or two
    # samples at most: keep the same steps running, untimed, for 0.5 s more
    # so that the clock record covers the kernel under the same load
    i = 0
    while time.time() - w1 < 0.5:
        for _ in range(16):
            step(W + K + i)
            i += 1
        torch.cuda.synchronize()
    w2 = time.time()
    if dist:
        dist.barrier()
    clocks = sampler.stop(w0, w2)
    clocks["window"] = (f"timed steps ({(w1 - w0) * 1e3:.0f} ms) and {(w2 - w1) * 1e3:.0f} ms "
                        f"of the same steps untimed right after; sampled every 20 ms")
    (ms_total,) = max_over_ranks([t_start.elapsed_time(t_end)], dist)
    stiff.plan.check_status()
    mass.plan.check_status()
    ms_step = ms_total / K
    value = job_throughput(N, world, ms_step)
    ms_stiff = sum(a.elapsed_time(b) for a, b in ev) / K
    alg_bytes = stiff.algorithmic_bytes()
    peak, peak_kind = _peaks()
    achieved = alg_bytes / (ms_stiff * 1e-3) / 1e9
    # the committed traffic figure is the pencil kernel's at this size
    traffic = _traffic_per_launch() if not stiff.tiled and args.ne == NBEL else None

    # ---- end to end through the public API with host buffers: every step
    # copies its input in from pinned host memory and its two results out;
    # the copies run on their own streams, so the H2D of step i+1 and the D2H
    # of step i-1 overlap the matvecs of step i (two buffers per side)
    NB = 2
    xh = torch.empty((NB, N), dtype=torch.float64).pin_memory()
    xh.copy_(xs[:NB].cpu())
    yh = torch.empty((NB, 2, N), dtype=torch.float64).pin_memory()
    xd = torch.empty((NB, N), dtype=torch.float64, device="cuda")
    yd = torch.empty((NB, 2, N), dtype=torch.float64, device="cuda")
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(NB)]
    ev_comp = [torch.cuda.Event() for _ in range(NB)]
    ev_out = [torch.cuda.Event() for _ in range(NB)]

    def e2e_step(i):
        b = i % NB
        with torch.cuda.stream(s_in):
            if i >= NB:
                s_in.wait_event(ev_comp[b])  # the matvecs of step i-NB read xd[b]
            xd[b].copy_(xh[b], non_blocking=True)
            ev_in[b].record(s_in)
        stream.wait_event(ev_in[b])
        if i >= NB:
            stream.wait_event(ev_out[b])  # yd[b] of step i-NB is on the host
        stiff.apply_into(xd[b], yd[b, 0])
        mass.apply_into(xd[b], yd[b, 1])
        ev_comp[b].record(stream)
        with torch.cuda.stream(s_out):
            s_out.wait_event(ev_comp[b])
            yh[b].copy_(yd[b], non_blocking=True)
            ev_out[b].record(s_out)

    for i in range(W):
        e2e_step(i)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s_in.wait_event(e0)
    s_out.wait_event(e0)
    for i in range(W, W + K):
        e2e_step(i)
    for b in range(NB):
        stream.wait_event(ev_out[b])
    e1.record(stream)
    torch.cuda.synchronize()
    (ms_e2e,) = max_over_ranks([e0.elapsed_time(e1) / K], dist)
    e2e_value = job_throughput(N, world, ms_e2e)

    line = {
        "metric": METRIC,
        "value": value,
        "unit": "GDOF/s",
        "n_gpus": world,
        "steps": K,
        "warmup": W,
        "ms_per_step": ms_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {
            "workload": WORKLOAD.format(ne=args.ne),
            "dofs": N,
            "quadrature_points": Nq,
            "degree": DEGREE,
            "elements": [args.ne] * 3,
            "quadrature": "weighted, type 2, endpoint",
            "l2": f"inputs larger than L2 (stiffness coefficients {Nq * 6 * 8 / 1e9:.2f} GB FP64)",
            "parallelism": f"replicas x{world}" if world > 1 else "single patch",
            "segments": ({"stiffness": stiff.plan.nseg, "mass": mass.plan.nseg,
                          "chosen_by": ("igaops_b200.tune (timed per shape)"
                                        if args.nseg == "auto" else "fixed (--nseg)")}
                         if not stiff.tiled else "one persistent CTA per SM"),
            "kernel": {"requested": args.kernel,
                       "stiffness": "tile" if stiff.tiled else "pencil",
                       "mass": "tile" if mass.tiled else "pencil",
                       "autotuner": tune_decisions},
        },
        "gpu_launches": 2 * K,
        "e2e": {"value": e2e_value, "unit": "GDOF/s", "h2d_bytes_per_step": N * 8,
                "d2h_bytes_per_step": 2 * N * 8,
                "copies": "pinned host buffers; H2D / D2H on their own streams, "
                          "overlapping the neighbouring steps' matvecs"},
        "roofline": {
            "kernel": ("mf3d_kernel (fused stiffness, FP64)" if not stiff.tiled
                       else "mf3d_tile_kernel (tensor-core tile stiffness, FP64)"),
            "bound": "hbm",
            "achieved": achieved,
            "peak": peak,
            "peak_kind": peak_kind,
            "unit": "GB/s",
            "frac": achieved / peak,
            "traffic": traffic,
            "algorithmic_bytes": alg_bytes,
            "ms_per_launch": ms_stiff,
        },
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb, Ns, frac = cpu_sample()
        line["cpu_baseline"] = {
            "value": cb["default"][0] / 1e9, "unit": "GDOF/s", "cores": 1, "kind": "port",
            "single_thread_value": cb["single"][0] / 1e9,
            "sample": f"oracle (numpy restatement of the reference, on the reference's own 1D "
                      f"factors) stiffness+mass matvec pair on 1/16 of the 128^3 p3 workload's "
                      f"quadrature points (one slab of the slowest direction; {Ns} DOFs x "
                      f"{frac:.4f}), one process: {cb['default'][1]:.2f} s per pair at numpy's "
                      f"default threading (value), {cb['single'][1]:.2f} s limited to one "
                      f"thread (single_thread_value); mean of 3",
        }
    if rank == 0 and world == 1 and not args.no_solves:
        # solve-level numbers (single patch at 96^3 per degree; batched patches)
        line["solves"] = {
            "single_patch_96": solve_single(),
            "batched": solve_batched(args.batch_patches),
            "batched_degree3": solve_batched(128, degrees=(3,)),
            "serving": serve_sample(args.serve_requests),
            "note": "wall time of whole solves to 1e-10 relative residual; the "
                    "FP64 reference solution is the plain FP64 GPU path; single-patch "
                    "solves stop on the FP64 Arnoldi estimate (the reference GMRES's "
                    "rule) and their true residuals are recomputed after timing; the "
                    "batched arms confirm each cycle with the true residual",
        }
    if rank == 0:
        print(json.dumps(line))
    finish(dist)
    return 0


if __name__ == "__main__":
    sys.exit(main())
