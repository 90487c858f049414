"""Launch-shape autotuner of the fused matrix-free kernels.

Two choices, both timed on the operator's own packed data (CUDA events,
best of a few launches) and kept per problem shape in a process-wide cache,
optionally persisted as JSON (``IGAOPS_B200_TUNE`` names the file):

* the tiling of the 3D work: the pencil kernel's (16 x 8 face tile,
  segment of the streamed direction) units or the tensor-core kernel's
  16 x 8 x 16 point tiles, one persistent CTA per SM (``choose_kernel``;
  the two pack the coefficients differently, so the candidate is packed
  once for the timing and kept if it wins);
* for the pencil kernel, the number of segments ``nseg``, which trades CTA
  count (filling 148 SMs x 3 resident CTAs) against per-CTA pipeline
  warm-up and halo work (``tune_nseg``; the packed layout does not depend on
  ``nseg``, so tuning re-launches the same data with a different plan field).
"""
from __future__ import annotations

import json
import os
from pathlib import Path
from typing import Dict, Iterable, Optional, Tuple

import torch

_CACHE: Dict[str, object] = {}
_TIMES: Dict[str, Dict[str, float]] = {}
_LOADED = False


def _path() -> Optional[Path]:
    p = os.environ.get("IGAOPS_B200_TUNE")
    return Path(p) if p else None


def _load():
    global _LOADED
    if _LOADED:
        return
    _LOADED = True
    p = _path()
    if p and p.exists():
        try:
            _CACHE.update({k: (v if isinstance(v, str) else int(v))
                           for k, v in json.loads(p.read_text()).items()})
        except (ValueError, OSError):
            pass


def _save():
    p = _path()
    if p:
        try:
            p.write_text(json.dumps(_CACHE, indent=0, sort_keys=True))
        except OSError:
            pass


def shape_key(plan) -> str:
    """Problem shape of a fused plan (what the best launch shape depends on)."""
    return "|".join(str(v) for v in (
        plan.ndim, plan.op, plan.st, plan.tt, plan.tr, int(plan.sym), str(plan.dtype)[6:],
        plan.W, *plan.n, *plan.nq, torch.cuda.get_device_name()))


def candidates(plan) -> Iterable[int]:
    nlast = plan.nq[-1]
    tiles = plan.units // max(plan.nseg, 1)
    out = {1, 2, 3, 4, 6, 8, 12, 16}
    # enough CTAs for about 3 resident CTAs x 148 SMs x k waves
    for k in (1, 2, 4):
        out.add(-(-444 * k // max(tiles, 1)))
    return sorted(n for n in out if 1 <= n <= max(1, nlast // 8))


def tune_nseg(plan, packed: torch.Tensor, x: torch.Tensor, y: torch.Tensor,
              reps: int = 3) -> Tuple[int, Dict[int, float]]:
    """Pick the fastest segment count for `plan` (a FusedPlan) on its packed
    coefficients; returns (best nseg, {nseg: ms}).  The plan is left set to
    the winner.  Cached per shape_key."""
    _load()
    key = shape_key(plan)
    if key in _CACHE:
        plan.set_nseg(_CACHE[key])
        return _CACHE[key], {}
    times: Dict[int, float] = {}
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    for ns in candidates(plan):
        plan.set_nseg(ns)
        plan.matvec(packed, x, y)  # warm-up (configures the kernel)
        best = float("inf")
        for _ in range(reps):
            e0.record()
            plan.matvec(packed, x, y)
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        times[ns] = best
    plan.check_status()
    win = min(times, key=times.get)
    plan.set_nseg(win)
    _CACHE[key] = win
    _save()
    return win, times


def _best_ms(fn, reps: int) -> float:
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    fn()  # warm-up (configures the kernel)
    best = float("inf")
    for _ in range(reps):
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def choose_kernel(plan, packed: torch.Tensor, make_tile, x: torch.Tensor, y: torch.Tensor,
                  reps: int = 3):
    """Pencil kernel (``plan`` / ``packed``, already at its tuned segment
    count) or tile kernel (``make_tile()`` -> (TilePlan, packed)) for this
    shape, whichever is faster.  Returns ("pencil", None) or ("tile",
    (plan, packed)); cached per shape_key of the pencil plan."""
    _load()
    key = "kernel|" + shape_key(plan)
    if key in _CACHE:
        return (_CACHE[key], make_tile() if _CACHE[key] == "tile" else None)
    t_pencil = _best_ms(lambda: plan.matvec(packed, x, y), reps)
    plan.check_status()
    tplan, tpacked = make_tile()
    t_tile = _best_ms(lambda: tplan.matvec(tpacked, x, y), reps)
    tplan.check_status()
    win = "tile" if t_tile < t_pencil else "pencil"
    _CACHE[key] = win
    _TIMES[key] = {"pencil_ms": t_pencil, "tile_ms": t_tile, "pencil_nseg": plan.nseg}
    _save()
    return win, ((tplan, tpacked) if win == "tile" else None)


def decisions() -> Dict[str, Dict[str, object]]:
    """Kernel choices made in this process: shape key -> the winner and the
    timings it was chosen on."""
    return {k[len("kernel|"):]: dict(_TIMES.get(k, {}), kernel=v)
            for k, v in _CACHE.items() if k.startswith("kernel|")}
