"""Launch-shape autotuner of the fused matrix-free kernels.

The fused 3D kernel's work unit is a (face tile, segment of the streamed
direction) pair; the face is fixed at compile time, the number of segments
``nseg`` is a run-time choice that trades CTA count (filling 148 SMs x 3
resident CTAs) against per-CTA pipeline warm-up and halo work.  ``tune_nseg``
times the candidate segment counts on the operator's own packed data
(CUDA events, best of a few launches) and keeps the winner per problem shape
in a process-wide cache, optionally persisted as JSON (``IGAOPS_B200_TUNE``
names the file).  The packed coefficient layout does not depend on ``nseg``,
so tuning re-launches the same data with a different plan field.
"""
from __future__ import annotations

import json
import os
from pathlib import Path
from typing import Dict, Iterable, Optional, Tuple

import torch

_CACHE: Dict[str, int] = {}
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
            _CACHE.update({k: int(v) for k, v in json.loads(p.read_text()).items()})
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
