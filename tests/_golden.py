"""Loaders for the golden fixtures produced by tests/golden/make_golden.py."""
from __future__ import annotations

from functools import lru_cache
from pathlib import Path

import numpy as np

from oracle.rules import FixtureRule, csr  # noqa: F401  (re-exported)

GOLDEN = Path(__file__).resolve().parent / "golden"


@lru_cache(maxsize=None)
def load(name: str):
    return dict(np.load(GOLDEN / f"{name}.npz", allow_pickle=False))


def rules(d: dict, name: str, ndim: int):
    return [FixtureRule(d, f"{name}_r{k}") for k in range(ndim)]
