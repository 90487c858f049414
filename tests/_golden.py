"""Loaders for the golden fixtures produced by tests/golden/make_golden.py."""
from __future__ import annotations

from functools import lru_cache
from pathlib import Path

import numpy as np
import scipy.sparse as sp

GOLDEN = Path(__file__).resolve().parent / "golden"


@lru_cache(maxsize=None)
def load(name: str):
    return dict(np.load(GOLDEN / f"{name}.npz", allow_pickle=False))


def csr(d: dict, prefix: str) -> sp.csr_array:
    shape = tuple(int(v) for v in d[prefix + "_shape"])
    return sp.csr_array((d[prefix + "_data"], d[prefix + "_indices"], d[prefix + "_indptr"]),
                        shape=shape)


class FixtureRule:
    """A 1D rule restored from a fixture (the reference's own factors)."""

    def __init__(self, d: dict, prefix: str):
        self.degree = int(d[prefix + "_degree"])
        self.knotvector = d[prefix + "_knotvector"]
        self.quadpts = d[prefix + "_quadpts"]
        self.basis = []
        k = 0
        while f"{prefix}_B{k}_shape" in d:
            self.basis.append(csr(d, f"{prefix}_B{k}"))
            k += 1
        self.weights = [csr(d, f"{prefix}_W{k}") for k in range(4)]
        self.nbctrlpts = self.basis[0].shape[1]
        self.nbquadpts = self.basis[0].shape[0]
        self.unique_kv = np.unique(np.clip(self.knotvector, 0, 1))


def rules(d: dict, name: str, ndim: int):
    return [FixtureRule(d, f"{name}_r{k}") for k in range(ndim)]
