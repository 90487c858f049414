"""Oracle: 1D rules restored from the reference's own factors.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).  A fixture written by
tests/golden/make_golden.py holds, per rule, the CSR arrays of the
reference's ``quadrule.basis`` and ``quadrule.weights`` lists
(src/igaops/quadrature/weighted_quad.py:238-363,
src/igaops/quadrature/gauss_quad.py:14-126).  ``FixtureRule`` exposes the
attributes the oracle's operators read, so the CPU legs of the benchmark and
the tests run the oracle on the reference's factors without building rules
with the product package.

``slab_rule`` restricts a rule to a range of its quadrature points: the
operators of oracle/mf.py are sums over quadrature points, so the product of
a patch is the sum of the products of its slabs along the slowest direction
(the last rule), each with the coefficients of its own points.  The
benchmark's reference arm splits one matvec this way over worker processes.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import scipy.sparse as sp

GOLDEN = Path(__file__).resolve().parent.parent / "tests" / "golden"


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


class SlabRule:
    """The quadrature points [q0, q1) of a rule: basis rows and weight
    columns of those points only."""

    def __init__(self, rule, q0: int, q1: int):
        self.degree = rule.degree
        self.basis = [sp.csr_array(B[q0:q1, :]) for B in rule.basis]
        self.weights = [sp.csr_array(W[:, q0:q1]) for W in rule.weights]
        self.nbctrlpts = rule.nbctrlpts
        self.nbquadpts = q1 - q0


def slab_rule(rule, q0: int, q1: int) -> SlabRule:
    return SlabRule(rule, q0, q1)


def bench_rule() -> FixtureRule:
    """Weighted quadrature type "2" (endpoint points), degree 3, 128
    elements, as the reference builds it (fixture ``bench_rule.npz``)."""
    d = dict(np.load(GOLDEN / "bench_rule.npz", allow_pickle=False))
    return FixtureRule(d, "wq2_p3_ne128")
