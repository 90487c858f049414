"""Seeded test problems shared by the CPU and GPU tests."""
from __future__ import annotations

import numpy as np

from igaops_b200.geometry import GeometryOps
from igaops_b200.quadrature import StandardGauss, WeightedQuadrature


def rules(ndim, degree, nbel, kind="wq2", rule="endpoint"):
    """One 1D rule per direction (the same object repeated, as the reference
    tests do) or per-direction rules when nbel/degree are sequences."""
    degs = degree if isinstance(degree, (list, tuple)) else [degree] * ndim
    nels = nbel if isinstance(nbel, (list, tuple)) else [nbel] * ndim
    out = []
    cache = {}
    for p, ne in zip(degs, nels):
        key = (p, ne)
        if key not in cache:
            kv = GeometryOps.make_open_knotvector(p, ne)
            if kind == "wq2":
                cache[key] = WeightedQuadrature(p, kv, "2", rule)
            elif kind == "wq1":
                cache[key] = WeightedQuadrature(p, kv, "1", rule)
            else:
                cache[key] = StandardGauss(p, kv, "legendre")
        out.append(cache[key])
    return out


def coefficients(op, rules_, rng, spd=None, symmetric=True):
    ndim = len(rules_)
    spd = spd or ndim
    nq = int(np.prod([q.nbquadpts for q in rules_]))
    if op == "u_v":
        return 1.0 + 0.5 * rng.random(nq)
    if op == "gradu_gradv":
        c = rng.standard_normal((ndim, ndim, nq)) * 0.3
        for i in range(ndim):
            c[i, i] += 2.0
        if symmetric:
            c = 0.5 * (c + c.transpose(1, 0, 2))
        return c
    return rng.standard_normal((ndim, nq))


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
