"""Constants, enums and the Kronecker helpers the hot path needs.

Mirrors src/igaops/common/utils.py:5-62 and the two helpers of
src/igaops/common/math.py used by the fast-diagonalisation setup
(combine_arrays :10-58, KronProduct.kron_nonzero_indices :62-90).
"""
from __future__ import annotations

from enum import Enum
from typing import Any, List, Optional, Sequence

import numpy as np


class Constants:
    """Same values as the reference (src/igaops/common/utils.py:5-21)."""

    INFTY = 1e14
    HUGE = 1e8
    BIG = 1e4
    SMALL = 1e-4
    TINY = 1e-8
    SAFEGUARD = 1e-14


class ParametricDirection(Enum):
    XI = 0
    ETA = 1
    NU = 2
    TAU = 3
    ALL = -1


class BoundarySide(Enum):
    MIN = 0
    MAX = 1
    BOTH = -1


def validate_entry(value: str, reference: List[str]) -> Any:
    """Raise unless `value` is a string among `reference` (utils.py:53-62)."""
    if not isinstance(value, str):
        raise TypeError(f"Value's type must be string, got {type(value)}")
    if value not in reference:
        raise ValueError(f"Invalid value. Got '{value}', but must be one of {reference}")
    return value


def _kron_all(vectors: Sequence[np.ndarray]) -> np.ndarray:
    """v_n (x) ... (x) v_1 for vectors given as [v_1, ..., v_n]."""
    out = np.asarray(vectors[0])
    for v in vectors[1:]:
        out = np.kron(v, out)
    return out


def combine_arrays(arr: Sequence[np.ndarray], coefs: np.ndarray,
                   brr: Optional[Sequence[np.ndarray]] = None) -> np.ndarray:
    """sum_i c_i (b_n x .. x a_i x .. x b_1)  (kron sum; math.py:10-58).

    With brr = None the b_k are all-ones vectors, so this is the
    Kronecker sum of the scaled 1D eigenvalue arrays.
    """
    ndim = len(arr)
    if ndim == 0:
        return np.array([])
    if brr is None:
        # all-ones b_k: the Kronecker products only place the scaled a_i
        # (every other factor is exactly 1), so broadcasting gives the same
        # values term by term, summed in the same order, without the
        # Kronecker temporaries
        shape = [np.asarray(a).shape[0] for a in arr][::-1]
        total = None
        for i in range(ndim):
            term = (np.asarray(arr[i]) * coefs[i]).reshape(
                [-1 if k == ndim - 1 - i else 1 for k in range(ndim)])
            total = np.broadcast_to(term, shape) if total is None else total + term
        return np.ascontiguousarray(total).reshape(-1)
    total = None
    for i in range(ndim):
        parts = [brr[k] for k in range(ndim)]
        parts[i] = arr[i] * coefs[i]
        term = _kron_all(parts)
        total = term if total is None else total + term
    return total


class KronProduct:
    @staticmethod
    def kron_nonzero_indices(indices_list: Sequence[List[int]], nnz_list: Sequence[int]) -> List[int]:
        """Flat indices of the nonzeros of A_n x ... x A_1 (math.py:62-90).

        indices_list / nnz_list are ordered slowest-first (A_n first), as in the
        reference.  Row-major flattening: the last entry varies fastest.
        """
        return KronProduct.kron_nonzero_array(indices_list, nnz_list).tolist()

    @staticmethod
    def kron_nonzero_array(indices_list: Sequence[List[int]], nnz_list: Sequence[int]) -> np.ndarray:
        """kron_nonzero_indices as an int64 array (no Python list)."""
        if len(indices_list) == 0:
            return np.zeros(1, dtype=np.int64)
        strides = []
        acc = 1
        for n in reversed(list(nnz_list)):
            strides.append(acc)
            acc *= int(n)
        strides = strides[::-1]
        flat = np.zeros(1, dtype=np.int64)
        for idx, s in zip(indices_list, strides):
            idx = np.asarray(idx, dtype=np.int64)
            flat = (flat[:, None] + idx[None, :] * s).reshape(-1)
        return flat
