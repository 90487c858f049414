"""Device vector operations of the Krylov solvers (thin wrappers over the
libigab200 gram / combine / scale kernels; no torch arithmetic)."""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np
import torch

from . import _lib
from ._device import iga_dtype, stream_handle


def _dt(t: torch.Tensor):
    if t.dtype == torch.complex128:
        return _lib.IGA_F64, 1
    return iga_dtype(t.dtype), 0


class Workspace:
    """Scratch of the two-stage reductions (grown on demand)."""

    def __init__(self, device):
        self.device = device
        self.partial = torch.empty(0, dtype=torch.float64, device=device)
        self.out = torch.empty(0, dtype=torch.float64, device=device)

    def ensure(self, n: int, m1: int, m2: int, cplx: int):
        nblk = ctypes.c_int(0)
        elems = ctypes.c_int64(0)
        _lib.check(_lib.LIB.iga_gram_workspace(n, m1, m2, cplx, ctypes.byref(nblk),
                                               ctypes.byref(elems)))
        if self.partial.numel() < elems.value:
            self.partial = torch.empty(int(elems.value * 1.5) + 64, dtype=torch.float64,
                                       device=self.device)
        need = m1 * m2 * (2 if cplx else 1)
        if self.out.numel() < need:
            self.out = torch.empty(max(need, 64), dtype=torch.float64, device=self.device)
        return nblk.value


def gram(ws: Workspace, A: torch.Tensor, B: torch.Tensor) -> torch.Tensor:
    """G[j1, j2] = sum_i conj(A[j1, i]) B[j2, i] on the device (FP64 / complex128).
    A: (m1, n) rows, B: (m2, n) rows (row stride = stride(0))."""
    if A.ndim == 1:
        A = A.unsqueeze(0)
    if B.ndim == 1:
        B = B.unsqueeze(0)
    dt, cplx = _dt(A)
    m1, n = A.shape
    m2 = B.shape[0]
    nblk = ws.ensure(n, m1, m2, cplx)
    _lib.check(_lib.LIB.iga_gram(dt, cplx, n, m1, A.data_ptr(), A.stride(0), m2, B.data_ptr(),
                                 B.stride(0), ws.out.data_ptr(), ws.partial.data_ptr(), nblk,
                                 stream_handle()))
    cnt = m1 * m2 * (2 if cplx else 1)
    out = ws.out[:cnt].clone()
    if cplx:
        return torch.view_as_complex(out.reshape(m1, m2, 2))
    return out.reshape(m1, m2)


def gram_host(ws: Workspace, A, B) -> np.ndarray:
    return gram(ws, A, B).cpu().numpy()


def dot(ws: Workspace, a: torch.Tensor, b: torch.Tensor):
    g = gram_host(ws, a, b)[0, 0]
    return g


def norm(ws: Workspace, a: torch.Tensor) -> float:
    g = gram_host(ws, a, a)[0, 0]
    return float(np.sqrt(max(float(np.real(g)), 0.0)))


def combine(A: torch.Tensor, coef, out: torch.Tensor, alpha: float = 1.0, beta: float = 0.0):
    """out[k] = beta*out[k] + alpha * sum_j coef[j, k] A[j]; A (m, n) rows,
    coef (m, kout) host or device array, out (kout, n) rows (or (n,) if kout=1)."""
    if A.ndim == 1:
        A = A.unsqueeze(0)
    o = out.unsqueeze(0) if out.ndim == 1 else out
    dt, cplx = _dt(A)
    m, n = A.shape
    if m == 0:
        if beta != 1.0:
            _scale(o, beta)
        return out
    c = coef
    if not isinstance(c, torch.Tensor):
        c = np.asarray(c)
        c = c.reshape(m, -1)
        c = torch.from_numpy(np.ascontiguousarray(c.astype(np.complex128 if cplx else np.float64)))
    c = c.to(A.device).contiguous()
    if cplx:
        c = torch.view_as_real(c.to(torch.complex128)).contiguous()
    kout = o.shape[0]
    _lib.check(_lib.LIB.iga_combine(dt, cplx, n, m, A.data_ptr(), A.stride(0), kout, c.data_ptr(),
                                    float(alpha), float(beta), o.data_ptr(), o.stride(0),
                                    stream_handle()))
    return out


def _scale(x: torch.Tensor, s: float):
    dt, cplx = _dt(x)
    if cplx:
        xr = torch.view_as_real(x).reshape(-1)
        _lib.check(_lib.LIB.iga_axpby(_lib.IGA_F64, xr.numel(), float(s), xr.data_ptr(), 0.0,
                                      xr.data_ptr(), stream_handle()))
    else:
        _lib.check(_lib.LIB.iga_axpby(dt, x.numel(), float(s), x.data_ptr(), 0.0, x.data_ptr(),
                                      stream_handle()))


def axpby(alpha: float, x: torch.Tensor, beta: float, y: torch.Tensor):
    """y = alpha x + beta y (real or complex with real scalars)."""
    dt, cplx = _dt(y)
    if cplx:
        xr = torch.view_as_real(x).reshape(-1)
        yr = torch.view_as_real(y).reshape(-1)
        _lib.check(_lib.LIB.iga_axpby(_lib.IGA_F64, yr.numel(), float(alpha), xr.data_ptr(),
                                      float(beta), yr.data_ptr(), stream_handle()))
    else:
        _lib.check(_lib.LIB.iga_axpby(dt, y.numel(), float(alpha), x.data_ptr(), float(beta),
                                      y.data_ptr(), stream_handle()))
    return y


def copy(src: torch.Tensor, dst: torch.Tensor):
    return axpby(1.0, src, 0.0, dst)


def scale(x: torch.Tensor, s: float):
    _scale(x, s)
    return x


def mask(x: torch.Tensor, idx: Optional[torch.Tensor]):
    if idx is None or idx.numel() == 0:
        return x
    _lib.check(_lib.LIB.iga_mask_zero(iga_dtype(x.dtype), idx.numel(), idx.data_ptr(), x.data_ptr(),
                                      stream_handle()))
    return x


def split_complex(z: torch.Tensor):
    n = z.numel()
    re = torch.empty(n, dtype=torch.float64, device=z.device)
    im = torch.empty(n, dtype=torch.float64, device=z.device)
    _lib.check(_lib.LIB.iga_complex_split(n, z.data_ptr(), re.data_ptr(), im.data_ptr(),
                                          stream_handle()))
    return re, im


def merge_complex(re: torch.Tensor, im: torch.Tensor, out: Optional[torch.Tensor] = None):
    n = re.numel()
    if out is None:
        out = torch.empty(n, dtype=torch.complex128, device=re.device)
    _lib.check(_lib.LIB.iga_complex_merge(n, re.data_ptr(), im.data_ptr(), out.data_ptr(),
                                          stream_handle()))
    return out
