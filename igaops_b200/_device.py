"""Device plumbing: CUDA availability, streams, dtype mapping, host<->device.

PyTorch provides device memory and streams only; every numerical step of the
operators runs in libigab200 kernels.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib

_DTYPES = {torch.float64: _lib.IGA_F64, torch.float32: _lib.IGA_F32}


def require_cuda() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError(
            "igaops_b200 runs on a CUDA device (B200, sm_100a) only; no GPU is visible "
            "and there is no CPU fallback"
        )
    return torch.device("cuda", torch.cuda.current_device())


def stream_handle() -> int:
    return torch.cuda.current_stream().cuda_stream


def iga_dtype(t: torch.dtype) -> int:
    try:
        return _DTYPES[t]
    except KeyError:
        raise TypeError(f"unsupported element type {t}; use float64 or float32") from None


def is_torch(a) -> bool:
    return isinstance(a, torch.Tensor)


def to_device(a, dtype: torch.dtype, device=None) -> torch.Tensor:
    """Contiguous device tensor of `dtype` holding `a` (numpy, scalar or torch)."""
    device = device or require_cuda()
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=dtype).contiguous()
    arr = np.ascontiguousarray(np.asarray(a))
    return torch.from_numpy(arr).to(device=device, dtype=dtype, non_blocking=False).contiguous()


def compute_dtype(a) -> torch.dtype:
    """Kernel element type for an input: torch float32 stays float32, else float64."""
    if isinstance(a, torch.Tensor) and a.dtype == torch.float32:
        return torch.float32
    return torch.float64


def like_input(result: torch.Tensor, template):
    """Return `result` in the container type of `template` (numpy in -> numpy out)."""
    if isinstance(template, torch.Tensor):
        return result
    return result.detach().cpu().numpy().astype(np.float64, copy=False)
