"""iga_gram_noalloc: the Gram / dot-product entry point for callers that
cannot allocate device memory (a host program that links only the C ABI and
owns no device allocator, or code that must not call cudaMalloc mid-pipeline).

It must return what iga_gram returns with caller-provided scratch, on
consecutive calls (its built-in scratch keeps the previous call's contents),
and refuse requests larger than its built-in scratch.  Calls go through the
C ABI (ctypes), with device buffers from torch.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-12  # FP64 tolerance used by the other GPU tests


def _lib():
    from igaops_b200 import _lib

    lib = ctypes.CDLL(_lib.library_path())
    vp, i32, i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64
    lib.iga_gram_noalloc.argtypes = [i32, i32, i64, i32, vp, i64, i32, vp, i64, vp, vp]
    lib.iga_gram_noalloc.restype = i32
    lib.iga_gram.argtypes = [i32, i32, i64, i32, vp, i64, i32, vp, i64, vp, vp, i32, vp]
    lib.iga_gram.restype = i32
    lib.iga_gram_workspace.argtypes = [i64, i32, i32, i32, ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int64)]
    lib.iga_gram_workspace.restype = i32
    lib.iga_last_error.restype = ctypes.c_char_p
    return lib


def _with_scratch(lib, A, B, cplx):
    n = A.shape[1]
    m1, m2 = A.shape[0], B.shape[0]
    nblk, elems = ctypes.c_int(0), ctypes.c_int64(0)
    assert lib.iga_gram_workspace(n, m1, m2, cplx, ctypes.byref(nblk), ctypes.byref(elems)) == 0
    part = torch.empty(int(elems.value), dtype=torch.float64, device="cuda")
    out = torch.empty(m1 * m2 * (2 if cplx else 1), dtype=torch.float64, device="cuda")
    rc = lib.iga_gram(0, cplx, n, m1, A.data_ptr(), A.stride(0), m2, B.data_ptr(), B.stride(0),
                      out.data_ptr(), part.data_ptr(), nblk.value, None)
    assert rc == 0, lib.iga_last_error()
    return out


def _noalloc(lib, A, B, cplx):
    n = A.shape[1]
    m1, m2 = A.shape[0], B.shape[0]
    out = torch.full((m1 * m2 * (2 if cplx else 1),), float("nan"), dtype=torch.float64,
                     device="cuda")
    rc = lib.iga_gram_noalloc(0, cplx, n, m1, A.data_ptr(), A.stride(0), m2, B.data_ptr(),
                              B.stride(0), out.data_ptr(), None)
    assert rc == 0, lib.iga_last_error()
    return out


def _rel(a, b):
    a, b = a.cpu().numpy(), b.cpu().numpy()
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


# (64, 64, 1e6): the default 296 reduction blocks of 4096 partials would not
# fit the built-in array, so the call runs with 16 blocks
@pytest.mark.parametrize("m1,m2,n", [(1, 1, 1_000_003), (37, 1, 250_000), (12, 9, 4096),
                                     (64, 64, 1_000_000)])
def test_noalloc_matches_caller_scratch_twice(m1, m2, n):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = _lib()
    g = torch.Generator(device="cuda").manual_seed(m1 * 1000 + m2)
    for call in range(2):  # two calls in a row share the built-in scratch
        A = torch.randn((m1, n), dtype=torch.float64, device="cuda", generator=g)
        B = torch.randn((m2, n), dtype=torch.float64, device="cuda", generator=g)
        ref = _with_scratch(lib, A, B, 0)
        got = _noalloc(lib, A, B, 0)
        torch.cuda.synchronize()
        assert _rel(got, ref) < TOL, f"call {call}"


# (32, 32, 5e5) complex: 2048 partials per block, 245 blocks cut to 32;
# (4096, 1, 3000) complex: a row set wider than the default shared-memory
# window of the first stage at one row per tile (64 KiB)
@pytest.mark.parametrize("m1,m2,n", [(6, 3, 70_001), (32, 32, 500_000), (4096, 1, 3000)])
def test_noalloc_complex_twice(m1, m2, n):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = _lib()
    g = torch.Generator(device="cuda").manual_seed(5)
    for call in range(2):
        A = torch.randn((m1, n), dtype=torch.complex128, device="cuda", generator=g)
        B = torch.randn((m2, n), dtype=torch.complex128, device="cuda", generator=g)
        ref = _with_scratch(lib, A, B, 1)
        got = _noalloc(lib, A, B, 1)
        torch.cuda.synchronize()
        assert _rel(got, ref) < TOL, f"call {call}"
        # and against the definition
        want = (A.conj() @ B.T).reshape(-1)
        assert _rel(torch.view_as_complex(got.reshape(-1, 2)), want) < 1e-12


def test_noalloc_rejects_oversize_request():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = _lib()
    A = torch.zeros((4097, 8), dtype=torch.float64, device="cuda")
    B = torch.zeros((17, 8), dtype=torch.float64, device="cuda")
    out = torch.zeros(4097 * 17, dtype=torch.float64, device="cuda")
    rc = lib.iga_gram_noalloc(0, 0, 8, 4097, A.data_ptr(), 8, 17, B.data_ptr(), 8,
                              out.data_ptr(), None)
    assert rc == 1  # IGA_ERR_INVALID_ARG
    assert b"iga_gram_noalloc" in lib.iga_last_error()
    assert b"4096 pairs" in lib.iga_last_error()
