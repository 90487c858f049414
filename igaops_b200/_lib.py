"""ctypes binding of ``libigab200.so`` (the C ABI declared in include/igab200.h).

The library is loaded from ``igaops_b200/_lib/`` only.  If it is missing the
import fails loudly: there is no CPU or JIT fallback for any operator.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_LIBPATH = Path(__file__).resolve().parent / "_lib" / "libigab200.so"

IGA_OK = 0
IGA_ERR_INVALID_ARG = 1
IGA_ERR_UNSUPPORTED = 2
IGA_ERR_CUDA = 3
IGA_ERR_NOT_CONVERGED = 4
IGA_ERR_BREAKDOWN = 5
IGA_ERR_NONFINITE = 6
IGA_ERR_GEOMETRY = 7
IGA_ERR_TIMEOUT = 8

IGA_F64, IGA_F32, IGA_BF16 = 0, 1, 2
IGA_OP_MASS, IGA_OP_STIFF, IGA_OP_GRADU_V, IGA_OP_U_GRADV = 0, 1, 2, 3


class IgaError(RuntimeError):
    """A libigab200 call returned an error status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[iga status {status}] {message}")
        self.status = status


class UnsupportedError(IgaError, NotImplementedError):
    pass


class DeviceTimeoutError(IgaError, TimeoutError):
    pass


class NonFiniteError(IgaError, FloatingPointError):
    """A non-finite value (NaN / Inf) in an input or in a solver's iterates."""


class iga_band(C.Structure):
    _fields_ = [
        ("rows", C.c_int32),
        ("cols", C.c_int32),
        ("width", C.c_int32),
        ("reserved", C.c_int32),
        ("start", C.c_void_p),
        ("vals", C.c_void_p),
    ]


class iga_factor(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("rows", C.c_int32),
        ("cols", C.c_int32),
        ("reserved", C.c_int32),
        ("ld_row", C.c_int64),
        ("ld_col", C.c_int64),
        ("band", iga_band),
        ("dense", C.c_void_p),
    ]


class iga_mf_plan(C.Structure):
    _fields_ = [
        ("ndim", C.c_int32),
        ("op", C.c_int32),
        ("spacetime", C.c_int32),
        ("time_test", C.c_int32),
        ("time_trial", C.c_int32),
        ("sym", C.c_int32),
        ("width", C.c_int32),
        ("rwidth", C.c_int32),
        ("n", C.c_int32 * 3),
        ("nq", C.c_int32 * 3),
        ("face", C.c_int32 * 2),
        ("nseg", C.c_int32),
        ("nstream", C.c_int32),
        ("src_row", C.c_int32 * 9),
        ("cmax", C.c_int32 * 2),
        ("dmax", C.c_int32 * 2),
        ("tile_off", C.c_void_p),
        ("trial", iga_band * 3),
        ("trial_d1", C.c_void_p * 3),
        ("testT", iga_band * 3),
        ("testT_d1", C.c_void_p * 3),
        ("testR", iga_band * 3),
        ("testR_d1", C.c_void_p * 3),
        ("status", C.c_void_p),
        ("step_table", C.c_void_p),
        ("wait_test", C.c_int32),
    ]


class iga_mft_plan(C.Structure):
    _fields_ = [
        ("op", C.c_int32),
        ("nstream", C.c_int32),
        ("n", C.c_int32 * 3),
        ("nq", C.c_int32 * 3),
        ("ntile", C.c_int32 * 3),
        ("wsum", C.c_int32 * 3),
        ("src_row", C.c_int32 * 6),
        ("geom", C.c_void_p),
        ("frag", C.c_void_p),
        ("status", C.c_void_p),
    ]


# y = op(x) callback of the solve entry points (include/igab200.h iga_apply_fn)
APPLY_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p)


def _load():
    if not _LIBPATH.exists():
        raise ImportError(
            f"{_LIBPATH} is missing: build the CUDA library first "
            "(python -m igaops_b200.build). igaops_b200 has no CPU fallback."
        )
    lib = C.CDLL(str(_LIBPATH))
    vp, i32, i64 = C.c_void_p, C.c_int, C.c_int64
    sig = {
        "iga_abi_version": ([], C.c_int),
        "iga_last_error": ([], C.c_char_p),
        "iga_mode_product": ([i32, C.POINTER(iga_factor), i64, i64, vp, vp, i32, vp], i32),
        "iga_lmode_apply": ([i32, i32, C.POINTER(iga_factor), i64, vp, vp, vp, vp, vp], i32),
        "iga_pointwise_scale": ([i32, i64, i64, vp, i64, vp, vp, i32, vp], i32),
        "iga_axpby": ([i32, i64, C.c_double, vp, C.c_double, vp, vp], i32),
        "iga_mf_layout": ([C.POINTER(iga_mf_plan), i32, C.POINTER(C.c_int64), vp], i32),
        "iga_mf_pack": ([C.POINTER(iga_mf_plan), i32, vp, i64, i32, vp, vp], i32),
        "iga_mf_table": ([C.POINTER(iga_mf_plan), i32, C.POINTER(C.c_int64), vp, vp], i32),
        "iga_mf_matvec": ([C.POINTER(iga_mf_plan), i32, vp, i64, vp, vp, vp], i32),
        "iga_mft_pack": ([C.POINTER(iga_mft_plan), i32, vp, i64, vp, i64, vp], i32),
        "iga_mft_smem_bytes": ([C.POINTER(iga_mft_plan), C.POINTER(C.c_int64)], i32),
        "iga_mft_matvec": ([C.POINTER(iga_mft_plan), vp, i64, vp, vp, vp], i32),
        "iga_geometry_pointwise": ([i32, i32, i64, vp, vp, vp, vp, vp, vp], i32),
        "iga_nurbs_coefficients": ([i32, i32, i64, vp, vp, vp, vp, vp, vp, vp, vp, vp], i32),
        "iga_wq_min_norm_rows": ([i32, i32, i32, vp, vp, vp, C.c_double, vp], i32),
        "iga_wq_point_counts": ([i32, i32, vp, i32, vp, vp, vp], i32),
        "iga_bspline_basis": ([i32, i32, vp, C.c_int64, vp, i32, vp, vp], i32),
        "iga_mf_batch_table_bytes": ([i32, i32, C.POINTER(C.c_int64)], i32),
        "iga_mf_batch_prepare": ([C.POINTER(iga_mf_plan), i32, i32, vp, vp, vp,
                                  C.POINTER(C.c_int32), C.POINTER(C.c_int64)], i32),
        "iga_mf_batch_matvec": ([C.POINTER(iga_mf_plan), i32, i32, vp, C.c_int32, i64, vp, vp,
                                 i64, i32, vp, vp], i32),
        "iga_fd_tc_batch_table_bytes": ([i32, C.POINTER(C.c_int64)], i32),
        "iga_fd_tc_batch_prepare": ([i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, i32, vp, vp, vp,
                                     C.POINTER(C.c_int64)], i32),
        "iga_fd_tc_batch_apply": ([i32, i32, vp, vp, i64, vp, vp, i64, vp, vp], i32),
        "iga_seg_chunk": ([], C.c_int),
        "iga_seg_gram": ([i32, i32, vp, vp, i32, i32, vp, i64, vp, vp, vp, i64, vp], i32),
        "iga_seg_combine": ([i32, i32, vp, vp, i32, i32, vp, i64, vp, i64, C.c_double,
                             C.c_double, vp, vp], i32),
        "iga_seg_scale": ([i32, i32, vp, vp, i32, vp, vp, i64, i32, vp], i32),
        "iga_seg_givens_init": ([i32, i32, vp, vp, vp, vp, vp], i32),
        "iga_seg_givens_step": ([i32, i32, i32, vp, vp, i64, vp, vp, vp, vp, C.c_double, vp, vp,
                                 vp], i32),
        "iga_seg_trisolve": ([i32, i32, i32, vp, vp, vp, vp, vp], i32),
        "iga_fd_apply": ([i32, i32, vp, vp, vp, vp, vp, i64, vp, vp, vp, vp, vp], i32),
        "iga_fd_tc_workspace": ([vp, C.POINTER(C.c_int64)], i32),
        "iga_box_copy": ([i32, i32, vp, vp, vp, i64, vp, vp, i32, vp], i32),
        "iga_arrowhead_solve": ([i32, i32, i64, vp, vp, vp, vp, vp, vp], i32),
        "iga_fd_sptime_apply": ([i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, i32, vp, vp, vp, vp,
                                 vp, vp], i32),
        "iga_fd_sptime_qz_apply": ([i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, C.c_double,
                                    vp, i32, vp, vp, vp, vp, vp, vp], i32),
        "iga_fd_apply_tc": ([i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp], i32),
        "iga_gmres_workspace": ([i64, i32, C.POINTER(C.c_int64)], i32),
        "iga_gmres_solve": ([i64, vp, vp, C.c_double, i32, APPLY_FN, APPLY_FN, vp, vp, i64, vp,
                             i64, vp, C.POINTER(C.c_int), vp], i32),
        "iga_gram_workspace": ([i64, i32, i32, i32, C.POINTER(C.c_int), C.POINTER(C.c_int64)], i32),
        "iga_gram": ([i32, i32, i64, i32, vp, i64, i32, vp, i64, vp, vp, i32, vp], i32),
        "iga_gram_noalloc": ([i32, i32, i64, i32, vp, i64, i32, vp, i64, vp, vp], i32),
        "iga_combine": ([i32, i32, i64, i32, vp, i64, i32, vp, C.c_double, C.c_double, vp, i64,
                         vp], i32),
        "iga_scale_dev": ([i32, i32, i64, vp, vp, i32, vp], i32),
        "iga_mask_zero": ([i32, i64, vp, vp, vp], i32),
        "iga_convert": ([i32, i32, i64, vp, vp, vp], i32),
        "iga_complex_split": ([i64, vp, vp, vp, vp], i32),
        "iga_complex_merge": ([i64, vp, vp, vp, vp], i32),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


class _LazyLib:
    """Loads libigab200.so on first use (so that the build step can run
    before the library exists); a missing library raises ImportError."""

    _lib = None

    def __getattr__(self, name):
        if _LazyLib._lib is None:
            _LazyLib._lib = _load()
        return getattr(_LazyLib._lib, name)


LIB = _LazyLib()


def load() -> None:
    """Load the library now (raises ImportError when it is missing)."""
    LIB.iga_abi_version()


def check(status: int) -> None:
    """Raise the Python exception matching a non-OK status."""
    if status == IGA_OK:
        return
    msg = (LIB.iga_last_error() or b"").decode(errors="replace")
    if status == IGA_ERR_INVALID_ARG:
        raise ValueError(msg)
    if status == IGA_ERR_UNSUPPORTED:
        raise UnsupportedError(status, msg)
    if status == IGA_ERR_TIMEOUT:
        raise DeviceTimeoutError(status, msg or "a bounded device wait ran out")
    if status == IGA_ERR_NONFINITE:
        raise NonFiniteError(status, msg or "non-finite value")
    if status == IGA_ERR_GEOMETRY:
        raise ValueError(msg)
    raise IgaError(status, msg)


def library_path() -> str:
    return str(_LIBPATH)


def exported_symbols():
    """Names of the C entry points this binding declares."""
    return [
        "iga_abi_version",
        "iga_last_error",
        "iga_mode_product",
        "iga_lmode_apply",
        "iga_pointwise_scale",
        "iga_axpby",
        "iga_mf_layout",
        "iga_mf_pack",
        "iga_mf_table",
        "iga_mf_matvec",
        "iga_mft_pack",
        "iga_mft_smem_bytes",
        "iga_mft_matvec",
        "iga_geometry_pointwise",
        "iga_nurbs_coefficients",
        "iga_wq_min_norm_rows",
        "iga_wq_point_counts",
        "iga_bspline_basis",
        "iga_mf_batch_table_bytes",
        "iga_mf_batch_prepare",
        "iga_mf_batch_matvec",
        "iga_fd_tc_batch_table_bytes",
        "iga_fd_tc_batch_prepare",
        "iga_fd_tc_batch_apply",
        "iga_seg_chunk",
        "iga_seg_gram",
        "iga_seg_combine",
        "iga_seg_scale",
        "iga_seg_givens_init",
        "iga_seg_givens_step",
        "iga_seg_trisolve",
        "iga_fd_apply",
        "iga_fd_tc_workspace",
        "iga_box_copy",
        "iga_arrowhead_solve",
        "iga_fd_sptime_apply",
        "iga_fd_sptime_qz_apply",
        "iga_fd_apply_tc",
        "iga_gmres_workspace",
        "iga_gmres_solve",
        "iga_gram_workspace",
        "iga_gram",
        "iga_gram_noalloc",
        "iga_combine",
        "iga_scale_dev",
        "iga_mask_zero",
        "iga_convert",
        "iga_complex_split",
        "iga_complex_merge",
    ]
