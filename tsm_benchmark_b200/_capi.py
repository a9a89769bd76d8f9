"""ctypes binding of the C ABI in include/tsm.h (libtsm_b200.so, built in-tree).

This module is the only place Python touches the library.  There is no CPU
fallback: if the shared library is missing or fails to load, every entry
point raises ``TsmLibraryError`` with the build command.
"""
from __future__ import annotations

import ctypes
import os
import threading

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libtsm_b200.so")

c_int64 = ctypes.c_int64
c_int = ctypes.c_int
c_size_t = ctypes.c_size_t
c_void_p = ctypes.c_void_p
c_uint64 = ctypes.c_uint64

DTYPE = {"f64": 0, "f32": 1}

STATUS = {
    0: "TSM_SUCCESS",
    1: "TSM_ERROR_INVALID_VALUE",
    2: "TSM_ERROR_WORKSPACE",
    3: "TSM_ERROR_CUDA",
    4: "TSM_ERROR_UNSUPPORTED",
    5: "TSM_ERROR_DEVICE_TIMEOUT",
}


class TsmLibraryError(RuntimeError):
    """The CUDA library is not built or cannot be loaded."""


class TsmError(RuntimeError):
    """A C ABI call returned a non-success tsm_status."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class VariantInfo(ctypes.Structure):
    _fields_ = [
        ("name", ctypes.c_char * 64),
        ("kind", c_int),
        ("dtype", c_int),
        ("wa", c_int), ("wb", c_int),
        ("ta", c_int), ("tb", c_int),
        ("exact", c_int),
        ("threads", c_int), ("stages", c_int), ("rows", c_int), ("unroll", c_int),
        ("smem_bytes", c_size_t),
        ("gram", c_int),
    ]


class BatchedProblem(ctypes.Structure):
    _fields_ = [("A", c_void_p), ("B", c_void_p), ("C", c_void_p), ("n", c_int64), ("m", c_int), ("k", c_int),
                ("ldc", c_int64), ("accumulate", c_int)]


class BatchedPlan(ctypes.Structure):
    _fields_ = [("device", c_void_p), ("bytes", c_size_t), ("count", c_int), ("segments", c_int),
                ("grid", c_int), ("flags", c_int)]


# Every function declared in include/tsm.h: name -> (restype, argtypes).
SIGNATURES = {
    "tsm_version": (c_int, []),
    "tsm_status_string": (ctypes.c_char_p, [c_int]),
    "tsm_last_cuda_error": (ctypes.c_char_p, []),
    "tsm_gemm_tn_workspace_size": (c_size_t, [c_int64, c_int, c_int]),
    "tsm_gemm_tn_f64": (c_int, [c_void_p, c_int64, c_int, c_int, c_void_p, c_int64, c_void_p, c_int64,
                                c_void_p, c_int64, c_int, c_void_p, c_size_t]),
    "tsm_gram_f64": (c_int, [c_void_p, c_int64, c_int, c_void_p, c_int64, c_void_p, c_int64, c_int, c_void_p,
                             c_size_t]),
    "tsm_gemm_tn_strided_f64": (c_int, [c_void_p, c_int64, c_int, c_int, c_void_p, c_int64, c_int64, c_void_p,
                                        c_int64, c_int64, c_void_p, c_int64, c_int, c_void_p, c_size_t]),
    "tsm_gemm_tn_f64_variant": (c_int, [c_void_p, c_int64, c_int, c_int, c_void_p, c_int64, c_void_p, c_int64,
                                        c_void_p, c_int64, c_int, c_void_p, c_size_t, c_int]),
    "tsm_gemm_tn_f64_launch": (c_int, [c_void_p, c_int64, c_int, c_int, c_void_p, c_int64, c_void_p, c_int64,
                                       c_void_p, c_int64, c_int, c_void_p, c_size_t, c_int, c_int64]),
    "tsm_gemm_tn_f32": (c_int, [c_void_p, c_int64, c_int, c_int, c_void_p, c_int64, c_void_p, c_int64,
                                c_void_p, c_int64, c_int, c_void_p, c_size_t]),
    "tsm_gemm_tn_f32_variant": (c_int, [c_void_p, c_int64, c_int, c_int, c_void_p, c_int64, c_void_p, c_int64,
                                        c_void_p, c_int64, c_int, c_void_p, c_size_t, c_int]),
    "tsm_gemm_tn_f32_split_bf16": (c_int, [c_void_p, c_int64, c_int, c_int, c_void_p, c_int64, c_void_p, c_int64,
                                           c_void_p, c_int64, c_int, c_int, c_void_p, c_size_t]),
    "tsm_gemm_tn_f32_split": (c_int, [c_void_p, c_int64, c_int, c_int, c_void_p, c_int64, c_void_p, c_int64,
                                      c_void_p, c_int64, c_int, c_void_p, c_size_t]),
    "tsm_gemm_tn_default_variant": (c_int, [c_int, c_int64, c_int, c_int, c_void_p, c_int64, c_void_p, c_int64]),
    "tsm_variant_count": (c_int, []),
    "tsm_variant_get_info": (c_int, [c_int, ctypes.POINTER(VariantInfo)]),
    "tsm_selftest_wait_timeout": (c_int, [c_void_p, c_void_p, c_size_t, ctypes.c_uint]),
    "tsm_workspace_check": (c_int, [c_void_p, c_void_p, ctypes.POINTER(ctypes.c_uint)]),
    "tsm_fill_uniform_f64": (c_int, [c_void_p, c_void_p, c_int64, c_uint64, c_uint64]),
    "tsm_tsmm_f64": (c_int, [c_void_p, c_int64, c_int, c_int, c_void_p, c_int64, c_void_p, c_int64, c_int64,
                             c_void_p, c_int64, c_int, c_void_p, c_size_t]),
    "tsm_tsmm_f32": (c_int, [c_void_p, c_int64, c_int, c_int, c_void_p, c_int64, c_void_p, c_int64, c_int64,
                             c_void_p, c_int64, c_int, c_void_p, c_size_t]),
    "tsm_gemm_tn_backward_f64": (c_int, [c_void_p, c_int64, c_int, c_int, c_void_p, c_int64, c_void_p, c_int64,
                                         c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int64, c_int,
                                         c_void_p, c_size_t]),
    "tsm_gemm_tn_backward_f32": (c_int, [c_void_p, c_int64, c_int, c_int, c_void_p, c_int64, c_void_p, c_int64,
                                         c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int64, c_int,
                                         c_void_p, c_size_t]),
    "tsm_block_orth_f64": (c_int, [c_void_p, c_int64, c_int, c_int, c_void_p, c_int64, c_void_p, c_int64,
                                   c_void_p, c_int64, c_void_p, c_size_t]),
    "tsm_batched_plan_size_f64": (c_size_t, [c_int, ctypes.POINTER(BatchedProblem)]),
    "tsm_batched_plan_init_f64": (c_int, [c_void_p, c_int, ctypes.POINTER(BatchedProblem), c_void_p, c_size_t,
                                          ctypes.POINTER(BatchedPlan)]),
    "tsm_batched_plan_init_paths_f64": (c_int, [c_void_p, c_int, ctypes.POINTER(BatchedProblem),
                                                ctypes.POINTER(c_int), c_void_p, c_size_t,
                                                ctypes.POINTER(BatchedPlan)]),
    "tsm_gemm_tn_batched_f64": (c_int, [c_void_p, ctypes.POINTER(BatchedPlan)]),
    "tsm_gemm_tn_f64_noalloc": (c_int, [c_void_p, c_int64, c_int, c_int, c_void_p, c_int64, c_void_p, c_int64,
                                        c_void_p, c_int64, c_int]),
    "tsm_noalloc_check": (c_int, [c_void_p, ctypes.POINTER(ctypes.c_uint)]),
}

_lib = None
_lock = threading.Lock()


def load() -> ctypes.CDLL:
    """Loads libtsm_b200.so once; raises TsmLibraryError if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise TsmLibraryError(
                f"{LIB_PATH} is missing: build it with `python -m tsm_benchmark_b200.build` "
                "(there is no CPU fallback)")
        try:
            lib = ctypes.CDLL(LIB_PATH)
        except OSError as e:  # pragma: no cover - depends on the host
            raise TsmLibraryError(f"cannot load {LIB_PATH}: {e}") from e
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(status: int, what: str = "") -> None:
    """Raises TsmError for a non-success status."""
    if status == 0:
        return
    lib = load()
    msg = lib.tsm_status_string(status).decode()
    if status == 3:
        msg += f" ({lib.tsm_last_cuda_error().decode()})"
    raise TsmError(status, f"{what}: {STATUS.get(status, status)}: {msg}" if what else msg)


_KINDS = {0: "bulk", 1: "direct", 2: "dmma"}


def variants() -> list[dict]:
    """All compiled variants, in table order."""
    lib = load()
    out = []
    for i in range(lib.tsm_variant_count()):
        info = VariantInfo()
        check(lib.tsm_variant_get_info(i, ctypes.byref(info)), "tsm_variant_get_info")
        out.append(dict(index=i, name=info.name.decode(), kind=_KINDS.get(info.kind, str(info.kind)),
                        dtype="f64" if info.dtype == 0 else "f32",
                        wa=info.wa, wb=info.wb, ta=info.ta, tb=info.tb, exact=bool(info.exact),
                        threads=info.threads, stages=info.stages, rows=info.rows, unroll=info.unroll,
                        smem_bytes=info.smem_bytes, gram=bool(info.gram)))
    return out
