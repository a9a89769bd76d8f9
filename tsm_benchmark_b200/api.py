"""Python entry points over the C ABI, taking torch CUDA tensors.

torch is used for device memory and streams only; every computation is a
call into libtsm_b200.so.  Shapes follow include/tsm.h: A (n x m), B (n x k)
row-major (unit column stride, any row stride), C (m x k).
"""
from __future__ import annotations

import ctypes
import threading

import torch

from . import _capi

_ws_lock = threading.Lock()
_workspaces: dict[tuple[int, int], torch.Tensor] = {}


def _stream_handle(device: torch.device, stream: torch.cuda.Stream | None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream(device)
    return int(s.cuda_stream)


def workspace(device: torch.device, nbytes: int, stream_handle: int) -> torch.Tensor:
    """A zero-initialised device workspace of at least `nbytes`, one per
    (device, stream): calls on one stream are ordered, so they may share it."""
    key = (device.index if device.index is not None else torch.cuda.current_device(), stream_handle)
    with _ws_lock:
        ws = _workspaces.get(key)
        if ws is None or ws.numel() < nbytes:
            ws = torch.zeros(max(nbytes, 1 << 20), dtype=torch.uint8, device=device)
            _workspaces[key] = ws
        return ws


def _check_operand(x: torch.Tensor, name: str, dtype: torch.dtype) -> None:
    if not x.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor (there is no CPU path)")
    if x.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {x.dtype}")
    if x.dim() != 2:
        raise ValueError(f"{name} must be 2-D, got shape {tuple(x.shape)}")
    if x.shape[1] > 1 and x.stride(1) != 1:
        raise ValueError(f"{name} must have unit column stride (row-major rows)")


def _ld(x: torch.Tensor) -> int:
    return max(int(x.stride(0)), int(x.shape[1])) if x.shape[0] > 1 else int(x.shape[1])


def tsmttsm(A: torch.Tensor, B: torch.Tensor, C: torch.Tensor | None = None, *, accumulate: bool = False,
            variant: int = -1, stream: torch.cuda.Stream | None = None) -> torch.Tensor:
    """C = A^T B (or C += A^T B with ``accumulate=True``) in FP64.

    The Python face of ``tsm_gemm_tn_f64`` (the reference's
    ``tsmttsm*<double, M, ...>(q, K, A, B, C)``, tsmttsm.hh:15-586, which
    always accumulates).  Returns C; allocates it (m x k) when not given.
    """
    _check_operand(A, "A", torch.float64)
    _check_operand(B, "B", torch.float64)
    if A.shape[0] != B.shape[0]:
        raise ValueError(f"A and B must have the same number of rows, got {A.shape[0]} and {B.shape[0]}")
    if A.device != B.device:
        raise ValueError("A and B must be on the same device")
    n, m = A.shape
    k = B.shape[1]
    if C is None:
        if accumulate:
            raise ValueError("accumulate=True needs an existing C")
        C = torch.empty((m, k), dtype=torch.float64, device=A.device)
    else:
        _check_operand(C, "C", torch.float64)
        if tuple(C.shape) != (m, k):
            raise ValueError(f"C must be {m}x{k}, got {tuple(C.shape)}")
    lib = _capi.load()
    with torch.cuda.device(A.device):
        sh = _stream_handle(A.device, stream)
        need = lib.tsm_gemm_tn_workspace_size(n, m, k)
        if need == 0:
            _capi.check(1, "tsm_gemm_tn_workspace_size")
        ws = workspace(A.device, need, sh)
        st = lib.tsm_gemm_tn_f64_variant(sh, n, m, k, A.data_ptr(), _ld(A), B.data_ptr(), _ld(B), C.data_ptr(),
                                         _ld(C), 1 if accumulate else 0, ws.data_ptr(), ws.numel(), int(variant))
        _capi.check(st, "tsm_gemm_tn_f64")
    return C


def default_variant(A: torch.Tensor, B: torch.Tensor) -> int:
    """Index of the variant tsmttsm() would run for these operands."""
    lib = _capi.load()
    return lib.tsm_gemm_tn_default_variant(A.shape[0], A.shape[1], B.shape[1], A.data_ptr(), _ld(A),
                                           B.data_ptr(), _ld(B))


def workspace_status(device: torch.device | None = None, stream: torch.cuda.Stream | None = None) -> int:
    """Reads and clears the device error word of the (device, stream)
    workspace; nonzero means a kernel gave up a bounded wait."""
    device = device or torch.device("cuda", torch.cuda.current_device())
    lib = _capi.load()
    sh = _stream_handle(device, stream)
    key = (device.index if device.index is not None else torch.cuda.current_device(), sh)
    ws = _workspaces.get(key)
    if ws is None:
        return 0
    bits = ctypes.c_uint(0)
    st = lib.tsm_workspace_check(sh, ws.data_ptr(), ctypes.byref(bits))
    if st not in (0, 5):
        _capi.check(st, "tsm_workspace_check")
    return int(bits.value)


def fill_uniform(x: torch.Tensor, seed: int, stream_id: int = 0, stream: torch.cuda.Stream | None = None) -> torch.Tensor:
    """Fills a contiguous FP64 CUDA tensor with the library's reproducible
    uniform[-1, 1) values (the same bits as the oracle's host generator)."""
    if not (x.is_cuda and x.dtype == torch.float64 and x.is_contiguous()):
        raise ValueError("fill_uniform needs a contiguous float64 CUDA tensor")
    lib = _capi.load()
    with torch.cuda.device(x.device):
        st = lib.tsm_fill_uniform_f64(_stream_handle(x.device, stream), x.data_ptr(), x.numel(),
                                      seed & 0xFFFFFFFFFFFFFFFF, stream_id & 0xFFFFFFFFFFFFFFFF)
    _capi.check(st, "tsm_fill_uniform_f64")
    return x
