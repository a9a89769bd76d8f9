"""Python entry points over the C ABI, taking torch CUDA tensors.

torch is used for device memory and streams only; every computation is a
call into libtsm_b200.so.  Shapes follow include/tsm.h: A (n x m), B (n x k)
row-major (unit column stride, any row stride), C (m x k); FP64 operands
in other layouts (column-major ``X.T`` views included) go through
``tsm_gemm_tn_strided_f64``.
"""
from __future__ import annotations

import contextlib
import ctypes
import threading

import torch

from . import _capi

_ws_lock = threading.Lock()
_workspaces: dict[tuple[int, int], torch.Tensor] = {}


def _stream(device: torch.device, stream: torch.cuda.Stream | None) -> torch.cuda.Stream:
    return stream if stream is not None else torch.cuda.current_stream(device)


def _stream_handle(device: torch.device, stream: torch.cuda.Stream | None) -> int:
    return int(_stream(device, stream).cuda_stream)


def _on_stream(device: torch.device, stream):
    """Context in which torch allocates and launches on `stream` (a
    torch.cuda.Stream or a raw cudaStream_t handle)."""
    if isinstance(stream, torch.cuda.Stream):
        return torch.cuda.stream(stream)
    if torch.cuda.is_available():
        if int(stream) == 0:  # the legacy default stream, torch's default stream
            return torch.cuda.stream(torch.cuda.default_stream(device))
        return torch.cuda.stream(torch.cuda.ExternalStream(int(stream), device=device))
    return contextlib.nullcontext()  # no device: only fake allocators reach here


def workspace(device: torch.device, nbytes: int, stream) -> torch.Tensor:
    """A zero-initialised device workspace of at least `nbytes`, one per
    (device, stream): calls on one stream are ordered, so they may share it.

    `stream` is the torch.cuda.Stream (or raw handle) the kernels will run
    on.  The buffer is allocated and zero-filled ON that stream, so the
    zero-fill is ordered before the first launch that uses it, and the
    caching allocator hands a replaced (smaller) buffer out again only to
    later work on the same stream, after the launches that used it."""
    handle = int(stream.cuda_stream) if isinstance(stream, torch.cuda.Stream) else int(stream)
    key = (device.index if device.index is not None else torch.cuda.current_device(), handle)
    with _ws_lock:
        ws = _workspaces.get(key)
        if ws is None or ws.numel() < nbytes:
            with _on_stream(device, stream):
                ws = torch.zeros(max(nbytes, 1 << 20), dtype=torch.uint8, device=device)
            _workspaces[key] = ws
        return ws


def _check_operand(x: torch.Tensor, name: str, dtype: torch.dtype, any_strides: bool = False) -> None:
    if not x.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor (there is no CPU path)")
    if x.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {x.dtype}")
    if x.dim() != 2:
        raise ValueError(f"{name} must be 2-D, got shape {tuple(x.shape)}")
    if not any_strides and x.shape[0] > 0 and x.shape[1] > 1 and x.stride(1) != 1:
        raise ValueError(f"{name} must have unit column stride (row-major rows)")


def _row_major(x: torch.Tensor) -> bool:
    return x.shape[0] == 0 or x.shape[1] == 1 or x.stride(1) == 1


def _strides(x: torch.Tensor) -> tuple[int, int]:
    """(row stride, column stride) in elements, >= 1: strides along an
    extent of one carry no layout and are reported as 1."""
    r = int(x.stride(0)) if x.shape[0] > 1 else 1
    c = int(x.stride(1)) if x.shape[1] > 1 else 1
    if r < 1 or c < 1:
        raise ValueError("operands need positive strides (no broadcast or reversed views)")
    return r, c


def _ld(x: torch.Tensor) -> int:
    """Leading dimension (elements between rows); strides of empty or
    single-row tensors carry no layout, so those report their width."""
    return max(int(x.stride(0)), int(x.shape[1])) if x.shape[0] > 1 else max(1, int(x.shape[1]))


_PLAIN = {torch.float64: ("tsm_gemm_tn_f64_variant", 0), torch.float32: ("tsm_gemm_tn_f32_variant", 1)}


def tsmttsm(A: torch.Tensor, B: torch.Tensor, C: torch.Tensor | None = None, *, accumulate: bool = False,
            variant: int = -1, stream: torch.cuda.Stream | None = None) -> torch.Tensor:
    """C = A^T B (or C += A^T B with ``accumulate=True``), FP64 or FP32.

    The Python face of ``tsm_gemm_tn_f64`` / ``tsm_gemm_tn_f32`` (the
    reference's ``tsmttsm*<double, M, ...>(q, K, A, B, C)``,
    tsmttsm.hh:15-586, which always accumulates).  A, B and C share one
    dtype.  FP64 operands may have any positive strides: column-major ones
    (``X.T`` of a row-major m x n X) and mixed layouts run through
    ``tsm_gemm_tn_strided_f64`` (``variant`` is then ignored).  Returns C;
    allocates it (m x k) when not given.
    """
    if A.dtype not in _PLAIN:
        raise TypeError(f"A must be float64 or float32, got {A.dtype}")
    fn_name, _ = _PLAIN[A.dtype]
    f64 = A.dtype == torch.float64
    _check_operand(A, "A", A.dtype, any_strides=f64)
    _check_operand(B, "B", A.dtype, any_strides=f64)
    if A.shape[0] != B.shape[0]:
        raise ValueError(f"A and B must have the same number of rows, got {A.shape[0]} and {B.shape[0]}")
    if A.device != B.device:
        raise ValueError("A and B must be on the same device")
    n, m = A.shape
    k = B.shape[1]
    if C is None:
        if accumulate:
            raise ValueError("accumulate=True needs an existing C")
        C = torch.empty((m, k), dtype=A.dtype, device=A.device)
    else:
        _check_operand(C, "C", A.dtype)
        if tuple(C.shape) != (m, k):
            raise ValueError(f"C must be {m}x{k}, got {tuple(C.shape)}")
    lib = _capi.load()
    with torch.cuda.device(A.device):
        so = _stream(A.device, stream)
        sh = int(so.cuda_stream)
        need = lib.tsm_gemm_tn_workspace_size(n, m, k)
        if need == 0:
            _capi.check(1, "tsm_gemm_tn_workspace_size")
        ws = workspace(A.device, need, so)
        if _row_major(A) and _row_major(B):
            st = getattr(lib, fn_name)(sh, n, m, k, A.data_ptr(), _ld(A), B.data_ptr(), _ld(B), C.data_ptr(),
                                       _ld(C), 1 if accumulate else 0, ws.data_ptr(), ws.numel(), int(variant))
            _capi.check(st, fn_name)
        else:
            (ar, ac), (br, bc) = _strides(A), _strides(B)
            st = lib.tsm_gemm_tn_strided_f64(sh, n, m, k, A.data_ptr(), ar, ac, B.data_ptr(), br, bc, C.data_ptr(),
                                             _ld(C), 1 if accumulate else 0, ws.data_ptr(), ws.numel())
            _capi.check(st, "tsm_gemm_tn_strided_f64")
    return C


def gram(A: torch.Tensor, C: torch.Tensor | None = None, *, accumulate: bool = False,
         stream: torch.cuda.Stream | None = None) -> torch.Tensor:
    """C = A^T A (or C += A^T A), FP64: reads A once and writes C exactly
    symmetric (``tsm_gram_f64``).  ``tsmttsm(A, A)`` takes the same path.
    Returns C; allocates it (m x m) when not given."""
    _check_operand(A, "A", torch.float64)
    n, m = A.shape
    if C is None:
        if accumulate:
            raise ValueError("accumulate=True needs an existing C")
        C = torch.empty((m, m), dtype=torch.float64, device=A.device)
    else:
        _check_operand(C, "C", torch.float64)
        if tuple(C.shape) != (m, m):
            raise ValueError(f"C must be {m}x{m}, got {tuple(C.shape)}")
    lib = _capi.load()
    with torch.cuda.device(A.device):
        so = _stream(A.device, stream)
        sh = int(so.cuda_stream)
        need = lib.tsm_gemm_tn_workspace_size(n, m, m)
        if need == 0:
            _capi.check(1, "tsm_gemm_tn_workspace_size")
        ws = workspace(A.device, need, so)
        st = lib.tsm_gram_f64(sh, n, m, A.data_ptr(), _ld(A), C.data_ptr(), _ld(C), 1 if accumulate else 0,
                              ws.data_ptr(), ws.numel())
        _capi.check(st, "tsm_gram_f64")
    return C


def block_orthogonalize(A: torch.Tensor, B: torch.Tensor, C: torch.Tensor | None = None, *,
                        stream: torch.cuda.Stream | None = None) -> torch.Tensor:
    """C = A^T B, then B <- B - A C in place (FP64; ``tsm_block_orth_f64``):
    one block Gram-Schmidt step against A's columns when they are
    orthonormal.  Returns C (m x k), allocated when not given."""
    _check_operand(A, "A", torch.float64)
    _check_operand(B, "B", torch.float64)
    n, m = A.shape
    k = B.shape[1]
    if B.shape[0] != n:
        raise ValueError("A and B must have the same number of rows")
    if C is None:
        C = torch.empty((m, k), dtype=torch.float64, device=A.device)
    else:
        _check_operand(C, "C", torch.float64)
        if tuple(C.shape) != (m, k):
            raise ValueError(f"C must be {m}x{k}, got {tuple(C.shape)}")
    lib = _capi.load()
    with torch.cuda.device(A.device):
        so = _stream(A.device, stream)
        sh = int(so.cuda_stream)
        need = lib.tsm_gemm_tn_workspace_size(n, m, k)
        if need == 0:
            _capi.check(1, "tsm_gemm_tn_workspace_size")
        ws = workspace(A.device, need, so)
        st = lib.tsm_block_orth_f64(sh, n, m, k, A.data_ptr(), _ld(A), B.data_ptr(), _ld(B), C.data_ptr(), _ld(C),
                                    ws.data_ptr(), ws.numel())
        _capi.check(st, "tsm_block_orth_f64")
    return C


def default_variant(A: torch.Tensor, B: torch.Tensor) -> int:
    """Index of the variant tsmttsm() would run for these operands."""
    lib = _capi.load()
    dtype = _PLAIN[A.dtype][1] if A.dtype in _PLAIN else -1
    return lib.tsm_gemm_tn_default_variant(dtype, A.shape[0], A.shape[1], B.shape[1], A.data_ptr(), _ld(A),
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


_TSMM = {torch.float64: "tsm_tsmm_f64", torch.float32: "tsm_tsmm_f32"}
_BWD = {torch.float64: "tsm_gemm_tn_backward_f64", torch.float32: "tsm_gemm_tn_backward_f32"}


def tsmm(X: torch.Tensor, W: torch.Tensor, Y: torch.Tensor | None = None, *, transpose_w: bool = False,
         accumulate: bool = False, stream: torch.cuda.Stream | None = None) -> torch.Tensor:
    """Y = X @ W (or X @ W.T with ``transpose_w``), tall-skinny X (n x p),
    small W; ``accumulate=True`` adds into Y.  ``tsm_tsmm_f64`` / ``_f32``."""
    if X.dtype not in _TSMM:
        raise TypeError(f"X must be float64 or float32, got {X.dtype}")
    _check_operand(X, "X", X.dtype)
    if not W.is_cuda or W.dtype != X.dtype or W.dim() != 2:
        raise ValueError("W must be a 2-D CUDA tensor of X's dtype")
    n, p = X.shape
    if transpose_w:
        q, pw = W.shape
        w_row, w_col = W.stride(1), W.stride(0)
    else:
        pw, q = W.shape
        w_row, w_col = W.stride(0), W.stride(1)
    if pw != p:
        raise ValueError(f"W must have {p} rows (after transposition), got {pw}")
    if Y is None:
        if accumulate:
            raise ValueError("accumulate=True needs an existing Y")
        Y = torch.empty((n, q), dtype=X.dtype, device=X.device)
    else:
        _check_operand(Y, "Y", X.dtype)
        if tuple(Y.shape) != (n, q):
            raise ValueError(f"Y must be {n}x{q}, got {tuple(Y.shape)}")
    lib = _capi.load()
    with torch.cuda.device(X.device):
        so = _stream(X.device, stream)
        sh = int(so.cuda_stream)
        ws = workspace(X.device, 256, so)
        st = getattr(lib, _TSMM[X.dtype])(sh, n, p, q, X.data_ptr(), _ld(X), W.data_ptr(), w_row, w_col,
                                           Y.data_ptr(), _ld(Y), 1 if accumulate else 0, ws.data_ptr(), ws.numel())
        _capi.check(st, _TSMM[X.dtype])
    return Y


def tsmttsm_backward(A: torch.Tensor, B: torch.Tensor, dC: torch.Tensor, *, need_dA: bool = True,
                     need_dB: bool = True, stream: torch.cuda.Stream | None = None):
    """(dA, dB) = (B @ dC.T, A @ dC) for C = A^T B, in one launch
    (``tsm_gemm_tn_backward_*``); an output not needed is returned as None."""
    if A.dtype not in _BWD:
        raise TypeError(f"A must be float64 or float32, got {A.dtype}")
    _check_operand(A, "A", A.dtype)
    _check_operand(B, "B", A.dtype)
    n, m = A.shape
    k = B.shape[1]
    if B.shape[0] != n:
        raise ValueError("A and B must have the same number of rows")
    if tuple(dC.shape) != (m, k) or dC.dtype != A.dtype or not dC.is_cuda:
        raise ValueError(f"dC must be a {m}x{k} CUDA tensor of A's dtype")
    dC = dC.contiguous()
    dA = torch.empty((n, m), dtype=A.dtype, device=A.device) if need_dA else None
    dB = torch.empty((n, k), dtype=A.dtype, device=A.device) if need_dB else None
    lib = _capi.load()
    with torch.cuda.device(A.device):
        so = _stream(A.device, stream)
        sh = int(so.cuda_stream)
        ws = workspace(A.device, 256, so)
        st = getattr(lib, _BWD[A.dtype])(sh, n, m, k, A.data_ptr(), _ld(A), B.data_ptr(), _ld(B), dC.data_ptr(),
                                          k, dA.data_ptr() if dA is not None else None, m,
                                          dB.data_ptr() if dB is not None else None, k, 0, ws.data_ptr(),
                                          ws.numel())
        _capi.check(st, _BWD[A.dtype])
    return dA, dB


_SPLIT_KINDS = {"tf32": 0, "bf16x2": 2, "bf16x3": 3}


def tsmttsm_split(A: torch.Tensor, B: torch.Tensor, C: torch.Tensor | None = None, *, accumulate: bool = False,
                  kind: str = "tf32", stream: torch.cuda.Stream | None = None) -> torch.Tensor:
    """C (float64) = A^T B for float32 A, B (m, k <= 32) on the tensor cores,
    FP32 accumulation per tile, FP64 sums.  ``kind``: "tf32" -- TF32 hi/lo
    parts (``tsm_gemm_tn_f32_split``, error <= 1e-6); "bf16x2" -- BF16
    hi/lo (``tsm_gemm_tn_f32_split_bf16`` with 2 parts, about 1e-5);
    "bf16x3" -- BF16 hi/mid/lo (3 parts).  The BF16 kinds need m and k
    multiples of 4."""
    if kind not in _SPLIT_KINDS:
        raise ValueError(f"kind must be one of {sorted(_SPLIT_KINDS)}, got {kind!r}")
    _check_operand(A, "A", torch.float32)
    _check_operand(B, "B", torch.float32)
    n, m = A.shape
    k = B.shape[1]
    if B.shape[0] != n:
        raise ValueError("A and B must have the same number of rows")
    if C is None:
        if accumulate:
            raise ValueError("accumulate=True needs an existing C")
        C = torch.empty((m, k), dtype=torch.float64, device=A.device)
    else:
        _check_operand(C, "C", torch.float64)
    lib = _capi.load()
    with torch.cuda.device(A.device):
        so = _stream(A.device, stream)
        sh = int(so.cuda_stream)
        need = lib.tsm_gemm_tn_workspace_size(n, m, k)
        ws = workspace(A.device, need, so)
        if kind == "tf32":
            st = lib.tsm_gemm_tn_f32_split(sh, n, m, k, A.data_ptr(), _ld(A), B.data_ptr(), _ld(B), C.data_ptr(),
                                           _ld(C), 1 if accumulate else 0, ws.data_ptr(), ws.numel())
            _capi.check(st, "tsm_gemm_tn_f32_split")
        else:
            st = lib.tsm_gemm_tn_f32_split_bf16(sh, n, m, k, A.data_ptr(), _ld(A), B.data_ptr(), _ld(B),
                                                C.data_ptr(), _ld(C), 1 if accumulate else 0, _SPLIT_KINDS[kind],
                                                ws.data_ptr(), ws.numel())
            _capi.check(st, "tsm_gemm_tn_f32_split_bf16")
    return C
