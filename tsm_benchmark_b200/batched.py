"""The batching form: many FP64 products C_p = A_p^T B_p in one launch.

    bt = BatchedTSMTTSM(As, Bs)          # plan built once (host schedule)
    Cs = bt.run()                        # one persistent kernel launch
    g = bt.capture_graph(); g.replay()   # the same launch inside a CUDA graph

Widths m, k in {4, 8, 16, 32}, contiguous 16-byte aligned operands (the
library's batched kernel); the plan pins the operand and output pointers.
"""
from __future__ import annotations

import ctypes

import torch

from . import _capi
from .api import _stream


_PATHS = {"dmma": 0, "simt": 1}
_WIDTHS = (4, 8, 16, 32)


def _class_index(m: int, k: int) -> int:
    """Width class of the batched kernel: 4 log2(m / 4) + log2(k / 4)."""
    if m not in _WIDTHS or k not in _WIDTHS:
        return -1
    return 4 * _WIDTHS.index(m) + _WIDTHS.index(k)


class BatchedTSMTTSM:
    """A plan for C_p = A_p^T B_p (p = 0 .. count-1) and its launch."""

    def __init__(self, As, Bs, Cs=None, *, accumulate: bool = False, stream: torch.cuda.Stream | None = None,
                 class_paths: dict | None = None):
        """``class_paths`` maps a width class (m, k) to its consumer path,
        "dmma" (the FP64 tensor cores, the default of m, k >= 16) or "simt"
        (SIMT register tiles); classes not named take the autotuned path."""
        if len(As) != len(Bs) or not As:
            raise ValueError("As and Bs must be non-empty and of equal length")
        dev = As[0].device
        self.As, self.Bs = list(As), list(Bs)
        self.Cs = list(Cs) if Cs is not None else [
            torch.zeros((a.shape[1], b.shape[1]), dtype=torch.float64, device=dev) for a, b in zip(As, Bs)]
        probs = (_capi.BatchedProblem * len(As))()
        for i, (a, b, c) in enumerate(zip(self.As, self.Bs, self.Cs)):
            for name, x in (("A", a), ("B", b), ("C", c)):
                if not (x.is_cuda and x.dtype == torch.float64 and x.is_contiguous() and x.device == dev):
                    raise ValueError(f"{name}[{i}] must be a contiguous float64 tensor on {dev}")
            if a.shape[0] != b.shape[0] or tuple(c.shape) != (a.shape[1], b.shape[1]):
                raise ValueError(f"problem {i}: shapes {tuple(a.shape)}, {tuple(b.shape)}, {tuple(c.shape)}")
            probs[i] = _capi.BatchedProblem(a.data_ptr(), b.data_ptr(), c.data_ptr(), a.shape[0], a.shape[1],
                                            b.shape[1], b.shape[1], 1 if accumulate else 0)
        self._probs = probs
        lib = _capi.load()
        with torch.cuda.device(dev):
            nbytes = lib.tsm_batched_plan_size_f64(len(As), probs)
            if nbytes == 0:
                raise _capi.TsmError(4, "batched plan: a problem is invalid or outside widths {4, 8, 16, 32}")
            so = _stream(dev, stream)
            # allocated and zeroed on the stream the plan is written on (the
            # init below copies on it and synchronises it)
            with torch.cuda.stream(so):
                self.buffer = torch.zeros(nbytes, dtype=torch.uint8, device=dev)
            self.plan = _capi.BatchedPlan()
            paths = None
            if class_paths:
                paths = (ctypes.c_int * 16)(*([-1] * 16))
                for (m, k), name in class_paths.items():
                    cls = _class_index(m, k)
                    if cls < 0 or name not in _PATHS:
                        raise ValueError(f"class_paths: ({m}, {k}) -> {name!r}")
                    paths[cls] = _PATHS[name]
            st = lib.tsm_batched_plan_init_paths_f64(int(so.cuda_stream), len(As), probs, paths,
                                                     self.buffer.data_ptr(), nbytes, ctypes.byref(self.plan))
            _capi.check(st, "tsm_batched_plan_init_paths_f64")
        self.device = dev
        self._alloc_stream = int(so.cuda_stream)

    @property
    def segments(self) -> int:
        return self.plan.segments

    def run(self, stream: torch.cuda.Stream | None = None):
        """One launch computing every product; returns the list of C."""
        lib = _capi.load()
        with torch.cuda.device(self.device):
            so = _stream(self.device, stream)
            if int(so.cuda_stream) != self._alloc_stream and not torch.cuda.is_current_stream_capturing():
                # the plan's counters are used on another stream: the caching
                # allocator must not reuse the buffer before that work ends
                # (a captured graph's replays are the caller's to order)
                self.buffer.record_stream(so)
            st = lib.tsm_gemm_tn_batched_f64(int(so.cuda_stream), ctypes.byref(self.plan))
        _capi.check(st, "tsm_gemm_tn_batched_f64")
        return self.Cs

    def capture_graph(self) -> torch.cuda.CUDAGraph:
        """The launch captured in a CUDA graph (after one eager run)."""
        self.run()
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self.run(stream=s)
        torch.cuda.current_stream(self.device).wait_stream(s)
        return g
