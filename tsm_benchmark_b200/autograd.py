"""Differentiable C = A^T B (the differentiation form).

``TSMTTSMFunction`` runs the forward on the plain kernels (FP64 or FP32
storage) and the backward on one fused TSMM launch:
    dA = B . dC^T,   dB = A . dC
(``tsm_gemm_tn_backward_*``), skipping whichever input needs no gradient.
The reference has no backward; torch is used only for the autograd plumbing.
"""
from __future__ import annotations

import torch

from .api import tsmttsm, tsmttsm_backward


class TSMTTSMFunction(torch.autograd.Function):
    """C = A^T B with hand-written forward and backward kernels."""

    @staticmethod
    def forward(ctx, A: torch.Tensor, B: torch.Tensor) -> torch.Tensor:
        A = A if A.stride(-1) == 1 else A.contiguous()
        B = B if B.stride(-1) == 1 else B.contiguous()
        ctx.save_for_backward(A, B)
        return tsmttsm(A, B)

    @staticmethod
    def backward(ctx, dC: torch.Tensor):
        A, B = ctx.saved_tensors
        need_a, need_b = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        if not (need_a or need_b):
            return None, None
        dA, dB = tsmttsm_backward(A, B, dC.to(A.dtype), need_dA=need_a, need_dB=need_b)
        return dA, dB


def gram_tn(A: torch.Tensor, B: torch.Tensor) -> torch.Tensor:
    """Differentiable A^T B for tall-skinny A (n x m) and B (n x k)."""
    return TSMTTSMFunction.apply(A, B)
