"""Row-sharded TSMTTSM over several GPUs (one process per GPU).

C = A^T B is a sum over rows, so contiguous row blocks of A and B shard
across ranks with no exchange while streaming; the only exchange step is the
sum of the ranks' m x k partials (at most 32 KB).  It is done as an
all-gather followed by a sum in rank order, so every rank ends with the same,
bit-reproducible C (an all-reduce would leave the order to the library).
The reference has no multi-device path; this is the row split its single
kernel generalises to.
"""
from __future__ import annotations

from typing import Callable, Optional

import torch
import torch.distributed as dist


def reduce_partials_(C: torch.Tensor, group: Optional[dist.ProcessGroup] = None) -> torch.Tensor:
    """In place: C <- C_0 + C_1 + ... + C_{N-1} summed in rank order."""
    world = dist.get_world_size(group)
    if world == 1:
        return C
    src = C.contiguous()
    parts = [torch.empty_like(src) for _ in range(world)]
    dist.all_gather(parts, src, group=group)
    total = parts[0].clone()
    for p in parts[1:]:
        total += p
    C.copy_(total)
    return C


def shard_rows(n: int, rank: int, world: int) -> tuple[int, int]:
    """[start, stop) of this rank's contiguous row block (sizes differ by at
    most one row)."""
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def tsmttsm_sharded(A_local: torch.Tensor, B_local: torch.Tensor, C: Optional[torch.Tensor] = None, *,
                    accumulate: bool = False, group: Optional[dist.ProcessGroup] = None,
                    local_fn: Optional[Callable] = None) -> torch.Tensor:
    """C = sum over all ranks of A_local^T B_local (C += ... if accumulate).

    Each rank passes its own row block.  ``local_fn(A, B) -> C_partial``
    replaces the local product (default: the CUDA library); the cross-rank
    sum is always the deterministic rank-order reduction above."""
    if local_fn is None:
        from .api import tsmttsm
        part = tsmttsm(A_local, B_local)
    else:
        part = local_fn(A_local, B_local)
    reduce_partials_(part, group)
    if C is None:
        return part
    if accumulate:
        C += part
    else:
        C.copy_(part)
    return C
