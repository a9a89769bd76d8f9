"""Row-sharded TSMTTSM over several GPUs (one process per GPU).

C = A^T B is a sum over rows, so contiguous row blocks of A and B shard
across ranks with no exchange while streaming; the only exchange step is the
sum of the ranks' m x k partials (at most 32 KB).  It is done as an
all-gather followed by a sum in rank order, so every rank ends with the same,
bit-reproducible C (an all-reduce would leave the order to the library).
The reference has no multi-device path; this is the row split its single
kernel generalises to.  A batch of independent products shards by problem
instead (shard_problems / batched_sharded): no partial sums at all, one
all-gather of the results.
"""
from __future__ import annotations

from typing import Callable, Optional, Sequence

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


# ------------------------------------------------------------------ batches
def shard_problems(costs: Sequence[int], world: int) -> list[list[int]]:
    """Problems of a batch -> ranks, balanced by cost (e.g. the bytes
    8 n_i (m_i + k_i)): largest first, each to the least-loaded rank (the
    lowest rank on ties), so every rank computes the same assignment.
    Returns, per rank, its problem indices in increasing order."""
    load = [0] * world
    owned: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda j: (-int(costs[j]), j)):
        r = min(range(world), key=lambda q: (load[q], q))
        owned[r].append(i)
        load[r] += int(costs[i])
    return [sorted(o) for o in owned]


def gather_problem_results(owned_C: Sequence[torch.Tensor], assignment: Sequence[Sequence[int]],
                           shapes: Sequence[tuple[int, int]], group: Optional[dist.ProcessGroup] = None,
                           device: Optional[torch.device] = None) -> list[torch.Tensor]:
    """Every rank's C_i of a sharded batch, on every rank, bit for bit.

    ``owned_C`` are this rank's results in the order of
    ``assignment[rank]``; ``shapes[i]`` is (m_i, k_i).  One all-gather of a
    flat FP64 buffer per rank (padded to the largest), then each C_i is cut
    from its owner's buffer: no arithmetic, so the values are exact."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    sizes = [sum(shapes[i][0] * shapes[i][1] for i in owned) for owned in assignment]
    width = max(1, max(sizes))
    if device is not None:
        dev = device
    elif owned_C:
        dev = owned_C[0].device
    elif dist.get_backend(group) == "nccl":
        # a rank that owns no problem still joins the all-gather, from its GPU
        dev = torch.device("cuda", torch.cuda.current_device())
    else:
        dev = torch.device("cpu")
    flat = torch.zeros(width, dtype=torch.float64, device=dev)
    off = 0
    for c, i in zip(owned_C, assignment[rank]):
        mk = shapes[i][0] * shapes[i][1]
        flat[off:off + mk] = c.reshape(-1).to(torch.float64)
        off += mk
    if world == 1:
        parts = [flat]
    else:
        parts = [torch.empty_like(flat) for _ in range(world)]
        dist.all_gather(parts, flat, group=group)
    out: list[Optional[torch.Tensor]] = [None] * len(shapes)
    for r, owned in enumerate(assignment):
        off = 0
        for i in owned:
            m, k = shapes[i]
            out[i] = parts[r][off:off + m * k].view(m, k).clone()
            off += m * k
    return out  # type: ignore[return-value]


def batched_sharded(As: Sequence[torch.Tensor], Bs: Sequence[torch.Tensor], shapes: Sequence[tuple[int, int, int]],
                    *, group: Optional[dist.ProcessGroup] = None, local_fn: Optional[Callable] = None,
                    device: Optional[torch.device] = None) -> list[torch.Tensor]:
    """C_i = A_i^T B_i for a batch sharded by problem: ``shapes[i]`` is
    (n_i, m_i, k_i) of every problem (the same list on every rank); ``As``
    and ``Bs`` hold only this rank's problems, in the order of
    ``shard_problems`` (costs 8 n (m + k)).  This rank's problems run as one
    batched launch (``local_fn(As, Bs) -> [C]`` replaces it); every rank
    returns all C_i."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    assignment = shard_problems([8 * n * (m + k) for n, m, k in shapes], world)
    if len(As) != len(assignment[rank]) or len(Bs) != len(As):
        raise ValueError(f"rank {rank} owns {len(assignment[rank])} problems, got {len(As)} A and {len(Bs)} B")
    if local_fn is None:
        if As:
            from .batched import BatchedTSMTTSM
            bt = BatchedTSMTTSM(list(As), list(Bs))
            bt.run()
            Cs = list(bt.Cs)
        else:
            Cs = []
    else:
        Cs = list(local_fn(As, Bs))
    return gather_problem_results(Cs, assignment, [(m, k) for _, m, k in shapes], group, device)
