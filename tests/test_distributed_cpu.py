"""Row-sharded TSMTTSM across ranks: host logic on CPU with gloo, world 2.

The local product is injected (a CPU matmul stands in for the CUDA call,
which needs a GPU); what is tested is the sharding of rows and the
deterministic rank-order reduction of the partials."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, n: int, m: int, k: int, out_dir: str):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from tsm_benchmark_b200.distributed import shard_rows, tsmttsm_sharded
    g = torch.Generator().manual_seed(7)
    A = torch.rand((n, m), generator=g, dtype=torch.float64) * 2 - 1
    B = torch.rand((n, k), generator=g, dtype=torch.float64) * 2 - 1
    lo, hi = shard_rows(n, rank, world)
    C = tsmttsm_sharded(A[lo:hi], B[lo:hi], local_fn=lambda a, b: a.T @ b)
    # accumulate into an existing C
    C2 = torch.ones((m, k), dtype=torch.float64)
    tsmttsm_sharded(A[lo:hi], B[lo:hi], C2, accumulate=True, local_fn=lambda a, b: a.T @ b)
    torch.save({"C": C, "C2": C2, "rows": (lo, hi)}, os.path.join(out_dir, f"rank{rank}.pt"))
    dist.destroy_process_group()


@pytest.mark.parametrize("n", [1001, 4])
def test_sharded_product_two_ranks(tmp_path, n):
    world, m, k = 2, 5, 3
    mp.start_processes(_worker, args=(world, _free_port(), n, m, k, str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    res = [torch.load(tmp_path / f"rank{r}.pt") for r in range(world)]
    # contiguous, disjoint, covering
    assert res[0]["rows"][0] == 0 and res[0]["rows"][1] == res[1]["rows"][0] and res[1]["rows"][1] == n
    g = torch.Generator().manual_seed(7)
    A = torch.rand((n, m), generator=g, dtype=torch.float64) * 2 - 1
    B = torch.rand((n, k), generator=g, dtype=torch.float64) * 2 - 1
    parts = [A[lo:hi].T @ B[lo:hi] for lo, hi in (r["rows"] for r in res)]
    expected = parts[0].clone()
    expected += parts[1]
    for r in res:
        assert torch.equal(r["C"], expected)          # rank-order sum, bit for bit
        assert torch.equal(r["C2"], 1 + expected)
    assert torch.allclose(expected, A.T @ B, rtol=1e-12, atol=1e-12)


def test_shard_rows_balanced():
    from tsm_benchmark_b200.distributed import shard_rows
    for n in (0, 1, 7, 100, 2**26 + 3):
        for world in (1, 2, 3, 8):
            spans = [shard_rows(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1


def _batch_worker(rank: int, world: int, port: int, out_dir: str, count: int = 37):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from tsm_benchmark_b200.distributed import batched_sharded, shard_problems
    shapes = _batch_shapes(count)
    owned = shard_problems([8 * n * (m + k) for n, m, k in shapes], world)[rank]
    As, Bs = [], []
    for i in owned:
        a, b = _batch_operands(i, shapes[i])
        As.append(a)
        Bs.append(b)
    Cs = batched_sharded(As, Bs, shapes, local_fn=lambda xs, ys: [x.T @ y for x, y in zip(xs, ys)])
    torch.save({"Cs": Cs, "owned": owned}, os.path.join(out_dir, f"batch{rank}.pt"))
    dist.destroy_process_group()


def _batch_shapes(count: int = 37):
    g = torch.Generator().manual_seed(11)
    ns = torch.randint(1, 3000, (count,), generator=g).tolist()
    ms = torch.randint(1, 9, (count,), generator=g).tolist()
    ks = torch.randint(1, 9, (count,), generator=g).tolist()
    return list(zip(ns, ms, ks))


def _batch_operands(i, shape):
    n, m, k = shape
    g = torch.Generator().manual_seed(100 + i)
    return (torch.rand((n, m), generator=g, dtype=torch.float64) * 2 - 1,
            torch.rand((n, k), generator=g, dtype=torch.float64) * 2 - 1)


@pytest.mark.parametrize("count", [37, 1])
def test_batched_sharded_by_problem_two_ranks(tmp_path, count):
    """Problems of a batch spread over ranks by cost; every rank ends with
    every C_i, bit for bit the owner's result.  With one problem, rank 1
    owns none and still joins the exchange."""
    world = 2
    mp.start_processes(_batch_worker, args=(world, _free_port(), str(tmp_path), count), nprocs=world,
                       start_method="spawn", join=True)
    res = [torch.load(tmp_path / f"batch{r}.pt") for r in range(world)]
    shapes = _batch_shapes(count)
    if count == 1:
        assert res[0]["owned"] == [0] and res[1]["owned"] == []
    owned = sorted(res[0]["owned"] + res[1]["owned"])
    assert owned == list(range(len(shapes))), "each problem owned by exactly one rank"
    for i, shape in enumerate(shapes):
        a, b = _batch_operands(i, shape)
        ref = a.T @ b
        for r in res:
            assert torch.equal(r["Cs"][i], ref), (i, shape)


def test_shard_problems_balanced_and_deterministic():
    from tsm_benchmark_b200.distributed import shard_problems
    costs = [5, 1, 9, 3, 3, 7, 2, 8, 8, 1]
    for world in (1, 2, 3, 4, 16):
        a = shard_problems(costs, world)
        assert a == shard_problems(costs, world)
        assert sorted(i for o in a for i in o) == list(range(len(costs)))
        loads = [sum(costs[i] for i in o) for o in a]
        # longest-first greedy: no rank exceeds the lightest by more than the largest single cost
        assert max(loads) - min(loads) <= max(costs)
    assert shard_problems([], 3) == [[], [], []]
