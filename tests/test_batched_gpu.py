"""The batching form: many FP64 products in one persistent launch, eager and
under a CUDA graph, against the oracle and the plain path."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

WIDTHS = (4, 8, 16, 32)


def make_problems(dev, oracle_mod, count, nmin, nmax, seed, host=True):
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(nmin), np.log(nmax), size=count)).astype(np.int64)
    ms = rng.choice(WIDTHS, size=count)
    ks = rng.choice(WIDTHS, size=count)
    As, Bs, hostAB = [], [], []
    for i, (n, m, k) in enumerate(zip(ns, ms, ks)):
        if host:
            A, B = oracle_mod.operands(int(n), int(m), int(k), seed * 1000 + i)
            As.append(torch.from_numpy(A).to(dev))
            Bs.append(torch.from_numpy(B).to(dev))
            hostAB.append((A, B))
        else:
            from tsm_benchmark_b200 import fill_uniform
            A = torch.empty((int(n), int(m)), dtype=torch.float64, device=dev)
            B = torch.empty((int(n), int(k)), dtype=torch.float64, device=dev)
            fill_uniform(A, seed * 1000 + i, 0)
            fill_uniform(B, seed * 1000 + i, 1)
            As.append(A)
            Bs.append(B)
    return As, Bs, hostAB


def test_batched_parity_with_oracle(gpu, oracle_mod):
    from tsm_benchmark_b200 import BatchedTSMTTSM
    As, Bs, host = make_problems(gpu, oracle_mod, 96, 1, 20000, 3)
    bt = BatchedTSMTTSM(As, Bs)
    Cs = bt.run()
    torch.cuda.synchronize()
    assert bt.segments >= len(As)
    for i, ((A, B), C) in enumerate(zip(host, Cs)):
        ref = oracle_mod.naive(A, B)
        got = C.cpu().numpy()
        assert oracle_mod.check(ref, got) == -1, i
        nw = oracle_mod.normwise(A, B, ref, got)
        assert nw["err"] <= nw["bound"], (i, nw)


def test_batched_graph_replay_and_determinism(gpu, oracle_mod):
    from tsm_benchmark_b200 import BatchedTSMTTSM, fill_uniform
    As, Bs, _ = make_problems(gpu, oracle_mod, 64, 1000, 300000, 4, host=False)
    bt = BatchedTSMTTSM(As, Bs)
    first = [c.clone() for c in bt.run()]
    g = bt.capture_graph()
    for _ in range(3):
        g.replay()
        torch.cuda.synchronize()
        for c, f in zip(bt.Cs, first):
            assert torch.equal(c, f)
    # new input values, same buffers: the replay sees them
    fill_uniform(As[0], 999, 0)
    g.replay()
    torch.cuda.synchronize()
    assert torch.allclose(bt.Cs[0], As[0].T @ Bs[0], rtol=1e-12, atol=1e-9)


def test_batched_empty_and_accumulate(gpu, oracle_mod):
    from tsm_benchmark_b200 import BatchedTSMTTSM
    As = [torch.zeros((0, 4), dtype=torch.float64, device=gpu), torch.ones((10, 8), dtype=torch.float64, device=gpu)]
    Bs = [torch.zeros((0, 8), dtype=torch.float64, device=gpu), torch.ones((10, 16), dtype=torch.float64, device=gpu)]
    Cs = [torch.full((4, 8), 2.0, dtype=torch.float64, device=gpu),
          torch.full((8, 16), 1.0, dtype=torch.float64, device=gpu)]
    BatchedTSMTTSM(As, Bs, Cs, accumulate=True).run()
    torch.cuda.synchronize()
    assert torch.all(Cs[0] == 2.0) and torch.all(Cs[1] == 11.0)
    BatchedTSMTTSM(As, Bs, Cs).run()
    torch.cuda.synchronize()
    assert torch.all(Cs[0] == 0.0) and torch.all(Cs[1] == 10.0)


def test_batched_rejects_other_widths(gpu):
    from tsm_benchmark_b200 import BatchedTSMTTSM, TsmError
    A = torch.zeros((10, 5), dtype=torch.float64, device=gpu)
    with pytest.raises(TsmError):
        BatchedTSMTTSM([A], [A])


def test_batched_full_config_against_plain(gpu, oracle_mod):
    """The batched form's configuration: 512 problems, n log-uniform in
    [10^3, 10^6], widths in {4, 8, 16, 32}; every C_p equals the plain path's
    within the normwise bound."""
    from tsm_benchmark_b200 import BatchedTSMTTSM, tsmttsm
    As, Bs, _ = make_problems(gpu, oracle_mod, 512, 1000, 1000000, 5, host=False)
    Cs = BatchedTSMTTSM(As, Bs).run()
    torch.cuda.synchronize()
    for A, B, C in zip(As, Bs, Cs):
        ref = tsmttsm(A, B)
        bound = 8 * np.sqrt(A.shape[0]) * 2.0**-53 * float(torch.linalg.norm(A)) * float(torch.linalg.norm(B))
        assert float(torch.linalg.norm(C - ref)) <= bound
    del As, Bs
    torch.cuda.empty_cache()


@pytest.mark.parametrize("path", ["dmma", "simt"])
def test_batched_both_paths_of_the_tensor_core_classes(gpu, oracle_mod, path):
    """The tensor-core classes (m, k in {16, 32}) have two compiled consumer
    paths, FP64 tensor cores and SIMT register tiles; each, forced for every
    class through the plan, matches the oracle on ragged problems mixed with
    the SIMT-only classes (whose path the override leaves alone)."""
    from tsm_benchmark_b200 import BatchedTSMTTSM
    rng = np.random.default_rng(21)
    shapes = [(int(n), m, k) for n, m, k in zip(rng.integers(1, 30000, size=40), rng.choice(WIDTHS, size=40),
                                                 rng.choice(WIDTHS, size=40))]
    shapes += [(70001, 16, 16), (65537, 16, 32), (33333, 32, 16), (100003, 32, 32), (3, 32, 32), (0, 16, 16)]
    As, Bs, host = [], [], []
    for i, (n, m, k) in enumerate(shapes):
        A, B = oracle_mod.operands(n, m, k, 900 + i)
        As.append(torch.from_numpy(A).to(gpu))
        Bs.append(torch.from_numpy(B).to(gpu))
        host.append((A, B))
    paths = {(m, k): path for m in (16, 32) for k in (16, 32)}
    bt = BatchedTSMTTSM(As, Bs, class_paths=paths)
    # the plan runs the kernel instantiation with the SIMT tensor-core paths
    # only when a class was sent down one
    assert bt.plan.flags == (1 if path == "simt" else 0)
    Cs = bt.run()
    torch.cuda.synchronize()
    for i, ((A, B), C) in enumerate(zip(host, Cs)):
        ref = oracle_mod.naive(A, B)
        got = C.cpu().numpy()
        assert oracle_mod.check(ref, got) == -1, (path, shapes[i])
        nw = oracle_mod.normwise(A, B, ref, got)
        assert nw["err"] <= nw["bound"], (path, shapes[i], nw)


def test_batched_class_paths_argument_errors(gpu):
    from tsm_benchmark_b200 import BatchedTSMTTSM
    A = torch.zeros((10, 16), dtype=torch.float64, device=gpu)
    with pytest.raises(ValueError):
        BatchedTSMTTSM([A], [A], class_paths={(16, 16): "tensor"})
    with pytest.raises(ValueError):
        BatchedTSMTTSM([A], [A], class_paths={(12, 16): "simt"})
