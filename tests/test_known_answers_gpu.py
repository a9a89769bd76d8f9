"""Known-answer tests: inputs whose products and sums are exact in floating
point, so every kernel -- whatever its summation order, tile or grid -- must
return the exact C bit for bit.

* all ones: C = n in every entry;
* stacked identity blocks: A = B = [I; I; ...] (reps blocks) gives C = reps I;
* rank one in small integers: A[r][i] = a_r u_i, B[r][j] = a_r v_j with
  |a_r| <= 3, |u_i|, |v_j| <= 4, so C = (sum_r a_r^2) u v^T, every partial sum
  an integer far below 2^53 (FP64), 2^24 within one FP32 tile of the split
  forms (256 rows), and every value exact in TF32 and BF16.

The expected C is formed with integer arithmetic on the host.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

N = 100003  # not a multiple of any chunk or tile


def rank_one(n, m, k, seed):
    rng = np.random.default_rng(seed)
    a = (np.arange(n) % 7) - 3
    u = rng.integers(-4, 5, size=m)
    v = rng.integers(-4, 5, size=k)
    A = np.outer(a, u)
    B = np.outer(a, v)
    C = int(np.sum(a * a)) * np.outer(u, v)
    return A, B, C


def cases(m, k):
    """(name, A, B, exact C) as int64 arrays."""
    out = [("ones", np.ones((N, m), np.int64), np.ones((N, k), np.int64), np.full((m, k), N, np.int64))]
    if m == k:
        reps = N // m
        Id = np.tile(np.eye(m, dtype=np.int64), (reps, 1))
        out.append(("identity blocks", Id, Id, reps * np.eye(m, dtype=np.int64)))
    out.append(("rank one",) + rank_one(N, m, k, 7 * m + k))
    return out


def dev64(x, gpu):
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).to(gpu)


SHAPES = [(1, 1), (3, 5), (8, 8), (16, 16), (32, 32), (48, 48), (64, 64), (4, 32), (1, 64), (12, 40)]


@pytest.mark.parametrize("m,k", SHAPES)
def test_every_variant_exact(gpu, m, k):
    """Every compiled FP64 variant that takes (m, k) -- SIMT, direct, FP64
    tensor cores, and the Gram kernels when B is A -- returns the exact C;
    so do the column-major path and the allocation-free entry point."""
    from tsm_benchmark_b200 import _capi, tsmttsm, variants
    ran = 0
    for name, A, B, C in cases(m, k):
        dA, dB = dev64(A, gpu), dev64(B, gpu)
        same = name == "identity blocks"  # A is B
        for v in variants():
            if v["dtype"] != "f64":
                continue
            fits = (m == v["wa"] and k == v["wb"]) if v["exact"] else (m <= v["wa"] and k <= v["wb"])
            if not fits or (v["gram"] and not same):
                continue
            got = tsmttsm(dA, dA if same else dB, variant=v["index"]).cpu().numpy()
            assert np.array_equal(got, C.astype(np.float64)), (name, v["name"])
            ran += 1
        # column-major operands, read in place
        At, Bt = dev64(A.T, gpu), dev64(B.T, gpu)
        assert np.array_equal(tsmttsm(At.t(), Bt.t()).cpu().numpy(), C), (name, "column-major")
        # the allocation-free entry point
        lib = _capi.load()
        out = torch.full((m, k), float("nan"), dtype=torch.float64, device=gpu)
        st = lib.tsm_gemm_tn_f64_noalloc(int(torch.cuda.current_stream(gpu).cuda_stream), A.shape[0], m, k,
                                         dA.data_ptr(), m, dB.data_ptr(), k, out.data_ptr(), k, 0)
        if st == 0:
            assert np.array_equal(out.cpu().numpy(), C), (name, "noalloc")
        else:
            assert st == 2  # beyond the built-in scratch (wide shapes)
    assert ran >= 1


@pytest.mark.parametrize("m,k", [(32, 32), (8, 24), (4, 4), (16, 32)])
def test_split_forms_exact(gpu, m, k):
    """The precision forms on FP32 data that every part represents exactly
    (lo parts zero): TF32 hi/lo, BF16 hi/lo and hi/mid/lo all return the
    exact C."""
    from tsm_benchmark_b200 import tsmttsm_split
    for name, A, B, C in cases(m, k):
        A32 = torch.from_numpy(A.astype(np.float32)).to(gpu)
        B32 = torch.from_numpy(B.astype(np.float32)).to(gpu)
        for kind in ("tf32", "bf16x2", "bf16x3"):
            got = tsmttsm_split(A32, B32, kind=kind).cpu().numpy()
            assert np.array_equal(got, C), (name, kind)


def test_batched_gram_and_backward_exact(gpu):
    """The batched launch (every width class), the Gram product and the
    fused backward (integer dC) on exact data."""
    from tsm_benchmark_b200 import BatchedTSMTTSM, gram, tsmttsm_backward
    As, Bs, Cs = [], [], []
    for i, (m, k) in enumerate([(a, b) for a in (4, 8, 16, 32) for b in (4, 8, 16, 32)]):
        A, B, C = rank_one(N // 3 + 17 * i, m, k, i)
        As.append(dev64(A, gpu))
        Bs.append(dev64(B, gpu))
        Cs.append(C)
    for path in ("dmma", "simt"):
        paths = {(m, k): path for m in (16, 32) for k in (16, 32)}
        got = BatchedTSMTTSM(As, Bs, class_paths=paths).run()
        for i, (g, C) in enumerate(zip(got, Cs)):
            assert np.array_equal(g.cpu().numpy(), C), (path, i)
    for m in (8, 16, 32, 64):
        A, _, _ = rank_one(N, m, m, m)
        assert np.array_equal(gram(dev64(A, gpu)).cpu().numpy(), A.T @ A), m
    A, B, _ = rank_one(N, 16, 16, 3)
    dC = np.random.default_rng(4).integers(-3, 4, size=(16, 16))
    dA, dB = tsmttsm_backward(dev64(A, gpu), dev64(B, gpu), dev64(dC, gpu))
    assert np.array_equal(dA.cpu().numpy(), B @ dC.T)
    assert np.array_equal(dB.cpu().numpy(), A @ dC)
