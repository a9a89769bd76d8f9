"""The precision form: FP32 storage, TF32 hi/lo split on tcgen05, FP64
result, against the oracle's FP64 product of the same FP32 values."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TARGET = 1e-6  # relative error target vs the FP64 oracle


def scaled_normal(n, w, seed):
    """Standard normal entries, column j scaled by 10^u_j, u_j ~ U[-3, 3]."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, w)).astype(np.float32)
    x *= (10.0 ** rng.uniform(-3, 3, size=w)).astype(np.float32)
    return x


def errors(ref, got, A, B):
    """normwise ||got - ref||_F / ||ref||_F and the largest per-entry error
    relative to sum_r |a_ri| |b_rj| (the entry's own condition scale)."""
    scale = np.abs(A.astype(np.float64)).T @ np.abs(B.astype(np.float64))
    nw = np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-300)
    pe = float(np.max(np.abs(got - ref) / np.maximum(scale, 1e-300)))
    return nw, pe


# Widths that are multiples of 4 take the 2-D TMA kernel (columns beyond the
# width and rows beyond n zero-filled by the tensor maps); (5, 17) takes the
# 1-D bulk kernel with its converter pass.
@pytest.mark.parametrize("n,m,k", [(4096, 32, 32), (100003, 32, 32), (3, 32, 32), (0, 8, 8), (65539, 5, 17),
                                   (20000, 32, 4), (1 << 20, 16, 16), (70001, 8, 24), (129, 12, 28), (1, 4, 4),
                                   (257, 32, 8), (33333, 3, 32)])
def test_split_parity(gpu, oracle_mod, n, m, k):
    from tsm_benchmark_b200 import tsmttsm_split, workspace_status
    A = scaled_normal(n, m, n + m)
    B = scaled_normal(n, k, n + k + 1)
    C = tsmttsm_split(torch.from_numpy(A).to(gpu), torch.from_numpy(B).to(gpu))
    torch.cuda.synchronize()
    assert workspace_status(gpu) == 0
    got = C.cpu().numpy()
    ref = oracle_mod.naive(A, B)
    if n == 0:
        assert np.all(got == 0)
        return
    nw, pe = errors(ref, got, A, B)
    assert nw <= TARGET and pe <= TARGET, (nw, pe)


def test_split_deterministic_and_accumulate(gpu):
    from tsm_benchmark_b200 import tsmttsm_split
    A = torch.from_numpy(scaled_normal(50000, 32, 1)).to(gpu)
    B = torch.from_numpy(scaled_normal(50000, 32, 2)).to(gpu)
    first = tsmttsm_split(A, B).clone()
    for _ in range(3):
        assert torch.equal(tsmttsm_split(A, B), first)
    C = first.clone()
    tsmttsm_split(A, B, C, accumulate=True)
    assert torch.allclose(C, 2 * first, rtol=1e-15, atol=0)


def test_split_full_config(gpu):
    """The precision form's configuration: n = 2^25, m = k = 32, scaled
    normal FP32 data; error against the plain FP64 path on FP64 copies."""
    from tsm_benchmark_b200 import tsmttsm, tsmttsm_split
    n, w = 1 << 25, 32
    g = torch.Generator(device=gpu).manual_seed(3)
    sa = 10.0 ** (torch.rand(w, device=gpu, generator=g) * 6 - 3)
    sb = 10.0 ** (torch.rand(w, device=gpu, generator=g) * 6 - 3)
    A = (torch.randn((n, w), device=gpu, generator=g) * sa).float()
    B = (torch.randn((n, w), device=gpu, generator=g) * sb).float()
    C = tsmttsm_split(A, B)
    ref = tsmttsm(A.double(), B.double())
    nw = float(torch.linalg.norm(C - ref) / torch.linalg.norm(ref))
    scale = tsmttsm(A.double().abs(), B.double().abs())
    pe = float(((C - ref).abs() / scale).max())
    assert nw <= TARGET and pe <= TARGET, (nw, pe)
    del A, B
    torch.cuda.empty_cache()


# BF16 parts (tsm_gemm_tn_f32_split_bf16).  Per value |x - sum of parts| <=
# 2^-16 |x| (2 parts) or 2^-24 |x| (3 parts), so each product is off by at most
# (2 2^-16 + 2^-32) |a b| (2 parts: ~3.05e-5) or ~2^-23 |a b| (3 parts), plus
# the FP32 accumulation of 64-row tiles.
BF16_TOL = {2: 4e-5, 3: TARGET}
BF16_SHAPES = [(4096, 32, 32), (100003, 32, 32), (3, 32, 32), (0, 8, 8), (20000, 32, 4), (1 << 20, 16, 16),
               (70001, 8, 24), (129, 12, 28), (1, 4, 4), (63, 4, 8), (64, 8, 8), (65, 32, 32), (257, 32, 8)]


@pytest.mark.parametrize("parts", [2, 3])
@pytest.mark.parametrize("n,m,k", BF16_SHAPES)
def test_split_bf16_parity(gpu, oracle_mod, parts, n, m, k):
    from tsm_benchmark_b200 import tsmttsm_split, workspace_status
    A = scaled_normal(n, m, 7 * n + m)
    B = scaled_normal(n, k, 7 * n + k + 1)
    C = tsmttsm_split(torch.from_numpy(A).to(gpu), torch.from_numpy(B).to(gpu), kind=f"bf16x{parts}")
    torch.cuda.synchronize()
    assert workspace_status(gpu) == 0
    got = C.cpu().numpy()
    ref = oracle_mod.naive(A, B)
    if n == 0:
        assert np.all(got == 0)
        return
    nw, pe = errors(ref, got, A, B)
    assert nw <= BF16_TOL[parts] and pe <= BF16_TOL[parts], (nw, pe)


def test_split_bf16_deterministic_accumulate_and_limits(gpu):
    from tsm_benchmark_b200 import tsmttsm_split
    A = torch.from_numpy(scaled_normal(50000, 32, 3)).to(gpu)
    B = torch.from_numpy(scaled_normal(50000, 32, 4)).to(gpu)
    for kind in ("bf16x2", "bf16x3"):
        first = tsmttsm_split(A, B, kind=kind).clone()
        for _ in range(3):
            assert torch.equal(tsmttsm_split(A, B, kind=kind), first)
        C = first.clone()
        tsmttsm_split(A, B, C, accumulate=True, kind=kind)
        assert torch.allclose(C, 2 * first, rtol=1e-15, atol=0)
    # widths that are not multiples of 4 are not taken (the TF32 kind takes them)
    from tsm_benchmark_b200._capi import TsmError
    A5 = torch.zeros((100, 5), dtype=torch.float32, device=gpu)
    with pytest.raises(TsmError):
        tsmttsm_split(A5, A5, kind="bf16x3")
