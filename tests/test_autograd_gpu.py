"""The differentiation form: TSMM kernels, the fused backward and the
torch.autograd.Function, against the oracle, finite differences
(torch.autograd.gradcheck) and torch's own gradient of A.T @ B."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def to_dev(x, dev):
    return torch.from_numpy(np.ascontiguousarray(x)).to(dev)


def tsmm_bound(X, W, dtype):
    """||Y - Y_ref||_F bound for one dot of length p per output."""
    u = 2.0**-53 if dtype == np.float64 else 2.0**-24
    p = X.shape[1]
    return (p + 2) * u * np.linalg.norm(X.astype(np.float64)) * np.linalg.norm(W.astype(np.float64)) + 1e-300


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("p,q", [(1, 1), (4, 4), (16, 16), (3, 7), (32, 5), (8, 64), (64, 64), (64, 1), (13, 33)])
def test_tsmm_parity(gpu, oracle_mod, dtype, p, q):
    from tsm_benchmark_b200 import tsmm
    rng = np.random.default_rng(p * 100 + q)
    for n in (0, 1, 3, 4099, 70001):
        X = oracle_mod.uniform(n * p, 5 + n, 0).reshape(n, p).astype(dtype)
        W = rng.standard_normal((p, q)).astype(dtype)
        ref = oracle_mod.tsmm(X.astype(np.float64), W.astype(np.float64))
        Y = tsmm(to_dev(X, gpu), to_dev(W, gpu)).cpu().numpy().astype(np.float64)
        assert np.linalg.norm(Y - ref) <= tsmm_bound(X, W, dtype), (n, p, q)
        # W given transposed (the dA = B dC^T case), and accumulation into Y
        Wt = to_dev(W.T.copy(), gpu)
        Y0 = rng.standard_normal((n, q)).astype(dtype)
        Yd = to_dev(Y0, gpu)
        tsmm(to_dev(X, gpu), Wt, Yd, transpose_w=True, accumulate=True)
        got = Yd.cpu().numpy().astype(np.float64) - Y0.astype(np.float64)
        assert np.linalg.norm(got - ref) <= 2 * tsmm_bound(X, W, dtype) + 4 * np.finfo(dtype).eps * np.linalg.norm(Y0)


def test_tsmm_strided_operands(gpu, oracle_mod):
    """A column slice of a wider X takes the direct-load kernel."""
    from tsm_benchmark_b200 import tsmm
    Xw = oracle_mod.uniform(5003 * 24, 9, 0).reshape(5003, 24)
    W = np.random.default_rng(1).standard_normal((16, 8))
    Y = tsmm(to_dev(Xw, gpu)[:, 4:20], to_dev(W, gpu)).cpu().numpy()
    ref = oracle_mod.tsmm(np.ascontiguousarray(Xw[:, 4:20]), W)
    assert np.linalg.norm(Y - ref) <= tsmm_bound(Xw[:, 4:20], W, np.float64)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("m,k", [(16, 16), (4, 4), (8, 32), (5, 3)])
def test_fused_backward(gpu, oracle_mod, dtype, m, k):
    from tsm_benchmark_b200 import tsmttsm_backward
    n = 65537
    A = oracle_mod.uniform(n * m, 3, 0).reshape(n, m).astype(dtype)
    B = oracle_mod.uniform(n * k, 3, 1).reshape(n, k).astype(dtype)
    dC = np.random.default_rng(2).standard_normal((m, k)).astype(dtype)
    dA, dB = tsmttsm_backward(to_dev(A, gpu), to_dev(B, gpu), to_dev(dC, gpu))
    refA = oracle_mod.tsmm(B.astype(np.float64), dC.astype(np.float64).T.copy())
    refB = oracle_mod.tsmm(A.astype(np.float64), dC.astype(np.float64))
    assert np.linalg.norm(dA.cpu().numpy().astype(np.float64) - refA) <= tsmm_bound(B, dC.T, dtype)
    assert np.linalg.norm(dB.cpu().numpy().astype(np.float64) - refB) <= tsmm_bound(A, dC, dtype)
    # one of the two only
    dA2, none = tsmttsm_backward(to_dev(A, gpu), to_dev(B, gpu), to_dev(dC, gpu), need_dB=False)
    assert none is None and torch.equal(dA2, dA)


def test_gradcheck_fp64(gpu):
    """The gradient check of the differentiation form: n = 2^12, m = k = 4, FP64, finite differences."""
    from tsm_benchmark_b200 import gram_tn
    g = torch.Generator(device=gpu).manual_seed(0)
    A = torch.rand((1 << 12, 4), dtype=torch.float64, device=gpu, generator=g).requires_grad_()
    B = torch.rand((1 << 12, 4), dtype=torch.float64, device=gpu, generator=g).requires_grad_()
    assert torch.autograd.gradcheck(gram_tn, (A, B), eps=1e-4, atol=1e-6, rtol=1e-5)


@pytest.mark.parametrize("dtype,rtol", [(torch.float64, 1e-12), (torch.float32, 2e-5)])
def test_matches_torch_gradient(gpu, dtype, rtol):
    """loss = sum(W * C), W an m x k normal matrix (the differentiation form's loss), n = 2^22,
    m = k = 16: forward and both gradients against torch's A.T @ B."""
    from tsm_benchmark_b200 import gram_tn
    g = torch.Generator(device=gpu).manual_seed(1)
    n, m, k = 1 << 22, 16, 16
    A = (torch.rand((n, m), device=gpu, generator=g, dtype=torch.float64) * 2 - 1).to(dtype).requires_grad_()
    B = (torch.rand((n, k), device=gpu, generator=g, dtype=torch.float64) * 2 - 1).to(dtype).requires_grad_()
    Wl = torch.randn((m, k), device=gpu, generator=g, dtype=torch.float64).to(dtype)
    C = gram_tn(A, B)
    (C * Wl).sum().backward()
    gA, gB = A.grad.clone(), B.grad.clone()
    A64 = A.detach().double().requires_grad_()
    B64 = B.detach().double().requires_grad_()
    C64 = A64.T @ B64
    (C64 * Wl.double()).sum().backward()
    scale = float(C64.detach().abs().max())
    assert float((C.double() - C64).abs().max()) <= rtol * scale * (100 if dtype == torch.float32 else 1) + 1e-9
    assert torch.allclose(gA.double(), A64.grad, rtol=rtol, atol=rtol * float(A64.grad.abs().max()))
    assert torch.allclose(gB.double(), B64.grad, rtol=rtol, atol=rtol * float(B64.grad.abs().max()))
    del A, B, A64, B64
    torch.cuda.empty_cache()


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_tsmm_accumulate_staged_and_unstaged_agree(gpu, dtype):
    """Y += X W through the staged-Y kernel (dense Y: the old rows ride the
    TMA ring) and through the unstaged one (Y a column slice of a wider
    buffer: old pairs read from global memory) add the same product to the
    same old values in the same order: bit-identical results."""
    from tsm_benchmark_b200 import tsmm
    for p, q in ((16, 16), (8, 64), (64, 4), (4, 32), (32, 32)):
        for n in (5, 4099, 70001, (1 << 20) + 3):
            g = torch.Generator().manual_seed(n + 7 * p + q)
            X = torch.randn(n, p, generator=g, dtype=torch.float64).to(dtype).to(gpu)
            W = torch.randn(p, q, generator=g, dtype=torch.float64).to(dtype).to(gpu)
            Y0 = torch.randn(n, q, generator=g, dtype=torch.float64).to(dtype).to(gpu)
            dense = Y0.clone()
            wide = torch.zeros(n, q + 4, dtype=dtype, device=gpu)
            wide[:, 2:2 + q] = Y0
            tsmm(X, W, dense, accumulate=True)
            tsmm(X, W, wide[:, 2:2 + q], accumulate=True)
            assert torch.equal(dense, wide[:, 2:2 + q]), (p, q, n)
            assert not torch.equal(dense, Y0), (p, q, n)
