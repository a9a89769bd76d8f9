"""Parity at the benchmark configurations' full sizes, against the oracle.

Every shape of the plain FP64 width sweep at its benchmark row count (n =
2^26; 2^23 for 64 x 64), the split-precision configuration (n = 2^25, m = k =
32, FP32 storage), the batched configuration (512 problems of log-uniform n
in [10^3, 10^6]) and the differentiation configuration (n = 2^22, m = k = 16)
are checked against the oracle, not against another GPU library:

* plain and batched: the operands are the library's counter-based uniform
  values (``fill_uniform`` on the GPU); the oracle regenerates the same bits
  on the host, block by block, and forms a compensated (Dot2) product, so no
  operand is held whole on the host.  Acceptance is the normwise bound
  ||C - C_oracle||_F <= 4 sqrt(n) 2^-53 ||A||_F ||B||_F -- exactly, not a
  multiple of it -- and the reference's element rule (main.cc:29-41).
* split precision: the FP32 operands are copied to the host in row chunks
  and fed to the same compensated product; acceptance is the stated error of
  each kind, normwise and per entry relative to sum_r |a_ri| |b_rj|.
* differentiation: dA = B dC^T and dB = A dC against the oracle's TSMM;
* the Gram product and column-major operands at their benchmark sizes, the
  oracle regenerating A alone, or the values written into A^T and B^T.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

REL_TOL, ABS_TOL = 1e-6, 1e-10

# The plain FP64 sweep: (n, m, k).
SWEEP = [(1 << 26, 1, 1), (1 << 26, 2, 2), (1 << 26, 4, 4), (1 << 26, 8, 8), (1 << 26, 16, 16),
         (1 << 26, 32, 32), (1 << 23, 64, 64), (1 << 26, 4, 32), (1 << 26, 32, 4), (1 << 26, 1, 64)]


def _free():
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


@pytest.mark.parametrize("n,m,k", SWEEP, ids=[f"2^{n.bit_length() - 1}x{m}x{k}" for n, m, k in SWEEP])
def test_sweep_shape_against_oracle(gpu, oracle_mod, n, m, k):
    from tsm_benchmark_b200 import default_variant, fill_uniform, tsmttsm, variants, workspace_status
    seed = 123 + m * 65 + k
    A = torch.empty((n, m), dtype=torch.float64, device=gpu)
    B = torch.empty((n, k), dtype=torch.float64, device=gpu)
    fill_uniform(A, seed, 0)
    fill_uniform(B, seed, 1)
    got = tsmttsm(A, B).cpu().numpy()
    name = variants()[default_variant(A, B)]["name"]
    assert workspace_status(gpu) == 0
    del A, B
    _free()
    ref = oracle_mod.dot2_uniform(n, m, k, seed)
    err = float(np.linalg.norm(got - ref["C"]))
    assert err <= ref["bound"], f"{name}: normwise {err:.3e} > bound {ref['bound']:.3e}"
    bad = oracle_mod.check(ref["C"], got, REL_TOL, ABS_TOL)
    assert bad == -1, f"{name}: entry {bad}: oracle {ref['C'].ravel()[bad]} got {got.ravel()[bad]}"


def test_split_config_against_oracle(gpu, oracle_mod):
    """n = 2^25, m = k = 32, standard normal entries with column j scaled by
    10^u_j, u_j ~ U[-3, 3] (FP32 storage): TF32 hi/lo and BF16 hi/mid/lo within
    1e-6 of the oracle, BF16 hi/lo within its stated 4e-5."""
    from tsm_benchmark_b200 import tsmttsm_split
    n, w = 1 << 25, 32
    g = torch.Generator(device=gpu).manual_seed(3)
    sa = 10.0 ** (torch.rand(w, device=gpu, generator=g) * 6 - 3)
    sb = 10.0 ** (torch.rand(w, device=gpu, generator=g) * 6 - 3)
    A = (torch.randn((n, w), device=gpu, generator=g) * sa).float()
    B = (torch.randn((n, w), device=gpu, generator=g) * sb).float()
    got = {kind: tsmttsm_split(A, B, kind=kind).cpu().numpy() for kind in ("tf32", "bf16x2", "bf16x3")}
    d = oracle_mod.Dot2Stream(w, w, with_abs=True)
    step = 1 << 22
    for r in range(0, n, step):
        d.add(A[r:r + step].cpu().numpy(), B[r:r + step].cpu().numpy())
    del A, B
    _free()
    ref = d.result()
    for kind, tol in (("tf32", 1e-6), ("bf16x3", 1e-6), ("bf16x2", 4e-5)):
        nw = float(np.linalg.norm(got[kind] - ref["C"]) / np.linalg.norm(ref["C"]))
        pe = float(np.max(np.abs(got[kind] - ref["C"]) / ref["absC"]))
        assert nw <= tol and pe <= tol, (kind, nw, pe)


def test_batched_config_against_oracle(gpu, oracle_mod):
    """512 problems, n log-uniform in [10^3, 10^6], widths in {4, 8, 16, 32}:
    one launch; every C_p within its own normwise bound of the oracle."""
    from tsm_benchmark_b200 import BatchedTSMTTSM, fill_uniform
    rng = np.random.default_rng(5)
    ns = np.exp(rng.uniform(np.log(1e3), np.log(1e6), size=512)).astype(np.int64)
    ms = rng.choice((4, 8, 16, 32), size=512)
    ks = rng.choice((4, 8, 16, 32), size=512)
    As, Bs = [], []
    for i, (n, m, k) in enumerate(zip(ns, ms, ks)):
        a = torch.empty((int(n), int(m)), dtype=torch.float64, device=gpu)
        b = torch.empty((int(n), int(k)), dtype=torch.float64, device=gpu)
        fill_uniform(a, 5000 + i, 0)
        fill_uniform(b, 5000 + i, 1)
        As.append(a)
        Bs.append(b)
    bt = BatchedTSMTTSM(As, Bs)
    got = [c.cpu().numpy() for c in bt.run()]
    del As, Bs, bt
    _free()
    for i, (n, m, k) in enumerate(zip(ns, ms, ks)):
        ref = oracle_mod.dot2_uniform(int(n), int(m), int(k), 5000 + i)
        err = float(np.linalg.norm(got[i] - ref["C"]))
        assert err <= ref["bound"], (i, int(n), int(m), int(k), err, ref["bound"])
        assert oracle_mod.check(ref["C"], got[i], REL_TOL, ABS_TOL) == -1, i


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_autograd_config_backward_against_oracle(gpu, oracle_mod, dtype):
    """n = 2^22, m = k = 16: the fused backward's dA = B dC^T and dB = A dC
    against the oracle's TSMM of the same values (FP32 storage: the oracle
    works on the FP32 values widened to FP64; the kernel rounds each output
    once)."""
    from tsm_benchmark_b200 import tsmttsm_backward
    n, w = 1 << 22, 16
    A, B = oracle_mod.operands(n, w, w, seed=17)
    dC = np.random.default_rng(18).standard_normal((w, w))
    if dtype == torch.float32:
        A, B, dC = A.astype(np.float32), B.astype(np.float32), dC.astype(np.float32)
    dA, dB = tsmttsm_backward(torch.from_numpy(A).to(gpu), torch.from_numpy(B).to(gpu), torch.from_numpy(dC).to(gpu))
    A64, B64, dC64 = A.astype(np.float64), B.astype(np.float64), dC.astype(np.float64)
    ref_dA = oracle_mod.tsmm(B64, dC64.T.copy())
    ref_dB = oracle_mod.tsmm(A64, dC64)
    # each output is one 16-term FP64 dot product (error <= gamma_16 of the
    # scale, on both sides of the comparison), rounded once more to FP32
    tol = 2.0**-24 * 1.01 if dtype == torch.float32 else 2 * 17 * 2.0**-53
    for got, ref, X in ((dA, ref_dA, B64), (dB, ref_dB, A64)):
        g = got.cpu().numpy().astype(np.float64)
        scale = np.abs(X) @ np.abs(dC64 if X is A64 else dC64.T)
        rel = np.max(np.abs(g - ref) / np.maximum(scale, 1e-300))
        assert rel <= tol, (dtype, rel, tol)
    del dA, dB
    _free()


GRAM = [(1 << 26, 8), (1 << 26, 32), (1 << 23, 64)]


@pytest.mark.parametrize("n,m", GRAM, ids=[f"2^{n.bit_length() - 1}x{m}" for n, m in GRAM])
def test_gram_at_benchmark_size_against_oracle(gpu, oracle_mod, n, m):
    """C = A^T A (A streamed once, upper triangle) at the Gram benchmark's
    sizes: the exact normwise bound against the oracle, and C exactly
    symmetric."""
    from tsm_benchmark_b200 import fill_uniform, gram
    seed = 77 + m
    A = torch.empty((n, m), dtype=torch.float64, device=gpu)
    fill_uniform(A, seed, 0)
    got = gram(A).cpu().numpy()
    del A
    _free()
    assert np.array_equal(got, got.T)
    ref = oracle_mod.dot2_uniform(n, m, m, seed, gram=True)
    err = float(np.linalg.norm(got - ref["C"]))
    assert err <= ref["bound"], (n, m, err, ref["bound"])
    assert oracle_mod.check(ref["C"], got, REL_TOL, ABS_TOL) == -1


COLUMN_MAJOR = [(1 << 26, 8, 8), (1 << 25, 4, 32), (1 << 25, 32, 32), (1 << 23, 64, 64)]


@pytest.mark.parametrize("n,m,k", COLUMN_MAJOR, ids=[f"2^{n.bit_length() - 1}x{m}x{k}" for n, m, k in COLUMN_MAJOR])
def test_column_major_at_benchmark_size_against_oracle(gpu, oracle_mod, n, m, k):
    """Column-major operands (A^T, B^T stored row-major, read in place by
    the tensor-map kernels) at the column-major benchmark's sizes, against
    the oracle at the exact bound."""
    from tsm_benchmark_b200 import fill_uniform, tsmttsm
    seed = 91 + m + k
    At = torch.empty((m, n), dtype=torch.float64, device=gpu)
    Bt = torch.empty((k, n), dtype=torch.float64, device=gpu)
    fill_uniform(At, seed, 0)
    fill_uniform(Bt, seed, 1)
    got = tsmttsm(At.t(), Bt.t()).cpu().numpy()
    del At, Bt
    _free()
    ref = oracle_mod.dot2_uniform(n, m, k, seed, col_major=True)
    err = float(np.linalg.norm(got - ref["C"]))
    assert err <= ref["bound"], (n, m, k, err, ref["bound"])
    assert oracle_mod.check(ref["C"], got, REL_TOL, ABS_TOL) == -1
