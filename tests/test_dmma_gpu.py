"""The FP64 tensor-core (DMMA) kernels of the plain path, C = A^T B for
exact widths m, k in {16, 32, 48, 64}: every variant against the oracle on
ragged row counts (partial chunks, rows the tensor maps zero-fill), strided
operands, repeatability and the variant choice."""
import numpy as np
import pytest
import torch

from tests.test_plain_gpu import assert_parity, to_dev

pytestmark = pytest.mark.gpu


def dmma_variants():
    """The two-operand DMMA variants (the Gram ones are in test_gram_gpu.py)."""
    from tsm_benchmark_b200 import variants
    return [v for v in variants() if v["kind"] == "dmma" and not v["gram"]]


def test_sixteen_dmma_variants_exist(gpu):
    shapes = {(v["wa"], v["wb"]) for v in dmma_variants()}
    assert shapes == {(a, b) for a in (16, 32, 48, 64) for b in (16, 32, 48, 64)}


@pytest.mark.parametrize("m", [16, 32, 48, 64])
@pytest.mark.parametrize("k", [16, 32, 48, 64])
def test_dmma_variant_parity(gpu, oracle_mod, m, k):
    from tsm_benchmark_b200 import tsmttsm
    vs = [v for v in dmma_variants() if (v["wa"], v["wb"]) == (m, k)]  # every ring shape of the pair
    assert vs
    for v in vs:
        for n in (0, 1, 5, v["rows"] - 1, v["rows"] + 3, 3 * v["rows"] + 11, 40013):
            A, B = oracle_mod.operands(n, m, k, 100 + n % 97 + m + k)
            C = tsmttsm(to_dev(A, gpu), to_dev(B, gpu), variant=v["index"])
            assert_parity(oracle_mod, A, B, C, what=f"{v['name']} n={n}")


def test_dmma_strided_operands(gpu, oracle_mod):
    """Column slices with 16-byte row pitches and 16-byte aligned starts are
    read through the tensor maps directly (no copy, no direct-load kernel)."""
    from tsm_benchmark_b200 import default_variant, tsmttsm, variants
    names = [v["name"] for v in variants()]
    n = 20011
    A_wide, B_wide = oracle_mod.operands(n, 80, 66, 5)
    dA = to_dev(A_wide, gpu)[:, 16:48]   # m = 32, lda = 80, start 128 bytes in
    dB = to_dev(B_wide, gpu)[:, 2:18]    # k = 16, ldb = 66, start 16 bytes in
    idx = default_variant(dA, dB)
    assert names[idx].startswith("dmma_32x16")
    C = tsmttsm(dA, dB)
    assert_parity(oracle_mod, np.ascontiguousarray(A_wide[:, 16:48]), np.ascontiguousarray(B_wide[:, 2:18]), C,
                  what="dmma strided")
    # an odd pitch (8-byte aligned rows) is not a tensor-map layout
    A_odd, _ = oracle_mod.operands(n, 33, 16, 6)
    dA_odd = to_dev(A_odd, gpu)[:, 0:32]
    assert not names[default_variant(dA_odd, dB)].startswith("dmma")


def test_dmma_repeatable(gpu, oracle_mod):
    from tsm_benchmark_b200 import tsmttsm
    vs = [v for v in dmma_variants() if (v["wa"], v["wb"]) == (64, 64)]  # every ring shape
    assert vs
    A, B = oracle_mod.operands(300007, 64, 64, 9)
    dA, dB = to_dev(A, gpu), to_dev(B, gpu)
    for v in vs:
        C1 = tsmttsm(dA, dB, variant=v["index"])
        C2 = tsmttsm(dA, dB, variant=v["index"])
        assert torch.equal(C1, C2), v["name"]
        assert_parity(oracle_mod, A, B, C1, what=f"{v['name']} large")


def test_dmma_accumulate(gpu, oracle_mod):
    from tsm_benchmark_b200 import tsmttsm
    (v,) = [v for v in dmma_variants() if (v["wa"], v["wb"]) == (32, 48)]
    A, B = oracle_mod.operands(9001, 32, 48, 12)
    C0 = np.random.default_rng(0).standard_normal((32, 48))
    C = to_dev(C0.copy(), gpu)
    tsmttsm(to_dev(A, gpu), to_dev(B, gpu), C, accumulate=True, variant=v["index"])
    ref = oracle_mod.naive(A, B) + C0
    scale = np.abs(A).T @ np.abs(B) + np.abs(C0)
    assert np.max(np.abs(C.cpu().numpy() - ref) / scale) < 1e-13
