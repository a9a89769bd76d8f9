"""The Gram product C = A^T A (B is A): the Gram variants stream A once and
write C exactly symmetric; tsm_gram_f64 and tsmttsm(A, A) both take them.
Checked against the oracle's naive product on the same values."""
import numpy as np
import pytest
import torch

from tests.test_plain_gpu import assert_parity, to_dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m", [1, 2, 4, 8, 16, 32, 48, 64, 5, 24])
def test_gram_parity_and_symmetry(gpu, oracle_mod, m):
    from tsm_benchmark_b200 import gram
    for n in (0, 1, 7, 4099, 100003):
        A, _ = oracle_mod.operands(n, m, m, 40 + m + n % 13)
        C = gram(to_dev(A, gpu))
        assert_parity(oracle_mod, A, A, C, what=f"gram m={m} n={n}")
        assert torch.equal(C, C.T), (m, n)


def test_every_gram_variant(gpu, oracle_mod):
    """Every compiled Gram variant (each ring shape, chunks of one or several
    tensor boxes) on row counts around its chunk and box edges."""
    from tsm_benchmark_b200 import tsmttsm, variants
    for v in (v for v in variants() if v["gram"] and v["dtype"] == "f64"):
        m = v["wa"]
        for n in (1, 5, v["rows"] // 2 + 1, v["rows"] - 1, v["rows"] + 3, 3 * v["rows"] + 11, 40013):
            A, _ = oracle_mod.operands(n, m, m, 70 + m + n % 31)
            dA = to_dev(A, gpu)
            C = tsmttsm(dA, dA, variant=v["index"])
            assert_parity(oracle_mod, A, A, C, what=f"{v['name']} n={n}")
            assert torch.equal(C, C.T), (v["name"], n)


def test_gram_variant_is_chosen_for_same_operand(gpu, oracle_mod):
    from tsm_benchmark_b200 import default_variant, tsmttsm, variants
    vs = variants()
    A, _ = oracle_mod.operands(30001, 32, 32, 9)
    dA = to_dev(A, gpu)
    assert vs[default_variant(dA, dA)]["gram"]
    B = dA.clone()
    assert not vs[default_variant(dA, B)]["gram"]  # same values, different operand
    C1 = tsmttsm(dA, dA)
    C2 = tsmttsm(dA, B)
    assert_parity(oracle_mod, A, A, C1, what="tsmttsm(A, A)")
    assert_parity(oracle_mod, A, A, C2, what="tsmttsm(A, copy of A)")
    # the two paths sum in different orders: both within the normwise bound
    bound = 4 * A.shape[0] ** 0.5 * 2.0**-53 * np.linalg.norm(A) ** 2
    assert float(torch.linalg.norm(C1 - C2)) <= 2 * bound
    for w in (1, 2, 4, 8, 16, 32, 48, 64):
        assert any(v["gram"] and v["wa"] == w and v["wb"] == w for v in vs), w


def test_gram_strided_and_accumulate(gpu, oracle_mod):
    """A column slice (16-byte pitch: the tensor-core Gram variant reads it in
    place) and C += A^T A."""
    from tsm_benchmark_b200 import gram
    A_wide, _ = oracle_mod.operands(20011, 80, 8, 3)
    dA = to_dev(A_wide, gpu)[:, 16:48]
    A = np.ascontiguousarray(A_wide[:, 16:48])
    C = gram(dA)
    assert_parity(oracle_mod, A, A, C, what="gram strided")
    C0 = np.random.default_rng(1).standard_normal((32, 32))
    Cd = to_dev(C0.copy(), gpu)
    gram(dA, Cd, accumulate=True)
    ref = oracle_mod.naive(A, A) + C0
    scale = np.abs(A).T @ np.abs(A) + np.abs(C0)
    assert np.max(np.abs(Cd.cpu().numpy() - ref) / scale) < 1e-13


def test_gram_repeatable_full_size(gpu):
    """n = 2^24, m = 16: repeatable to the bit, symmetric, and within the
    normwise bound of the two-operand path on the same values."""
    from tsm_benchmark_b200 import fill_uniform, gram, tsmttsm
    n, m = 1 << 24, 16
    A = torch.empty((n, m), dtype=torch.float64, device=gpu)
    fill_uniform(A, 5, 0)
    C1 = gram(A)
    C2 = gram(A)
    assert torch.equal(C1, C2) and torch.equal(C1, C1.T)
    ref = tsmttsm(A, A.clone())
    bound = 4 * n**0.5 * 2.0**-53 * float(torch.linalg.norm(A)) ** 2
    assert float(torch.linalg.norm(C1 - ref)) <= 2 * bound
    del A
    torch.cuda.empty_cache()
