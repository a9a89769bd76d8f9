"""Block orthogonalisation B <- B - A (A^T B): the product and the TSMM
update in one call, against the oracle; with orthonormal A the result is
orthogonal to A's columns."""
import numpy as np
import pytest

from tests.test_plain_gpu import to_dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m,k", [(4, 4), (16, 16), (8, 32), (32, 8), (5, 7), (64, 64)])
def test_block_orth_matches_oracle(gpu, oracle_mod, m, k):
    from tsm_benchmark_b200 import block_orthogonalize
    for n in (0, 3, 20001):
        A, B = oracle_mod.operands(n, m, k, 60 + m + k + n % 11)
        dB = to_dev(B, gpu)
        C = block_orthogonalize(to_dev(A, gpu), dB).cpu().numpy()
        C_ref = oracle_mod.naive(A, B)
        nw = oracle_mod.normwise(A, B, C_ref, C)
        assert nw["err"] <= nw["bound"], (m, k, n, nw)
        # the update against B - A C with the returned C (its own error is
        # the normwise bound above): one dot of length m and a subtraction
        B_ref = B - oracle_mod.tsmm(A, C)
        scale = np.abs(B) + oracle_mod.tsmm(np.abs(A), np.abs(C))
        got = dB.cpu().numpy()
        assert np.all(np.abs(got - B_ref) <= (m + 4) * 2.0**-52 * scale + 1e-300), (m, k, n)


def test_block_orth_removes_the_span(gpu):
    from tsm_benchmark_b200 import block_orthogonalize, tsmttsm
    rng = np.random.default_rng(7)
    n, m, k = 200003, 16, 8
    Q, _ = np.linalg.qr(rng.standard_normal((n, m)))
    B = rng.standard_normal((n, k))
    dQ, dB = to_dev(Q, gpu), to_dev(B, gpu)
    block_orthogonalize(dQ, dB)
    R = tsmttsm(dQ, dB).cpu().numpy()
    assert np.max(np.abs(R)) <= 1e-12 * np.linalg.norm(B)
