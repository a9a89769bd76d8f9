"""The oracle (CPU, no GPU): pinned against the reference's own outputs.

The reference has no golden vectors; tests/golden/ holds outputs of its own
code run here (tests/golden/make_golden.py).  Where oracle/_ref is built (this
container) the live reference is compared as well.
"""
import ctypes
import os

import numpy as np
import pytest

from tests.conftest import GOLDEN


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def test_naive_bit_exact_against_reference_compute_naive(oracle_mod):
    from tests.golden.make_golden import SQUARE_CASES
    g = load("ref_square_cases.npz")
    for n, M, seed in SQUARE_CASES:
        A, B = oracle_mod.operands(n, M, M, seed)
        C = oracle_mod.naive(A, B)
        ref = g[f"n{n}_M{M}_s{seed}"]
        assert np.array_equal(C, ref), (n, M, seed)


def test_main_cc_generator_restated_bit_exact(oracle_mod):
    g = load("ref_config0.npz")
    A, B = oracle_mod.main_cc_inputs(1 << 20, 8, 123)
    assert np.array_equal(A[:4], g["A_head"]) and np.array_equal(B[:4], g["B_head"])
    assert np.array_equal(A[-4:], g["A_tail"]) and np.array_equal(B[-4:], g["B_tail"])
    assert A.min() >= -1.0 and A.max() < 1.0


def test_config0_oracle_equals_reference(oracle_mod):
    """n = 2^20, M = 8 with main.cc's inputs: the restated oracle reproduces
    compute_naive bit for bit, and the reference's own tsmttsm4/6/9 passed
    is_correct against it when the fixture was made."""
    g = load("ref_config0.npz")
    A, B = oracle_mod.main_cc_inputs(1 << 20, 8, 123)
    C = oracle_mod.naive(A, B)
    assert np.array_equal(C, g["C_naive"])
    for v in (4, 6, 9):
        assert int(g[f"is_correct_v{v}"]) == 1
        assert oracle_mod.check(g["C_naive"], g[f"C_v{v}"]) == -1


def test_every_reference_kernel_matches_oracle(oracle_mod):
    g = load("ref_variants.npz")
    A, B = oracle_mod.operands(4099, 8, 8, 7)
    C = oracle_mod.naive(A, B)
    assert np.array_equal(C, g["C_naive"])
    names = [k for k in g.files if k != "C_naive"]
    assert len(names) == 18
    for name in names:
        assert oracle_mod.check(C, g[name], 1e-6, 1e-10) == -1, name
        nw = oracle_mod.normwise(A, B, C, g[name])
        assert nw["err"] <= nw["bound"], name


def test_live_reference(oracle_mod):
    """Against the reference compiled in place (skipped where it is not)."""
    R = oracle_mod.ref()
    if R is None:
        pytest.skip("oracle/_ref not built (reference sources absent)")
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    # generator
    A = np.empty(5000)
    B = np.empty(5000)
    R.ref_fill_main_cc_f64(p(A), p(B), 5000, 77)
    A2, B2 = oracle_mod.main_cc_inputs(5000, 1, 77)
    assert np.array_equal(A, A2.ravel()) and np.array_equal(B, B2.ravel())
    # compute_naive on a few more shapes
    for n, M, seed in [(123, 3, 1), (4096, 5, 2), (777, 12, 3)]:
        A, B = oracle_mod.operands(n, M, M, seed)
        C = np.zeros(M * M)
        R.ref_compute_naive_f64(n, M, p(A), p(B), p(C))
        assert np.array_equal(oracle_mod.naive(A, B).ravel(), C)
    # one nd_range variant with barriers (fiber work-groups) at main.cc's shape
    A, B = oracle_mod.operands(20000, 16, 16, 5)
    C = np.zeros(256)
    assert R.ref_tsmttsm_f64(9, 16, 32768, 4, 20000, p(A), p(B), p(C), None) == 0
    assert oracle_mod.check(oracle_mod.naive(A, B), C.reshape(16, 16)) == -1


def test_v4_port_matches_oracle(oracle_mod):
    for M, tile in [(4, 2), (8, 4), (16, 4), (1, 1)]:
        A, B = oracle_mod.operands(30001, M, M, M)
        C = oracle_mod.v4_port(A, B, 4096, tile)
        assert oracle_mod.check(oracle_mod.naive(A, B), C) == -1


def test_known_answers(oracle_mod):
    # all ones: every entry equals n exactly
    n = 12345
    C = oracle_mod.naive(np.ones((n, 3)), np.ones((n, 5)))
    assert np.all(C == n)
    # stacked identities: A = B = [I; I; ...] -> C = reps * I
    reps, w = 7, 6
    Id = np.tile(np.eye(w), (reps, 1))
    assert np.array_equal(oracle_mod.naive(Id, Id), reps * np.eye(w))
    # rank one with small integers: exact
    rng = np.random.default_rng(0)
    u = rng.integers(-8, 8, size=(999, 1)).astype(np.float64)
    a = rng.integers(-8, 8, size=(1, 4)).astype(np.float64)
    b = rng.integers(-8, 8, size=(1, 9)).astype(np.float64)
    C = oracle_mod.naive(u @ a, u @ b)
    assert np.array_equal(C, (u.T @ u)[0, 0] * (a.T @ b))


def test_dot2_is_more_accurate(oracle_mod):
    """On cancelling data the compensated oracle sits closer to the exact
    value (computed in integers) than the plain FP64 sum."""
    rng = np.random.default_rng(1)
    n = 200000
    ints = rng.integers(-2**20, 2**20, size=(n, 2)).astype(np.float64)
    A = ints[:, :1] * 2.0**-10 + 1e6
    B = ints[:, 1:] * 2.0**-10 - 1e6
    exact = sum(int(a * 2**10) * int(b * 2**10) for a, b in zip(A[:, 0], B[:, 0])) / 2**20
    e_naive = abs(oracle_mod.naive(A, B)[0, 0] - exact)
    e_dot2 = abs(oracle_mod.dot2(A, B)[0, 0] - exact)
    assert e_dot2 <= e_naive
    assert e_dot2 <= 1e-16 * abs(exact) * 4


def test_check_rule_catches_planted_error(oracle_mod):
    """A mistake planted in an oracle output (on the CPU) is reported at its
    index; the reference's tolerances accept a last-bit difference."""
    A, B = oracle_mod.operands(1000, 4, 6, 3)
    C = oracle_mod.naive(A, B)
    bad = C.copy()
    bad[2, 5] *= 1 + 1e-5
    assert oracle_mod.check(C, bad) == 2 * 6 + 5
    bad = C.copy()
    bad[0, 0] = np.nan
    assert oracle_mod.check(C, bad) == 0
    close = np.nextafter(C, np.inf)
    assert oracle_mod.check(C, close) == -1


def test_normwise_bound(oracle_mod):
    A, B = oracle_mod.operands(50000, 8, 8, 9)
    C = oracle_mod.naive(A, B)
    D = oracle_mod.dot2(A, B)
    nw = oracle_mod.normwise(A, B, D, C)
    assert 0 <= nw["err"] <= nw["bound"]
    assert nw["bound"] == pytest.approx(4 * np.sqrt(50000) * 2.0**-53 * np.linalg.norm(A) * np.linalg.norm(B))


def test_uniform_generator_properties(oracle_mod):
    x = oracle_mod.uniform(1 << 16, 123, 0)
    y = oracle_mod.uniform(1 << 16, 123, 1)
    assert x.min() >= -1 and x.max() < 1
    assert abs(x.mean()) < 0.02 and abs(x.var() - 1 / 3) < 0.01
    assert not np.array_equal(x, y)
    # counter based: a prefix is the same whatever the count
    assert np.array_equal(oracle_mod.uniform(100, 123, 0), x[:100])


def test_tsmm_oracle(oracle_mod):
    rng = np.random.default_rng(2)
    X = rng.standard_normal((333, 7))
    W = rng.standard_normal((7, 5))
    assert np.allclose(oracle_mod.tsmm(X, W), X @ W, rtol=1e-13, atol=1e-13)
    assert np.allclose(oracle_mod.tsmm(X, W.T.copy(), transpose_w=True), X @ W, rtol=1e-13, atol=1e-13)


def test_transpose_identity_and_empty(oracle_mod):
    """naive(B, A) is naive(A, B) transposed bit for bit (the same products
    summed over rows in the same order), and zero rows give a zero C."""
    for n, m, k, seed in [(1, 1, 1, 1), (4099, 3, 5, 2), (30001, 8, 64, 3)]:
        A, B = oracle_mod.operands(n, m, k, seed)
        assert np.array_equal(oracle_mod.naive(B, A), oracle_mod.naive(A, B).T)
    Z = oracle_mod.naive(np.zeros((0, 4)), np.zeros((0, 6)))
    assert Z.shape == (4, 6) and not Z.any()


def test_streaming_dot2_is_correctly_rounded_and_chunk_invariant(oracle_mod):
    """The full-size oracle (compensated product over row blocks): against
    exact rational sums it rounds correctly; feeding the rows in chunks, or
    letting it generate the counter-based operands itself, gives the same C;
    the factor-splitting body (hosts without FMA) agrees with the FMA one."""
    from fractions import Fraction
    n, m, k = 2001, 3, 4
    A, B = oracle_mod.operands(n, m, k, 7)
    exact = np.array([[float(sum(Fraction(a) * Fraction(b) for a, b in zip(A[:, i], B[:, j])))
                       for j in range(k)] for i in range(m)])
    d = oracle_mod.Dot2Stream(m, k, with_abs=True)
    d.add(A[:700], B[:700])
    d.add(A[700:], B[700:])
    r = d.result()
    assert np.array_equal(r["C"], exact)
    assert r["rows"] == n
    assert np.allclose(r["absC"], np.abs(A).T @ np.abs(B), rtol=1e-13)
    assert r["normA"] == pytest.approx(np.linalg.norm(A), rel=1e-13)
    assert r["bound"] == pytest.approx(4 * np.sqrt(n) * 2.0**-53 * np.linalg.norm(A) * np.linalg.norm(B), rel=1e-12)
    assert np.array_equal(oracle_mod.dot2_uniform(n, m, k, 7)["C"], exact)
    g = oracle_mod.Dot2Stream(m, k)
    g.add_uniform(7, 0, 1000)
    g.add_uniform(7, 1000, n - 1000)
    assert np.array_equal(g.result()["C"], exact)
    oracle_mod.lib().tsm_oracle_force_split(1)
    try:
        assert np.array_equal(oracle_mod.dot2_uniform(n, m, k, 7)["C"], exact)
    finally:
        oracle_mod.lib().tsm_oracle_force_split(0)
    # FP32 input is widened exactly
    A32, B32 = A.astype(np.float32), B.astype(np.float32)
    f = oracle_mod.Dot2Stream(m, k)
    f.add(A32, B32)
    assert np.array_equal(f.result()["C"], oracle_mod.dot2(A32.astype(np.float64), B32.astype(np.float64)))


def test_streaming_dot2_decides_between_naive_and_blocked_sums(oracle_mod):
    """At 2^20 rows the compensated result is closer to every entry than the
    naive running sum (whose error grows with n), and the naive sum meets the
    normwise bound measured against it."""
    A, B = oracle_mod.operands(1 << 20, 4, 4, 11)
    ref = oracle_mod.dot2_uniform(1 << 20, 4, 4, 11)
    naive = oracle_mod.naive(A, B)
    assert np.linalg.norm(naive - ref["C"]) <= ref["bound"]
    assert np.all(np.abs(ref["C"] - oracle_mod.dot2(A, B)) <= np.spacing(np.abs(ref["C"])))


def test_streaming_dot2_gram_and_column_major_generation(oracle_mod):
    """The streaming oracle's other generated layouts: B is A (same stream),
    and column-major operands (the values a fill of A^T, B^T writes),
    against the compensated product of explicitly built host arrays."""
    n, m, k = 3001, 5, 7
    A, _ = oracle_mod.operands(n, m, k, 9)
    assert np.array_equal(oracle_mod.dot2_uniform(n, m, m, 9, gram=True)["C"], oracle_mod.dot2(A, A))
    At = oracle_mod.uniform(m * n, 9, 0).reshape(m, n)
    Bt = oracle_mod.uniform(k * n, 9, 1).reshape(k, n)
    ref = oracle_mod.dot2(np.ascontiguousarray(At.T), np.ascontiguousarray(Bt.T))
    assert np.array_equal(oracle_mod.dot2_uniform(n, m, k, 9, col_major=True)["C"], ref)
    d = oracle_mod.Dot2Stream(m, k)
    d.add_uniform(9, 0, 1000, col_major_n=n)
    d.add_uniform(9, 1000, n - 1000, col_major_n=n)
    assert np.array_equal(d.result()["C"], ref)
