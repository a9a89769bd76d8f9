"""Parity of the plain FP64 path (C ABI through ctypes) with the oracle.

Acceptance, per entry: the reference's is_correct rule (main.cc:29-41, rel
1e-6 / abs 1e-10); per matrix: the normwise bound
||C - C_oracle||_F <= 4 sqrt(n) 2^-53 ||A||_F ||B||_F.
"""
import ctypes
import os

import numpy as np
import pytest
import torch

from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu

REL_TOL, ABS_TOL = 1e-6, 1e-10


def to_dev(x, dev):
    return torch.from_numpy(np.ascontiguousarray(x)).to(dev)


def assert_parity(oracle_mod, A, B, C_got, C_ref=None, what=""):
    C_got = C_got.cpu().numpy() if isinstance(C_got, torch.Tensor) else C_got
    if C_ref is None:
        C_ref = oracle_mod.naive(A, B)
    bad = oracle_mod.check(C_ref, C_got, REL_TOL, ABS_TOL)
    assert bad == -1, f"{what}: entry {bad}: ref {C_ref.ravel()[bad]} got {C_got.ravel()[bad]}"
    nw = oracle_mod.normwise(A, B, C_ref, C_got)
    assert nw["err"] <= nw["bound"], f"{what}: normwise {nw}"


SHAPES = [(1, 1), (2, 2), (4, 4), (8, 8), (16, 16), (32, 32), (64, 64), (4, 32), (32, 4), (1, 64),
          (3, 5), (7, 13), (33, 17), (64, 1), (5, 64), (12, 12), (4, 8), (16, 32)]
ROWS = [0, 1, 2, 3, 255, 4099, 65537]


@pytest.mark.parametrize("m,k", SHAPES)
def test_parity_widths_and_ragged_rows(gpu, oracle_mod, m, k):
    from tsm_benchmark_b200 import tsmttsm, workspace_status
    for n in ROWS:
        if m * k >= 1024 and n > 4099:
            continue
        A, B = oracle_mod.operands(n, m, k, seed=1000 + n + 7 * m + k)
        C = tsmttsm(to_dev(A, gpu), to_dev(B, gpu))
        torch.cuda.synchronize()
        assert_parity(oracle_mod, A, B, C, what=f"n={n} m={m} k={k}")
    assert workspace_status(gpu) == 0


def test_golden_square_cases(gpu, oracle_mod):
    from tests.golden.make_golden import SQUARE_CASES
    from tsm_benchmark_b200 import tsmttsm
    g = np.load(os.path.join(GOLDEN, "ref_square_cases.npz"))
    for n, M, seed in SQUARE_CASES:
        A, B = oracle_mod.operands(n, M, M, seed)
        C = tsmttsm(to_dev(A, gpu), to_dev(B, gpu))
        assert_parity(oracle_mod, A, B, C, g[f"n{n}_M{M}_s{seed}"], what=f"golden n={n} M={M}")


def test_config0_main_cc_inputs(gpu, oracle_mod):
    """n = 2^20, m = k = 8 with main.cc's own inputs; checked, as main.cc
    checks its kernels, against the reference's compute_naive output, and
    against the reference's tsmttsm4/6/9 outputs recorded on the CPU."""
    from tsm_benchmark_b200 import tsmttsm
    g = np.load(os.path.join(GOLDEN, "ref_config0.npz"))
    A, B = oracle_mod.main_cc_inputs(1 << 20, 8, 123)
    C = torch.zeros((8, 8), dtype=torch.float64, device=gpu)
    tsmttsm(to_dev(A, gpu), to_dev(B, gpu), C, accumulate=True)  # main.cc: zero C, then add
    assert_parity(oracle_mod, A, B, C, g["C_naive"], what="config0")
    for v in (4, 6, 9):
        assert oracle_mod.check(g[f"C_v{v}"], C.cpu().numpy()) == -1


def test_accumulate_semantics(gpu, oracle_mod):
    from tsm_benchmark_b200 import tsmttsm
    A, B = oracle_mod.operands(5001, 8, 16, 3)
    C0 = np.random.default_rng(0).standard_normal((8, 16))
    C = to_dev(C0, gpu)
    tsmttsm(to_dev(A, gpu), to_dev(B, gpu), C, accumulate=True)
    assert_parity(oracle_mod, A, B, C.cpu().numpy() - C0, what="accumulate")
    # accumulate=False overwrites whatever C held (NaN included)
    C.fill_(float("nan"))
    tsmttsm(to_dev(A, gpu), to_dev(B, gpu), C, accumulate=False)
    assert_parity(oracle_mod, A, B, C, what="overwrite")
    # n = 0: C = 0, or C unchanged when accumulating
    E = torch.empty((0, 8), dtype=torch.float64, device=gpu)
    F = torch.empty((0, 16), dtype=torch.float64, device=gpu)
    C.fill_(3.0)
    tsmttsm(E, F, C, accumulate=True)
    assert torch.all(C == 3.0)
    tsmttsm(E, F, C, accumulate=False)
    assert torch.all(C == 0.0)


def test_deterministic(gpu, oracle_mod):
    from tsm_benchmark_b200 import tsmttsm
    A, B = oracle_mod.operands(1 << 18, 16, 16, 5)
    dA, dB = to_dev(A, gpu), to_dev(B, gpu)
    first = tsmttsm(dA, dB).clone()
    for _ in range(5):
        assert torch.equal(tsmttsm(dA, dB), first)


def test_every_applicable_variant(gpu, oracle_mod):
    """Each compiled variant that accepts a shape computes it correctly."""
    from tsm_benchmark_b200 import TsmError, tsmttsm, variants
    cases = {}
    for m, k in [(1, 1), (8, 8), (16, 16), (64, 64), (4, 32), (5, 12), (1, 64), (32, 32)]:
        cases[(m, k)] = oracle_mod.operands(3001, m, k, 11 + m + k)
    ran = 0
    for v in variants():
        if v["dtype"] != "f64":
            continue
        for (m, k), (A, B) in cases.items():
            fits = (m == v["wa"] and k == v["wb"]) if v["exact"] else (m <= v["wa"] and k <= v["wb"])
            if not fits:
                continue
            if v["gram"]:  # B is A: the Gram variants take one operand
                dA = to_dev(A, gpu)
                C = tsmttsm(dA, dA, variant=v["index"])
                assert_parity(oracle_mod, A, A, C, what=v["name"])
            else:
                C = tsmttsm(to_dev(A, gpu), to_dev(B, gpu), variant=v["index"])
                assert_parity(oracle_mod, A, B, C, what=v["name"])
            ran += 1
    assert ran >= 40


def test_strided_and_unaligned_operands(gpu, oracle_mod):
    """lda > m (column slice of a wider matrix) and operands that start 8
    bytes past a 16-byte boundary take the direct-load kernels."""
    from tsm_benchmark_b200 import default_variant, tsmttsm, variants
    names = [v["name"] for v in variants()]
    A_wide, B_wide = oracle_mod.operands(7777, 24, 40, 21)
    A, B = A_wide[:, 3:11], B_wide[:, 5:37]
    dA = to_dev(A_wide, gpu)[:, 3:11]
    dB = to_dev(B_wide, gpu)[:, 5:37]
    assert names[default_variant(dA, dB)].startswith("direct")
    C = tsmttsm(dA, dB)
    assert_parity(oracle_mod, np.ascontiguousarray(A), np.ascontiguousarray(B), C, what="strided")
    A, B = oracle_mod.operands(5000, 8, 8, 22)
    bufA = torch.zeros(A.size + 1, dtype=torch.float64, device=gpu)
    bufB = torch.zeros(B.size + 1, dtype=torch.float64, device=gpu)
    bufA[1:] = to_dev(A.ravel(), gpu)
    bufB[1:] = to_dev(B.ravel(), gpu)
    dA, dB = bufA[1:].view(5000, 8), bufB[1:].view(5000, 8)
    assert dA.data_ptr() % 16 == 8
    assert names[default_variant(dA, dB)].startswith("direct")
    assert_parity(oracle_mod, A, B, tsmttsm(dA, dB), what="unaligned")


def test_argument_errors(gpu):
    from tsm_benchmark_b200 import TsmError, tsmttsm
    from tsm_benchmark_b200 import _capi
    A = torch.zeros((10, 65), dtype=torch.float64, device=gpu)
    with pytest.raises(TsmError):
        tsmttsm(A, A)
    with pytest.raises(TypeError):
        tsmttsm(A.half(), A.half())
    with pytest.raises(TypeError):
        tsmttsm(A, A.float())
    lib = _capi.load()
    A = torch.zeros((10, 8), dtype=torch.float64, device=gpu)
    C = torch.zeros((8, 8), dtype=torch.float64, device=gpu)
    ws = torch.zeros(64, dtype=torch.uint8, device=gpu)
    st = lib.tsm_gemm_tn_f64(None, 10, 8, 8, A.data_ptr(), 8, A.data_ptr(), 8, C.data_ptr(), 8, 0, ws.data_ptr(), 64)
    assert st == 2  # workspace too small
    st = lib.tsm_gemm_tn_f64(None, 10, 8, 8, A.data_ptr(), 7, A.data_ptr(), 8, C.data_ptr(), 8, 0, ws.data_ptr(), 64)
    assert st == 1  # lda < m
    st = lib.tsm_gemm_tn_f64_variant(None, 10, 8, 8, A.data_ptr(), 8, A.data_ptr(), 8, C.data_ptr(), 8, 0,
                                     ws.data_ptr(), 1 << 30, 10**6)
    assert st in (2, 4)


def test_device_fill_matches_oracle_generator(gpu, oracle_mod):
    from tsm_benchmark_b200 import fill_uniform
    x = torch.empty(1 << 20, dtype=torch.float64, device=gpu)
    fill_uniform(x, seed=99, stream_id=3)
    assert np.array_equal(x.cpu().numpy(), oracle_mod.uniform(1 << 20, 99, 3))


@pytest.mark.parametrize("m,k", [(1, 1), (8, 8), (16, 16), (1, 64)])
def test_full_size_properties(gpu, m, k):
    """n = 2^26 (the sweep's row count): against cuBLAS DGEMM through torch
    within the normwise bound, and the checksum identity
    sum_ij C_ij = sum_r (sum_i A_ri)(sum_j B_rj)."""
    from tsm_benchmark_b200 import fill_uniform, tsmttsm
    n = 1 << 26 if m * k <= 256 else 1 << 24
    A = torch.empty((n, m), dtype=torch.float64, device=gpu)
    B = torch.empty((n, k), dtype=torch.float64, device=gpu)
    fill_uniform(A, 1, 0)
    fill_uniform(B, 1, 1)
    C = tsmttsm(A, B)
    C2 = A.T @ B
    bound = 4 * np.sqrt(n) * 2.0**-53 * float(torch.linalg.norm(A)) * float(torch.linalg.norm(B))
    assert float(torch.linalg.norm(C - C2)) <= 2 * bound
    chk = float((A.sum(1) * B.sum(1)).sum())
    assert abs(float(C.sum()) - chk) <= 4 * bound * np.sqrt(m * k)
    del A, B
    torch.cuda.empty_cache()


F32_SHAPES = [(1, 1), (2, 2), (3, 5), (4, 4), (8, 8), (16, 16), (32, 32), (64, 64), (4, 32), (7, 13)]


@pytest.mark.parametrize("m,k", F32_SHAPES)
def test_parity_fp32_storage(gpu, oracle_mod, m, k):
    """FP32 storage: per-thread FP32 accumulation, FP64 reductions, one
    rounding to FP32.  Checked against the oracle's FP64 product of the FP32
    values with a bound for FP32 accumulation over the rows one thread sums:
    ||C - C_ref||_F <= 2^-24 (rows per thread + 2) ||A||_F ||B||_F."""
    from tsm_benchmark_b200 import tsmttsm, variants
    for n in (0, 1, 3, 4099, 100003):
        A, B = oracle_mod.operands(n, m, k, seed=77 + n + m * k)
        A32, B32 = A.astype(np.float32), B.astype(np.float32)
        C = tsmttsm(to_dev(A32, gpu), to_dev(B32, gpu))
        assert C.dtype == torch.float32
        ref = oracle_mod.naive(A32, B32)
        got = C.cpu().numpy().astype(np.float64)
        err = np.linalg.norm(got - ref)
        per_thread = max(1, n // (148 * 8)) + 2
        bound = 2.0**-24 * per_thread * np.linalg.norm(A32.astype(np.float64)) * np.linalg.norm(B32.astype(np.float64))
        assert err <= bound + 1e-30, (n, m, k, err, bound)
    names = [v for v in variants() if v["dtype"] == "f32"]
    assert names


def test_every_fp32_exact_variant(gpu, oracle_mod):
    """Every FP32-storage exact square, each ring shape (2, 3 and 6 stages),
    on a ragged row count and on one shorter than a chunk, with the bound of
    the FP32 parity test."""
    from tsm_benchmark_b200 import tsmttsm, variants
    ran = 0
    for v in variants():
        if v["dtype"] != "f32" or not v["exact"] or v["kind"] != "bulk":
            continue
        m = k = v["wa"]
        for n in (v["rows"] - 3, 100003):
            A, B = oracle_mod.operands(n, m, k, seed=91 + m + n)
            A32, B32 = A.astype(np.float32), B.astype(np.float32)
            C = tsmttsm(to_dev(A32, gpu), to_dev(B32, gpu), variant=v["index"])
            ref = oracle_mod.naive(A32, B32)
            err = np.linalg.norm(C.cpu().numpy().astype(np.float64) - ref)
            per_thread = max(1, n // (148 * 8)) + 2
            bound = 2.0**-24 * per_thread * np.linalg.norm(A32.astype(np.float64)) * np.linalg.norm(B32.astype(np.float64))
            assert err <= bound + 1e-30, (v["name"], n, err, bound)
        ran += 1
    assert ran >= 21


def test_side_stream_with_fresh_workspace_cache(gpu, oracle_mod, monkeypatch):
    """A call on a caller-supplied stream creates its workspace ON that
    stream: the zero-fill is ordered before the kernel even while the
    current stream is busy.  The current stream is kept busy with a long
    fill, and the products run on a side stream with an empty cache; the
    batched plan is built and run on the side stream too."""
    from tsm_benchmark_b200 import BatchedTSMTTSM, api, gram, tsmttsm, tsmttsm_split
    monkeypatch.setattr(api, "_workspaces", {})
    side = torch.cuda.Stream(gpu)
    A, B = oracle_mod.operands(100003, 8, 16, 41)
    A32, B32 = A.astype(np.float32), B.astype(np.float32)
    dA, dB, dA32, dB32 = (to_dev(x, gpu) for x in (A, B, A32, B32))
    busy = torch.empty(1 << 28, dtype=torch.float64, device=gpu)
    torch.cuda.synchronize()
    for _ in range(2):
        busy.fill_(1.0)  # ~2 GiB of writes queued on the current stream
        with torch.cuda.stream(side):
            C = tsmttsm(dA, dB, stream=side)
            G = gram(dA, stream=side)
            S = tsmttsm_split(dA32, dB32, stream=side)
            bt = BatchedTSMTTSM([dA], [dB], stream=side)
            Cb = bt.run(stream=side)[0]
        side.synchronize()
        assert_parity(oracle_mod, A, B, C, what="side stream")
        assert_parity(oracle_mod, A, A, G, what="side stream gram")
        assert_parity(oracle_mod, A, B, Cb, what="side stream batched")
        ref32 = oracle_mod.naive(A32, B32)
        assert np.linalg.norm(S.cpu().numpy() - ref32) <= 1e-6 * np.linalg.norm(ref32)
        monkeypatch.setattr(api, "_workspaces", {})
    torch.cuda.synchronize()
    del busy


@pytest.mark.parametrize("m,k", [(8, 8), (16, 16), (64, 64), (3, 5), (1, 64), (32, 4)])
def test_launch_with_cta_caps(gpu, oracle_mod, m, k):
    """tsm_gemm_tn_f64_launch caps the grid (the generated drop-in kernels
    pass the reference's stride / local_size work-groups): every kernel
    family deals its rows over any grid of 1 CTA or more and gives the same
    product within the oracle's bounds; a cap above the variant's own grid
    changes nothing."""
    from tsm_benchmark_b200 import _capi, default_variant
    lib = _capi.load()
    sh = int(torch.cuda.current_stream(gpu).cuda_stream)
    for n in (777, 100003):
        A, B = oracle_mod.operands(n, m, k, seed=310 + n + m * k)
        dA, dB = to_dev(A, gpu), to_dev(B, gpu)
        need = lib.tsm_gemm_tn_workspace_size(n, m, k)
        ws = torch.zeros(need, dtype=torch.uint8, device=gpu)
        ref = oracle_mod.naive(A, B)
        full = None
        for cap in (1, 2, 7, 37, 0, 1 << 20):
            C = torch.full((m, k), float("nan"), dtype=torch.float64, device=gpu)
            st = lib.tsm_gemm_tn_f64_launch(sh, n, m, k, dA.data_ptr(), m, dB.data_ptr(), k, C.data_ptr(), k, 0,
                                            ws.data_ptr(), need, -1, cap)
            assert st == 0, _capi.STATUS[st]
            torch.cuda.synchronize()
            assert_parity(oracle_mod, A, B, C, ref, what=f"cap {cap}, n={n} {m}x{k}")
            if cap == 0:
                full = C.clone()
            if cap == 1 << 20:  # above the variant's grid: the same launch as no cap
                assert torch.equal(C, full)
        assert default_variant(dA, dB) >= 0
