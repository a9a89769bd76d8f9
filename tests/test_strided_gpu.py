"""Parity of the general-layout product (tsm_gemm_tn_strided_f64) with the
oracle: column-major operands (A stored as the m x n row-major A^T, the
tensor-map kernels -- SIMT below 64 products of the power-of-two widths,
FP64 tensor cores above), column pitches above n, mixed layouts, odd pitches
and unaligned bases (the strided register-tile kernel).

Acceptance as for the plain path: the reference's is_correct rule
(main.cc:29-41) per entry and ||C - C_oracle||_F <= 4 sqrt(n) 2^-53
||A||_F ||B||_F per matrix, against compute_naive on the same values.
"""
import numpy as np
import pytest
import torch

from tests.test_plain_gpu import assert_parity

pytestmark = pytest.mark.gpu


def column_major(x: np.ndarray, dev, pad: int = 0, offset: int = 0) -> torch.Tensor:
    """An n x w view with strides (1, n + pad) over a device buffer holding
    x^T row by row, starting `offset` elements into the buffer."""
    n, w = x.shape
    pitch = n + pad
    buf = torch.zeros(offset + w * pitch + 8, dtype=torch.float64, device=dev)
    rows = buf[offset:offset + w * pitch].view(w, pitch)
    rows[:, :n] = torch.from_numpy(np.ascontiguousarray(x.T)).to(dev)
    return rows[:, :n].t()


def row_major(x: np.ndarray, dev, pad: int = 0, offset: int = 0) -> torch.Tensor:
    n, w = x.shape
    pitch = w + pad
    buf = torch.zeros(offset + max(n, 1) * pitch + 8, dtype=torch.float64, device=dev)
    rows = buf[offset:offset + n * pitch].view(n, pitch)
    rows[:, :w] = torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    return rows[:, :w]


# (m, k): SIMT capacities (1x1 ... 8x8, 1x64, 64x1, 2x32, 16x4, 3x5 -> 4x8),
# tensor-core capacities 8 (4x32, 8x16 via 5x12 and 7x9, 40x8 -> 48x8,
# 64x3 -> 64x8, 8x64) and 16-64.
CM_SHAPES = [(1, 1), (2, 2), (4, 4), (8, 8), (3, 5), (1, 64), (64, 1), (2, 32), (16, 4), (5, 12),
             (16, 16), (32, 32), (64, 64), (48, 48), (16, 64), (20, 40), (33, 17), (7, 9), (64, 3),
             (4, 32), (40, 8), (8, 64)]
CM_ROWS = [0, 1, 15, 16, 17, 2047, 2049, 4096, 70001]


@pytest.mark.parametrize("m,k", CM_SHAPES)
def test_column_major_parity(gpu, oracle_mod, m, k):
    from tsm_benchmark_b200 import tsmttsm, workspace_status
    for n in CM_ROWS:
        A, B = oracle_mod.operands(n, m, k, seed=4000 + n + 7 * m + k)
        Ad, Bd = column_major(A, gpu), column_major(B, gpu)
        assert n <= 1 or (Ad.stride(0) == 1 and Bd.stride(0) == 1)
        C = tsmttsm(Ad, Bd)
        torch.cuda.synchronize()
        assert_parity(oracle_mod, A, B, C, what=f"column-major n={n} m={m} k={k}")
    assert workspace_status(gpu) == 0


@pytest.mark.parametrize("m,k,pad", [(8, 8, 6), (32, 32, 2), (3, 40, 10), (64, 64, 64)])
def test_column_major_pitch(gpu, oracle_mod, m, k, pad):
    """Column pitch above n (sub-blocks of wider matrices), even pitches:
    still the tensor-map kernels."""
    from tsm_benchmark_b200 import tsmttsm
    for n in (1000, 33335):
        n_even = n + (n + pad) % 2  # keeps n + pad even
        A, B = oracle_mod.operands(n_even, m, k, seed=77 + m + pad)
        C = tsmttsm(column_major(A, gpu, pad), column_major(B, gpu, pad))
        assert_parity(oracle_mod, A, B, C, what=f"pitch n={n_even} pad={pad} m={m} k={k}")


@pytest.mark.parametrize("layout", ["odd_pitch", "unaligned", "mixed_rc", "mixed_cr", "row_strided_cols"])
@pytest.mark.parametrize("m,k", [(1, 1), (5, 7), (8, 8), (16, 33), (64, 64)])
def test_general_layouts(gpu, oracle_mod, layout, m, k):
    from tsm_benchmark_b200 import tsmttsm
    for n in (0, 1, 4099, 20011):
        if m * k >= 1024 and n > 4099:
            continue
        A, B = oracle_mod.operands(n, m, k, seed=900 + n + m + k)
        if layout == "odd_pitch":      # column-major with an odd column pitch
            pad = 1 if n % 2 == 0 else 2
            Ad, Bd = column_major(A, gpu, pad), column_major(B, gpu, pad)
        elif layout == "unaligned":    # column-major, base 8 bytes past a 16-byte boundary
            Ad, Bd = column_major(A, gpu, 0, 1), column_major(B, gpu, 0, 1)
        elif layout == "mixed_rc":
            Ad, Bd = row_major(A, gpu, 3), column_major(B, gpu)
        elif layout == "mixed_cr":
            Ad, Bd = column_major(A, gpu), row_major(B, gpu)
        else:                          # every other element of a row: column stride 2
            wa = torch.zeros((n, 2 * m), dtype=torch.float64, device=gpu)
            wa[:, ::2] = torch.from_numpy(A).to(gpu)
            wb = torch.zeros((n, 2 * k), dtype=torch.float64, device=gpu)
            wb[:, ::2] = torch.from_numpy(B).to(gpu)
            Ad, Bd = wa[:, ::2], wb[:, ::2]
        C = tsmttsm(Ad, Bd)
        torch.cuda.synchronize()
        assert_parity(oracle_mod, A, B, C, what=f"{layout} n={n} m={m} k={k}")


def test_strided_accumulate_and_determinism(gpu, oracle_mod):
    from tsm_benchmark_b200 import tsmttsm
    for m, k in ((4, 4), (32, 32), (7, 33)):
        A, B = oracle_mod.operands(100003, m, k, 5)
        Ad, Bd = column_major(A, gpu), column_major(B, gpu)
        first = tsmttsm(Ad, Bd)
        again = tsmttsm(Ad, Bd)
        assert torch.equal(first, again), "bit-identical from run to run"
        C0 = np.random.default_rng(1).standard_normal((m, k))
        C = torch.from_numpy(C0).to(gpu)
        tsmttsm(Ad, Bd, C, accumulate=True)
        assert_parity(oracle_mod, A, B, C.cpu().numpy() - C0, what=f"accumulate {m}x{k}")


def test_strided_c_abi_row_major_forwarding(gpu, oracle_mod):
    """Unit column strides go to the plain path: same bits as tsmttsm on the
    row-major operands."""
    import ctypes
    from tsm_benchmark_b200 import _capi, tsmttsm
    from tsm_benchmark_b200.api import workspace
    lib = _capi.load()
    n, m, k = 65537, 16, 16
    A, B = oracle_mod.operands(n, m, k, 8)
    Ad = torch.from_numpy(A).to(gpu)
    Bd = torch.from_numpy(B).to(gpu)
    ref = tsmttsm(Ad, Bd)
    C = torch.empty((m, k), dtype=torch.float64, device=gpu)
    sh = int(torch.cuda.current_stream(gpu).cuda_stream)
    ws = workspace(gpu, lib.tsm_gemm_tn_workspace_size(n, m, k), sh)
    st = lib.tsm_gemm_tn_strided_f64(sh, n, m, k, Ad.data_ptr(), m, 1, Bd.data_ptr(), k, 1, C.data_ptr(), k, 0,
                                     ws.data_ptr(), ws.numel())
    assert st == 0
    assert torch.equal(C, ref)
    # invalid strides
    st = lib.tsm_gemm_tn_strided_f64(sh, n, m, k, Ad.data_ptr(), 0, 1, Bd.data_ptr(), k, 1, C.data_ptr(), k, 0,
                                     ws.data_ptr(), ws.numel())
    assert st == 1
    st = lib.tsm_gemm_tn_strided_f64(sh, n, m, k, Ad.data_ptr(), 1, n, Bd.data_ptr(), 1, n, C.data_ptr(), k, 0,
                                     ctypes.c_void_p(0), 0)
    assert st == 2
