"""Canaries: every kernel family writes only its outputs.  C (and dA / dB)
sit inside larger buffers filled with a sentinel, at a row pitch above
their width; the workspace has a sentinel tail past the size the library
asked for.  After each call the sentinels must be untouched."""
import numpy as np
import pytest
import torch

from tests.test_plain_gpu import to_dev

pytestmark = pytest.mark.gpu

SENTINEL = -12345.6789


def framed(rows, cols, dev, dtype=torch.float64):
    """A (rows x cols) view at offset (1, 1) of a (rows + 2) x (cols + 3)
    sentinel-filled buffer (row pitch cols + 3)."""
    buf = torch.full((rows + 2, cols + 3), SENTINEL, dtype=dtype, device=dev)
    return buf, buf[1:rows + 1, 1:cols + 1]


def assert_frame(buf, rows, cols, what):
    mask = torch.ones_like(buf, dtype=torch.bool)
    mask[1:rows + 1, 1:cols + 1] = False
    assert bool((buf[mask] == SENTINEL).all()), what


@pytest.mark.parametrize("m,k,gram", [(8, 8, False), (32, 32, False), (64, 64, False), (5, 12, False),
                                      (16, 16, True), (32, 32, True), (4, 4, True)])
def test_plain_and_gram_write_only_c(gpu, oracle_mod, m, k, gram):
    from tsm_benchmark_b200 import _capi
    lib = _capi.load()
    sh = torch.cuda.current_stream(gpu).cuda_stream
    n = 50021
    A, B = oracle_mod.operands(n, m, k, 13 + m + k)
    dA = to_dev(A, gpu)
    dB = dA if gram else to_dev(B, gpu)
    ldb, kk = (m, m) if gram else (k, k)
    need = lib.tsm_gemm_tn_workspace_size(n, m, kk)
    ws = torch.full((need + 4096,), 0xA5, dtype=torch.uint8, device=gpu)
    ws[:need] = 0
    buf, C = framed(m, kk, gpu)
    st = lib.tsm_gemm_tn_f64(sh, n, m, kk, dA.data_ptr(), m, dB.data_ptr(), ldb, C.data_ptr(), C.stride(0), 0,
                             ws.data_ptr(), need)
    assert st == 0
    torch.cuda.synchronize()
    assert_frame(buf, m, kk, f"C frame {m}x{kk} gram={gram}")
    assert bool((ws[need:] == 0xA5).all()), "workspace tail"
    ref = oracle_mod.naive(A, A if gram else B)
    assert np.allclose(C.cpu().numpy(), ref, rtol=1e-12, atol=1e-9 * np.abs(ref).max())


def test_split_and_backward_write_only_outputs(gpu, oracle_mod):
    from tsm_benchmark_b200 import _capi
    lib = _capi.load()
    sh = torch.cuda.current_stream(gpu).cuda_stream
    n, m, k = 20011, 16, 32
    A, B = oracle_mod.operands(n, m, k, 77)
    need = lib.tsm_gemm_tn_workspace_size(n, m, k)
    ws = torch.full((need + 4096,), 0xA5, dtype=torch.uint8, device=gpu)
    ws[:need] = 0
    # split precision: FP32 operands, FP64 C in a frame
    A32, B32 = to_dev(A.astype(np.float32), gpu), to_dev(B.astype(np.float32), gpu)
    buf, C = framed(m, k, gpu)
    assert lib.tsm_gemm_tn_f32_split(sh, n, m, k, A32.data_ptr(), m, B32.data_ptr(), k, C.data_ptr(), C.stride(0),
                                     0, ws.data_ptr(), need) == 0
    torch.cuda.synchronize()
    assert_frame(buf, m, k, "split C frame")
    for parts in (2, 3):  # BF16 parts
        buf, C = framed(m, k, gpu)
        assert lib.tsm_gemm_tn_f32_split_bf16(sh, n, m, k, A32.data_ptr(), m, B32.data_ptr(), k, C.data_ptr(),
                                              C.stride(0), 0, parts, ws.data_ptr(), need) == 0
        torch.cuda.synchronize()
        assert_frame(buf, m, k, f"split bf16 x{parts} C frame")
        assert bool((ws[need:] == 0xA5).all()), "workspace tail"
    # fused backward: dA (n x m) and dB (n x k) in frames
    dC = to_dev(np.random.default_rng(1).standard_normal((m, k)), gpu)
    dA_in, dB_in = to_dev(A, gpu), to_dev(B, gpu)
    bufA, gA = framed(n, m, gpu)
    bufB, gB = framed(n, k, gpu)
    assert lib.tsm_gemm_tn_backward_f64(sh, n, m, k, dA_in.data_ptr(), m, dB_in.data_ptr(), k, dC.data_ptr(), k,
                                        gA.data_ptr(), gA.stride(0), gB.data_ptr(), gB.stride(0), 0,
                                        ws.data_ptr(), need) == 0
    torch.cuda.synchronize()
    assert_frame(bufA, n, m, "dA frame")
    assert_frame(bufB, n, k, "dB frame")
    assert bool((ws[need:] == 0xA5).all()), "workspace tail"
    dCn = dC.cpu().numpy()
    assert np.allclose(gA.cpu().numpy(), oracle_mod.tsmm(B, dCn.T.copy()), rtol=1e-12, atol=1e-12)
    assert np.allclose(gB.cpu().numpy(), oracle_mod.tsmm(A, dCn), rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("m,k,layout", [(4, 4, "col"), (8, 8, "col"), (1, 64, "col"), (32, 32, "col"),
                                        (4, 32, "col"), (64, 64, "col"), (5, 7, "mixed"), (64, 64, "mixed")])
def test_strided_layouts_write_only_c(gpu, oracle_mod, m, k, layout):
    """Column-major operands (tensor-map SIMT and FP64 tensor-core kernels)
    and a mixed layout (the strided register-tile kernel)."""
    from tsm_benchmark_b200 import _capi
    lib = _capi.load()
    sh = torch.cuda.current_stream(gpu).cuda_stream
    n = 50021
    A, B = oracle_mod.operands(n, m, k, 31 + m + k)
    At = to_dev(A.T, gpu)  # m x n row-major: A column-major with pitch n
    Bt = to_dev(B.T, gpu)
    need = lib.tsm_gemm_tn_workspace_size(n, m, k)
    ws = torch.full((need + 4096,), 0xA5, dtype=torch.uint8, device=gpu)
    ws[:need] = 0
    buf, C = framed(m, k, gpu)
    if layout == "col":
        # pitch n + 1 is even for n = 50021: the pipelined kernels
        Ap = torch.zeros((m, n + 1), dtype=torch.float64, device=gpu)
        Bp = torch.zeros((k, n + 1), dtype=torch.float64, device=gpu)
        Ap[:, :n] = At
        Bp[:, :n] = Bt
        args = (Ap.data_ptr(), 1, n + 1, Bp.data_ptr(), 1, n + 1)
    else:
        Ar = to_dev(A, gpu)
        args = (Ar.data_ptr(), m, 1, Bt.data_ptr(), 1, n)
    st = lib.tsm_gemm_tn_strided_f64(sh, n, m, k, *args, C.data_ptr(), C.stride(0), 0, ws.data_ptr(), need)
    assert st == 0
    torch.cuda.synchronize()
    assert_frame(buf, m, k, f"C frame {m}x{k} {layout}")
    assert bool((ws[need:] == 0xA5).all()), "workspace tail"
    ref = oracle_mod.naive(A, B)
    assert np.allclose(C.cpu().numpy(), ref, rtol=1e-12, atol=1e-9 * np.abs(ref).max())
