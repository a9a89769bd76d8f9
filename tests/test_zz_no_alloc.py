"""tsm_gemm_tn_f64_noalloc: the entry point for callers that cannot allocate.

A caller that may not create device allocations of its own -- a plug-in
whose host program owns all device memory, or a loop where cudaMalloc and
its possible device-wide synchronisation are not allowed -- gets the same
product without passing a workspace: the scratch is a fixed 4 MiB array
inside the library.  These tests drive it through the C ABI and compare it
with tsm_gemm_tn_f64 (the workspace entry point) under the tolerance of the
other parity tests.  This file is collected last on purpose.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

REL_TOL, ABS_TOL = 1e-6, 1e-10  # the element rule of the parity tests (main.cc:29-41)


def assert_close(ref: torch.Tensor, got: torch.Tensor, what: str) -> None:
    r = ref.cpu().numpy()
    g = got.cpu().numpy()
    diff = np.abs(r - g)
    mag = np.maximum(np.abs(r), np.abs(g))
    ok = (diff <= ABS_TOL) | (diff <= REL_TOL * mag)
    assert ok.all(), f"{what}: {np.argwhere(~ok)[:4].tolist()} ref {r[~ok][:4]} got {g[~ok][:4]}"


def operands(dev, n, m, k, seed):
    from tsm_benchmark_b200 import fill_uniform
    A = torch.empty((n, m), dtype=torch.float64, device=dev)
    B = torch.empty((n, k), dtype=torch.float64, device=dev)
    fill_uniform(A, seed, 0)
    fill_uniform(B, seed, 1)
    return A, B


@pytest.mark.parametrize("n,m,k", [(1 << 20, 8, 8), (100003, 16, 16), (4099, 3, 5), (70001, 32, 64),
                                   (0, 4, 4), (3001, 64, 64)])
def test_noalloc_matches_workspace_entry_point(n, m, k):
    from tsm_benchmark_b200 import _capi
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    lib = _capi.load()
    sh = int(torch.cuda.current_stream(dev).cuda_stream)
    A, B = operands(dev, n, m, k, seed=n + 31 * m + k)

    need = lib.tsm_gemm_tn_workspace_size(n, m, k)
    ws = torch.zeros(need, dtype=torch.uint8, device=dev)
    C_ref = torch.empty((m, k), dtype=torch.float64, device=dev)
    st = lib.tsm_gemm_tn_f64(sh, n, m, k, A.data_ptr(), m, B.data_ptr(), k, C_ref.data_ptr(), k, 0,
                             ws.data_ptr(), need)
    assert st == 0, _capi.STATUS[st]

    # Two calls in a row on the shared static scratch, each into a C full of NaN.
    for call in range(2):
        C = torch.full((m, k), float("nan"), dtype=torch.float64, device=dev)
        st = lib.tsm_gemm_tn_f64_noalloc(sh, n, m, k, A.data_ptr(), m, B.data_ptr(), k, C.data_ptr(), k, 0)
        assert st == 0, _capi.STATUS[st]
        torch.cuda.synchronize()
        assert_close(C_ref, C, f"call {call + 1}, n={n} m={m} k={k}")

    # accumulate = 1 adds into C
    C = C_ref.clone()
    st = lib.tsm_gemm_tn_f64_noalloc(sh, n, m, k, A.data_ptr(), m, B.data_ptr(), k, C.data_ptr(), k, 1)
    assert st == 0
    torch.cuda.synchronize()
    assert_close(2 * C_ref, C, "accumulate")
    assert_no_device_error(lib, sh)


def assert_no_device_error(lib, sh):
    """No kernel of the calls above gave up a bounded wait: the scratch's
    error word, read and cleared by tsm_noalloc_check, is zero."""
    import ctypes
    bits = ctypes.c_uint(0xFFFFFFFF)
    st = lib.tsm_noalloc_check(sh, ctypes.byref(bits))
    assert st == 0 and bits.value == 0, (st, bits.value)


@pytest.mark.parametrize("n,m", [(1 << 20, 8), (100003, 16), (4099, 5), (20011, 32)])
def test_noalloc_gram_route_when_b_is_a(n, m):
    """B passed as A itself (same pointer, pitch and width) takes the Gram
    kernels, which stream A once and write C exactly symmetric; the result
    matches the workspace entry point's on the same request, twice."""
    from tsm_benchmark_b200 import _capi
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    lib = _capi.load()
    sh = int(torch.cuda.current_stream(dev).cuda_stream)
    A, _ = operands(dev, n, m, 1, seed=n + m)
    need = lib.tsm_gemm_tn_workspace_size(n, m, m)
    ws = torch.zeros(need, dtype=torch.uint8, device=dev)
    C_ref = torch.empty((m, m), dtype=torch.float64, device=dev)
    st = lib.tsm_gemm_tn_f64(sh, n, m, m, A.data_ptr(), m, A.data_ptr(), m, C_ref.data_ptr(), m, 0,
                             ws.data_ptr(), need)
    assert st == 0, _capi.STATUS[st]
    for call in range(2):
        C = torch.full((m, m), float("nan"), dtype=torch.float64, device=dev)
        st = lib.tsm_gemm_tn_f64_noalloc(sh, n, m, m, A.data_ptr(), m, A.data_ptr(), m, C.data_ptr(), m, 0)
        assert st == 0, _capi.STATUS[st]
        torch.cuda.synchronize()
        assert_close(C_ref, C, f"Gram call {call + 1}, n={n} m={m}")
        assert torch.equal(C, C.T)
    assert_no_device_error(lib, sh)


def test_noalloc_rejects_requests_beyond_its_scratch():
    """64 x 64 over 2^20 rows needs one 32 KB partial per CTA on every SM,
    more than the 4 MiB array: refused with TSM_ERROR_WORKSPACE, C untouched."""
    from tsm_benchmark_b200 import _capi
    dev = torch.device("cuda", 0)
    lib = _capi.load()
    sh = int(torch.cuda.current_stream(dev).cuda_stream)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    n, m, k = 1 << 20, 64, 64
    A, B = operands(dev, n, m, k, seed=5)
    C = torch.full((m, k), 7.0, dtype=torch.float64, device=dev)
    st = lib.tsm_gemm_tn_f64_noalloc(sh, n, m, k, A.data_ptr(), m, B.data_ptr(), k, C.data_ptr(), k, 0)
    if 256 + min(sms, n // 32) * m * k * 8 > (4 << 20):
        assert st == 2, _capi.STATUS[st]
        torch.cuda.synchronize()
        assert torch.all(C == 7.0)
    else:  # pragma: no cover - a GPU with fewer SMs fits the request
        assert st == 0
    # argument errors are reported like the workspace entry point's
    assert lib.tsm_gemm_tn_f64_noalloc(sh, 10, 65, 4, A.data_ptr(), 65, B.data_ptr(), 4, C.data_ptr(), 4, 0) == 1
