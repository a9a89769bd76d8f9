"""Device failure detection: a kernel's bounded wait that runs out (a
barrier nothing arrives on -- no fault, no trap) is recorded in the
workspace's error word, reported by tsm_workspace_check as
TSM_ERROR_DEVICE_TIMEOUT, cleared, and the context keeps working."""
import ctypes

import pytest
import torch

from tests.test_plain_gpu import assert_parity, to_dev

pytestmark = pytest.mark.gpu


def test_wait_timeout_is_reported_and_cleared(gpu, oracle_mod):
    from tsm_benchmark_b200 import _capi
    lib = _capi.load()
    sh = torch.cuda.current_stream(gpu).cuda_stream
    m = k = 8
    need = lib.tsm_gemm_tn_workspace_size(4096, m, k)
    ws = torch.zeros(need, dtype=torch.uint8, device=gpu)
    bits = ctypes.c_uint(0)
    assert lib.tsm_selftest_wait_timeout(sh, ws.data_ptr(), need, 1000) == 0
    assert lib.tsm_workspace_check(sh, ws.data_ptr(), ctypes.byref(bits)) == 5  # TSM_ERROR_DEVICE_TIMEOUT
    assert bits.value & 1
    assert lib.tsm_workspace_check(sh, ws.data_ptr(), ctypes.byref(bits)) == 0 and bits.value == 0  # cleared
    # the same workspace and context still compute a correct product
    A, B = oracle_mod.operands(4096, m, k, 3)
    dA, dB = to_dev(A, gpu), to_dev(B, gpu)
    C = torch.empty((m, k), dtype=torch.float64, device=gpu)
    st = lib.tsm_gemm_tn_f64(sh, 4096, m, k, dA.data_ptr(), m, dB.data_ptr(), k, C.data_ptr(), k, 0,
                             ws.data_ptr(), need)
    assert st == 0
    assert lib.tsm_workspace_check(sh, ws.data_ptr(), ctypes.byref(bits)) == 0 and bits.value == 0
    assert_parity(oracle_mod, A, B, C, what="after a timeout")


def test_selftest_argument_errors(gpu):
    from tsm_benchmark_b200 import _capi
    lib = _capi.load()
    sh = torch.cuda.current_stream(gpu).cuda_stream
    ws = torch.zeros(256, dtype=torch.uint8, device=gpu)
    assert lib.tsm_selftest_wait_timeout(sh, ws.data_ptr(), 256, 0) == 1             # TSM_ERROR_INVALID_VALUE
    assert lib.tsm_selftest_wait_timeout(sh, ws.data_ptr(), 255, 1000) != 0          # workspace too small
    assert lib.tsm_selftest_wait_timeout(sh, ws.data_ptr(), 256, 3_000_000) == 1     # above the 2 s cap
