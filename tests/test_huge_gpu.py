"""Row counts past 2^31 (the largest the 32-bit row coordinates of the
tensor-map kernels address): n = 2^31 + 4099 on the paths that take over
there -- the SIMT bulk kernels (1 x 1, 2 x 2, the Gram variant), the strided
kernel for column-major operands, and the 1-D split kernel (FP32 4 x 4).
Each case holds 34-69 GB on the device and releases it before returning.

The reference is cuBLAS FP64 (torch.matmul) over chunks of 2^28 rows,
summed in FP64; acceptance is twice the normwise bound of the plain-path
tests (the reference carries an error of the same size),
||C - C_ref||_F <= 2 * 4 sqrt(n) 2^-53 ||A||_F ||B||_F, and 1e-6 relative
for the split form.
"""
import math

import pytest
import torch

pytestmark = pytest.mark.gpu

N = (1 << 31) + 4099
CHUNK = 1 << 28


def chunked_ref(A, B):
    C = torch.zeros((A.shape[1], B.shape[1]), dtype=torch.float64, device=A.device)
    for r in range(0, A.shape[0], CHUNK):
        C += A[r:r + CHUNK].double().T @ B[r:r + CHUNK].double()
    return C


def fro(X):
    return math.sqrt(sum(float(torch.linalg.norm(X[r:r + CHUNK].double())) ** 2 for r in range(0, X.shape[0], CHUNK)))


def bound(A, B):
    return 2 * 4 * math.sqrt(A.shape[0]) * 2.0**-53 * fro(A) * fro(B)


@pytest.mark.parametrize("w", [1, 2])
def test_rows_past_int32_plain_and_gram(gpu, w):
    from tsm_benchmark_b200 import fill_uniform, gram, tsmttsm, workspace_status
    A = torch.empty((N, w), dtype=torch.float64, device=gpu)
    B = torch.empty((N, w), dtype=torch.float64, device=gpu)
    fill_uniform(A, 21, 0)
    fill_uniform(B, 21, 1)
    C = tsmttsm(A, B)
    err, lim = float(torch.linalg.norm(C - chunked_ref(A, B))), bound(A, B)
    G = gram(A)
    errg, limg = float(torch.linalg.norm(G - chunked_ref(A, A))), bound(A, A)
    sym = bool(torch.equal(G, G.T))
    bits = workspace_status(gpu)
    del A, B
    torch.cuda.empty_cache()
    assert err <= lim, (err, lim)
    assert errg <= limg and sym, (errg, limg, sym)
    assert bits == 0


def test_rows_past_int32_column_major(gpu):
    from tsm_benchmark_b200 import fill_uniform, tsmttsm
    X = torch.empty((2, N), dtype=torch.float64, device=gpu)  # A^T, B^T row-major: A, B column-major
    Y = torch.empty((2, N), dtype=torch.float64, device=gpu)
    fill_uniform(X, 22, 0)
    fill_uniform(Y, 22, 1)
    C = tsmttsm(X.t(), Y.t())
    ref = torch.zeros((2, 2), dtype=torch.float64, device=gpu)
    for r in range(0, N, CHUNK):
        ref += X[:, r:r + CHUNK].contiguous() @ Y[:, r:r + CHUNK].contiguous().T  # cuBLAS pitches < 2^31
    err, lim = float(torch.linalg.norm(C - ref)), bound(X.t(), Y.t())
    del X, Y
    torch.cuda.empty_cache()
    assert err <= lim, (err, lim)


def test_rows_past_int32_split(gpu):
    from tsm_benchmark_b200 import fill_uniform, tsmttsm_split
    A = torch.empty((N, 4), dtype=torch.float32, device=gpu)
    B = torch.empty((N, 4), dtype=torch.float32, device=gpu)
    for T, sid in ((A, 0), (B, 1)):
        for r in range(0, N, CHUNK):
            part = torch.empty((min(CHUNK, N - r), 4), dtype=torch.float64, device=gpu)
            fill_uniform(part, 23 + r // CHUNK, sid)
            T[r:r + CHUNK] = part.float()
            del part
    C = tsmttsm_split(A, B)
    ref = chunked_ref(A, B)
    rel = float(torch.linalg.norm(C - ref) / torch.linalg.norm(ref))
    del A, B
    torch.cuda.empty_cache()
    assert rel <= 1e-6, rel
