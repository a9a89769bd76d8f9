"""Host-side checks that need no GPU: the C ABI library loads and exports
every symbol include/*.h declares, the variant table and the generator agree,
and the Python layer rejects bad arguments before any compute call."""
import glob
import os
import re

import pytest

from tests.conftest import ROOT


def header_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(tsm_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_builds_loads_and_exports_header():
    from tsm_benchmark_b200 import _capi
    lib = _capi.load()
    declared = header_functions()
    assert "tsm_gemm_tn_f64" in declared and len(declared) >= 10
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in include/ but not exported"
    assert set(_capi.SIGNATURES) == declared, "ctypes signatures must cover exactly the header"
    assert lib.tsm_version() >= 100
    assert lib.tsm_status_string(0) == b"success"


def test_variant_table():
    from tsm_benchmark_b200 import codegen, variants
    vs = variants()
    names = [v["name"] for v in vs]
    assert len(names) == len(set(names))
    assert names == [v.name for v in codegen.default_variants()]
    exact_bulk = {(v["wa"], v["wb"]) for v in vs if v["kind"] == "bulk" and v["exact"]}
    for pair in [(1, 1), (2, 2), (4, 4), (8, 8), (16, 16), (32, 32), (64, 64), (4, 32), (32, 4), (1, 64)]:
        assert pair in exact_bulk
    for v in vs:
        assert v["smem_bytes"] <= 227 * 1024
        assert v["threads"] % 32 == 0


def test_generated_sources_current():
    from tsm_benchmark_b200 import codegen
    files = codegen.render(codegen.default_variants(), codegen.load_tuned())
    assert codegen.is_current(files), "run python -m tsm_benchmark_b200.codegen"
    compat = codegen.render_compat_header(codegen.default_variants())
    assert open(codegen.COMPAT_HEADER).read() == compat
    # the names the reference's v2 generator emits by default (sycl_codegen_new.py:645-661)
    for m in (4, 8, 16):
        for tm in (2, 4):
            for suffix in ("", "_lf", "_sg", "_sg_lf"):
                assert f"sycl::event tsmttsm_{m}_{m}_{tm}_{tm}{suffix}(" in compat
    assert "void run_all_benchmarks(sycl::queue& q, int K = 1 << 20, int warmup = 10, int runs = 30)" in compat


def test_generator_rejects_bad_variants():
    from tsm_benchmark_b200 import codegen
    bad = [codegen.BulkVariant(8, 8, 3, 4), codegen.BulkVariant(64, 64, 8, 8, cw=16),
           codegen.BulkVariant(8, 8, 4, 4, rows=255), codegen.DirectVariant(64, 64, 16, 16)]
    for v in bad:
        assert v.validate(), v


def test_python_layer_rejects_cpu_tensors():
    import torch
    from tsm_benchmark_b200 import tsmttsm
    A = torch.zeros((10, 4), dtype=torch.float64)
    with pytest.raises(ValueError):
        tsmttsm(A, A)


def test_c_abi_rejects_bad_arguments_before_any_cuda_call():
    """Argument checks that return before the first CUDA runtime call, so they
    run without a GPU: shapes, strides, part counts, pitches, alignment and
    the 32-bit row limit of the tensor-map kernels, for every entry point
    (plain, FP32, Gram, allocation-free, strided, split, TSMM, backward,
    block orthogonalisation, batched, self-test, fill).  The fake device
    addresses are never dereferenced."""
    import ctypes
    from tsm_benchmark_b200 import _capi
    lib = _capi.load()
    INVALID, WORKSPACE, UNSUPPORTED = 1, 2, 4
    P = ctypes.c_void_p(1 << 20)          # 16-byte aligned, never touched
    Q = ctypes.c_void_p((1 << 20) + 8)    # 8 bytes off a 16-byte boundary
    big = (1 << 31) - 10                  # past the tensor maps' 32-bit row coordinates
    # plain FP64: widths, leading dimensions, null C
    assert lib.tsm_gemm_tn_f64(None, 10, 0, 4, P, 4, P, 4, P, 4, 0, P, 1 << 20) == INVALID
    assert lib.tsm_gemm_tn_f64(None, 10, 65, 4, P, 65, P, 4, P, 4, 0, P, 1 << 20) == INVALID
    assert lib.tsm_gemm_tn_f64(None, 10, 8, 8, P, 7, P, 8, P, 8, 0, P, 1 << 20) == INVALID
    assert lib.tsm_gemm_tn_f64(None, 10, 8, 8, P, 8, P, 8, None, 8, 0, P, 1 << 20) == INVALID
    # general strides: every stride >= 1, widths <= 64, C present, operands when n > 0
    for strides in ((0, 1, 1, 8), (1, 0, 1, 8), (8, 1, -1, 1), (8, 1, 1, 0)):
        assert lib.tsm_gemm_tn_strided_f64(None, 10, 8, 8, P, strides[0], strides[1], P, strides[2], strides[3],
                                           P, 8, 0, P, 1 << 20) == INVALID
    assert lib.tsm_gemm_tn_strided_f64(None, 10, 8, 80, P, 1, 10, P, 1, 10, P, 80, 0, P, 1 << 20) == INVALID
    assert lib.tsm_gemm_tn_strided_f64(None, 10, 8, 8, None, 1, 10, P, 1, 10, P, 8, 0, P, 1 << 20) == INVALID
    # TF32 split: widths <= 32, contiguous 16-byte aligned operands
    assert lib.tsm_gemm_tn_f32_split(None, 10, 33, 8, P, 33, P, 8, P, 8, 0, P, 1 << 20) == INVALID
    assert lib.tsm_gemm_tn_f32_split(None, 10, 8, 8, P, 12, P, 8, P, 8, 0, P, 1 << 20) == UNSUPPORTED
    assert lib.tsm_gemm_tn_f32_split(None, 10, 8, 8, Q, 8, P, 8, P, 8, 0, P, 1 << 20) == UNSUPPORTED
    # BF16 split: 2 or 3 parts, widths multiples of 4, contiguous, aligned, rows below the tensor-map limit
    for parts in (0, 1, 4):
        assert lib.tsm_gemm_tn_f32_split_bf16(None, 10, 8, 8, P, 8, P, 8, P, 8, 0, parts, P, 1 << 20) == INVALID
    assert lib.tsm_gemm_tn_f32_split_bf16(None, 10, 5, 8, P, 5, P, 8, P, 8, 0, 3, P, 1 << 20) == UNSUPPORTED
    assert lib.tsm_gemm_tn_f32_split_bf16(None, 10, 8, 8, P, 16, P, 8, P, 8, 0, 3, P, 1 << 20) == UNSUPPORTED
    assert lib.tsm_gemm_tn_f32_split_bf16(None, 10, 8, 8, Q, 8, P, 8, P, 8, 0, 3, P, 1 << 20) == UNSUPPORTED
    assert lib.tsm_gemm_tn_f32_split_bf16(None, big, 8, 8, P, 8, P, 8, P, 8, 0, 2, P, 1 << 20) == UNSUPPORTED
    # FP32 storage, Gram, allocation-free: the same shape checks as FP64
    assert lib.tsm_gemm_tn_f32(None, 10, 8, 65, P, 8, P, 65, P, 65, 0, P, 1 << 20) == INVALID
    assert lib.tsm_gemm_tn_f32(None, -1, 8, 8, P, 8, P, 8, P, 8, 0, P, 1 << 20) == INVALID
    assert lib.tsm_gram_f64(None, 10, 8, P, 7, P, 8, 0, P, 1 << 20) == INVALID
    assert lib.tsm_gram_f64(None, 10, 8, None, 8, P, 8, 0, P, 1 << 20) == INVALID
    assert lib.tsm_gemm_tn_f64_noalloc(None, 10, 8, 8, P, 8, P, 8, P, 7, 0) == INVALID
    assert lib.tsm_gemm_tn_f64_noalloc(None, 10, 8, 8, P, 8, None, 8, P, 8, 0) == INVALID
    # TSMM Y = X W: workspace first, then widths, pitches and pointers
    assert lib.tsm_tsmm_f64(None, 10, 8, 8, P, 8, P, 8, 1, P, 8, 0, None, 0) == WORKSPACE
    assert lib.tsm_tsmm_f64(None, 10, 8, 8, P, 8, P, 8, 1, P, 8, 0, Q, 1 << 20) == WORKSPACE
    assert lib.tsm_tsmm_f64(None, 10, 65, 8, P, 65, P, 8, 1, P, 8, 0, P, 1 << 20) == INVALID
    assert lib.tsm_tsmm_f64(None, 10, 8, 8, P, 4, P, 8, 1, P, 8, 0, P, 1 << 20) == INVALID
    assert lib.tsm_tsmm_f64(None, 10, 8, 8, P, 8, None, 8, 1, P, 8, 0, P, 1 << 20) == INVALID
    assert lib.tsm_tsmm_f64(None, 10, 8, 8, P, 8, P, 8, 1, None, 8, 0, P, 1 << 20) == INVALID
    # backward: dC required, widths <= 64; with neither gradient asked for it does nothing
    assert lib.tsm_gemm_tn_backward_f64(None, 10, 8, 8, P, 8, P, 8, None, 8, P, 8, P, 8, 0, P, 1 << 20) == INVALID
    assert lib.tsm_gemm_tn_backward_f64(None, 10, 8, 65, P, 8, P, 65, P, 65, P, 8, P, 65, 0, P, 1 << 20) == INVALID
    assert lib.tsm_gemm_tn_backward_f64(None, 10, 8, 8, P, 8, P, 8, P, 8, None, 8, None, 8, 0, P, 1 << 20) == 0
    # block orthogonalisation: B is written, so it must be present
    assert lib.tsm_block_orth_f64(None, 10, 8, 8, P, 8, None, 8, P, 8, P, 1 << 20) == INVALID
    # batched: no plan, or a plan that was never initialised
    assert lib.tsm_gemm_tn_batched_f64(None, None) == INVALID
    assert lib.tsm_gemm_tn_batched_f64(None, ctypes.byref(_capi.BatchedPlan())) == INVALID
    assert lib.tsm_batched_plan_init_f64(None, 1, None, P, 1 << 20, None) == INVALID
    # self-test and fill: workspace and count checks
    assert lib.tsm_selftest_wait_timeout(None, None, 0, 1000) == WORKSPACE
    assert lib.tsm_fill_uniform_f64(None, P, -1, 1, 0) == INVALID
    assert lib.tsm_fill_uniform_f64(None, P, 0, 1, 0) == 0
