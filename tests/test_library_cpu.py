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
    # per-class paths: -1 (tuned), 0 (tensor cores), 1 (SIMT); others refused before any CUDA call
    plan = _capi.BatchedPlan()
    probs = (_capi.BatchedProblem * 1)()
    for bad in (2, -2, 7):
        paths = (ctypes.c_int * 16)(*([-1] * 16))
        paths[10] = bad
        assert lib.tsm_batched_plan_init_paths_f64(None, 1, probs, paths, P, 1 << 20, ctypes.byref(plan)) == INVALID
    assert lib.tsm_batched_plan_init_paths_f64(None, 0, probs, None, P, 1 << 20, ctypes.byref(plan)) == INVALID
    # self-test and fill: workspace and count checks
    assert lib.tsm_selftest_wait_timeout(None, None, 0, 1000) == WORKSPACE
    assert lib.tsm_fill_uniform_f64(None, P, -1, 1, 0) == INVALID
    assert lib.tsm_fill_uniform_f64(None, P, 0, 1, 0) == 0


def test_generator_command_line_matches_the_reference_generators():
    """`python -m tsm_benchmark_b200.codegen` with the reference generators'
    flags (--M, --tile-sizes, --stride, --local-size, --unroll,
    --with-benchmark; --style v1 for sycl_codegen.py's names) against the
    reference scripts' own output on the same flag sets
    (tests/golden/ref_codegen.json): same exit status, same kernel names in
    the same order, the same automatic stride, run_all_benchmarks exactly
    when asked for."""
    import contextlib
    import io
    import json
    import re

    from tests.conftest import GOLDEN
    from tsm_benchmark_b200 import codegen
    with open(os.path.join(GOLDEN, "ref_codegen.json")) as f:
        cases = json.load(f)
    assert len(cases) >= 14
    for case in cases:
        out, err = io.StringIO(), io.StringIO()
        with contextlib.redirect_stdout(out), contextlib.redirect_stderr(err):
            rc = codegen.main(["--style", case["style"], *case["flags"]])
        what = (case["style"], case["flags"])
        assert (rc != 0) == (case["rc"] != 0), (what, err.getvalue())
        if rc:
            assert err.getvalue().strip(), what
            continue
        text = out.getvalue()
        assert re.findall(r"sycl::event (tsmttsm_[0-9a-z_]+)\(", text) == case["names"], what
        if case["stride"] is not None:
            assert re.search(r"stride=(\d+)\s+local_size", text).group(1) == str(case["stride"]), what
        assert ("run_all_benchmarks" in text) == case["benchmark"], what


def test_generated_kernels_name_compiled_variants():
    """Every kernel of a generated header runs a variant the library has, and
    the four names of a (M, TM) pair run distinct kernels wherever the
    library compiles distinct ring depths for that tile."""
    import re

    from tsm_benchmark_b200 import codegen
    vs = codegen.default_variants()
    names = {v.name for v in vs}
    text = codegen.render_dropin_header(vs, widths=(4, 8, 16, 32, 64), tiles=(2, 4, 8))
    picked = re.findall(r'variant_by_name\("([^"]+)"\)', text)
    assert picked and set(picked) <= names
    # 8 x 8 with 4 x 4 tiles: deepest ring, double buffer, tuned default, middle ring
    kinds = [codegen.pick_dropin_variant(vs, 8, 4, lf, sg)[0] for lf, sg in
             ((False, False), (True, False), (False, True), (True, True))]
    assert kinds[2] is None and len({kinds[0], kinds[1], kinds[3]}) == 3
    # widths 16..64: the prefetching reduction-optimised name runs the FP64 tensor cores, on a
    # kernel that is not one of the tuned choices the plain reduction-optimised name runs
    tuned = codegen.load_tuned()
    for m in (16, 32, 64):
        name = codegen.pick_dropin_variant(vs, m, 4, True, True)[0]
        assert name.startswith("dmma_")
        tuned_m = {t[3] for t in tuned if (t[0], t[1]) == (m, m)}
        rings = {v.name for v in vs if isinstance(v, codegen.DmmaVariant) and not v.gram and (v.wa, v.wb) == (m, m)}
        assert name not in tuned_m or rings <= tuned_m  # else every compiled ring is a tuned choice
    fake = [(16, 16, 0, "dmma_16x16_t16x16_w8_s2_r384")]
    pick = codegen.pick_dropin_variant(vs, 16, 4, True, True, tuned=fake)[0]
    others = [v.resolved() for v in vs if isinstance(v, codegen.DmmaVariant) and not v.gram and (v.wa, v.wb) == (16, 16)
              and v.name != fake[0][3]]
    assert pick != fake[0][3] and pick in {v.name for v in others if v.stages == min(o.stages for o in others)}
    # the CTA cap is stride / local_size work-groups
    assert "K, 8, 8, A, B, C, variant, 2048);" in codegen.render_dropin_header(vs, widths=(8,), tiles=(4,))
