"""The reference's own drivers, compiled unmodified against this library
(tsm_benchmark_b200/compat/Makefile builds them where the reference sources
exist), run on the GPU: every kernel they check must be correct."""
import os
import re
import subprocess

import pytest

from tests.conftest import ROOT

pytestmark = pytest.mark.gpu

BUILD = os.path.join(ROOT, "tsm_benchmark_b200", "compat", "_build")


def run(binary):
    path = os.path.join(BUILD, binary)
    if not os.path.exists(path):
        pytest.skip(f"{binary} not built (needs the reference sources at build time)")
    r = subprocess.run([path], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


def test_main_cc_dropin(gpu):
    """main.cc: 18 (M, stride, tile) suites; its correctness check (against
    its own compute_naive, rel 1e-6 / abs 1e-10) must pass for tsmttsm4, 6
    and 9 in each, and every one must then be timed."""
    out = run("main_dropin")
    checks = re.findall(r"Variant [469]: (true|false)", out)
    assert len(checks) == 54 and all(c == "true" for c in checks), out[-3000:]
    timed = re.findall(r"Variant [469]: [0-9.]+ ms", out)
    assert len(timed) == 54
    assert "NVIDIA" in out


def test_main_codegen_dropin(gpu):
    """main_codegen.cc with the generated tsmttsm_kernels.hh: every kernel
    PASSes the generated harness's check (all K rows)."""
    out = run("main_codegen_dropin")
    rows = re.findall(r"^\s*(M\d+_T\d+_\w+)\s+(PASS|FAIL)", out, flags=re.M)
    assert len(rows) == 24, out[-3000:]  # 3 widths x 2 tiles x 4 names
    assert all(s == "PASS" for _, s in rows), out[-3000:]
