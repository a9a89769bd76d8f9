"""The reference's own drivers, compiled unmodified against this library
(tsm_benchmark_b200/compat/Makefile builds them where the reference sources
exist), run on the GPU: every kernel they check must be correct."""
import os
import re
import subprocess

import numpy as np
import pytest

from tests.conftest import GOLDEN, ROOT

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


@pytest.mark.parametrize("binary,labels", [("main_codegen_wide_dropin", ("basic", "lf", "sg", "sg_lf")),
                                           ("main_codegen_v1_dropin", ("basic", "leapfrog", "2level", "all"))])
def test_main_codegen_with_generated_wide_header(gpu, binary, labels):
    """main_codegen.cc against a header the generator wrote from the
    reference generators' command line, --M 4 8 16 32 64 --tile-sizes 2 4 8
    --with-benchmark, in the v2 (sycl_codegen_new.py) and v1
    (sycl_codegen.py) spellings: 14 (M, TM) pairs x 4 kernels, every one
    PASSes its harness's check (rel 1e-6, or 1e-8 for v1)."""
    out = run(binary)
    rows = re.findall(r"^\s*(M(\d+)_T(\d+)_(\w+))\s+(PASS|FAIL)", out, flags=re.M)
    assert len(rows) == 56, out[-3000:]
    assert all(s == "PASS" for *_, s in rows), [r for r in rows if r[-1] != "PASS"]
    pairs = {(int(m), int(t)) for _, m, t, _, _ in rows}
    assert pairs == {(m, t) for m in (4, 8, 16, 32, 64) for t in (2, 4, 8) if m % t == 0}
    assert {lab for *_, lab, _ in rows} == set(labels)


def test_compat_templates_match_reference_outputs(gpu, oracle_mod):
    """All nine tsmttsm.hh templates (tsmttsm8 with its default worker_mult)
    and the generators' default kernel names for M = 8, instantiated from the
    compat headers, against the reference's own outputs on the same inputs
    (tests/golden/ref_variants.npz: n = 4099, M = 8, seed 7): the reference's
    is_correct rule against each kernel's recorded C and against its
    compute_naive, and the normwise bound."""
    out = run("compat_templates")
    got = {}
    for line in out.splitlines():
        parts = line.split()
        if parts:
            got[parts[0]] = np.array([float(x) for x in parts[1:]]).reshape(8, 8)
    g = np.load(os.path.join(GOLDEN, "ref_variants.npz"))
    names = ["tsmttsm"] + [f"tsmttsm{v}" for v in range(2, 10)]
    names += [f"tsmttsm_8_8_{t}_{t}{s}" for t in (2, 4) for s in ("", "_lf", "_sg", "_sg_lf")]
    names += [f"tsmttsm_gen_8_8_4_4{s}" for s in ("_tr", "_lf_tr", "_2l_tr", "_lf_2l_tr")]
    assert set(names) <= set(got), set(names) - set(got)
    A, B = oracle_mod.operands(4099, 8, 8, 7)
    for name in names:
        assert oracle_mod.check(g["C_naive"], got[name], 1e-6, 1e-10) == -1, name
        nw = oracle_mod.normwise(A, B, g["C_naive"], got[name])
        assert nw["err"] <= nw["bound"], (name, nw)
        if name in g:  # the reference kernel of the same name, run on the host
            assert oracle_mod.check(g[name], got[name], 1e-6, 1e-10) == -1, name


def test_main_codegen_with_generated_odd_widths(gpu):
    """main_codegen.cc against a header generated for widths that are not
    powers of two, --M 12 24 48 --tile-sizes 3 4 6 (capacity kernels,
    tiles with no compiled match, the 48-wide tensor-core kernel): every one
    of the 9 (M, TM) pairs x 4 kernels PASSes."""
    out = run("main_codegen_odd_dropin")
    rows = re.findall(r"^\s*(M(\d+)_T(\d+)_(\w+))\s+(PASS|FAIL)", out, flags=re.M)
    pairs = {(int(m), int(t)) for _, m, t, _, _ in rows}
    assert pairs == {(m, t) for m in (12, 24, 48) for t in (3, 4, 6) if m % t == 0}, pairs
    assert len(rows) == 4 * len(pairs)
    assert all(s == "PASS" for *_, s in rows), [r for r in rows if r[-1] != "PASS"]
