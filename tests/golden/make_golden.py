#!/usr/bin/env python3
"""Writes the golden fixtures in tests/golden/ from the reference's own code.

Run here, where the reference sources exist (oracle/Makefile builds
oracle/_ref/libtsm_ref.so from them in place):

    make -C oracle && python tests/golden/make_golden.py

The reference ships no golden vectors, known-answer tests or fixtures, so
these are outputs of its own functions run on the host:

  ref_square_cases.npz   compute_naive (main.cc:14-27) on seeded SplitMix64
                         inputs for square widths 1..64 and ragged n;
  ref_config0.npz        the first benchmark configuration: n = 2^20, M = 8,
                         inputs drawn exactly as main.cc:71-86 draws them
                         (one std::minstd_rand0(123)), C from compute_naive
                         and from tsmttsm4 / tsmttsm6 / tsmttsm9 with
                         main.cc's launch shape (stride 16384, local size
                         32, tile 4), plus input samples;
  ref_variants.npz       all nine tsmttsm.hh variants and the kernels the
                         two generators emit by default, M = 8, n = 4099;
  ref_codegen.json       the generators' command lines (sycl_codegen.py,
                         sycl_codegen_new.py run as scripts) on a few flag
                         sets: exit code, kernel names, stride.

The inputs are not stored: tests regenerate them with the oracle's
generators (pinned to the reference's by tests/test_oracle.py).

Re-running the script reproduces every compute_naive output bit for bit.
The kernel outputs are reproduced only to rounding: the reference kernels
add into C with FP64 atomics, whose order depends on the host's thread
count and scheduling (a re-run on 8 threads against fixtures made on 16
moved entries of magnitude 46-849 by at most 3.7e-12).  The tests therefore
hold kernel outputs to the reference's is_correct rule and the normwise
bound, and compute_naive outputs to exact equality.
"""
from __future__ import annotations

import ctypes
import json
import os
import re
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

SQUARE_CASES = [  # (n, M, seed)
    (1, 1, 11), (2, 2, 12), (3, 4, 13), (17, 8, 14), (1000, 16, 15), (4099, 8, 16),
    (4097, 32, 17), (2049, 64, 18), (65536, 4, 19), (100003, 1, 20), (31, 64, 21), (8192, 16, 22),
]

# Command lines run through both reference generators (ref_codegen.json).
CODEGEN_FLAG_SETS = [
    [],
    ["--with-benchmark"],
    ["--M", "4", "8", "16", "32", "64", "--tile-sizes", "2", "4", "8", "--with-benchmark"],
    ["--M", "12", "48", "--tile-sizes", "3", "4", "6"],
    ["--M", "8", "--stride", "1000"],
    ["--M", "12", "--stride", "4096"],
    ["--M", "16", "--local-size", "128", "--unroll", "2"],
]

MAIN_CC_SHAPE = dict(n=1 << 20, M=8, stride=16384, tile=4)
VARIANTS_SHAPE = dict(n=4099, M=8, seed=7)


def p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def ref_naive(R, A, B):
    n, M = A.shape
    C = np.zeros(M * M)
    assert R.ref_compute_naive_f64(n, M, p(A), p(B), p(C)) == 0
    return C.reshape(M, M)


def main() -> int:
    oracle.build()
    R = oracle.ref()
    if R is None:
        print("oracle/_ref/libtsm_ref.so is not built (reference sources absent?)", file=sys.stderr)
        return 1
    meta = {"generator": "tests/golden/make_golden.py", "reference": "nilsfriess/tsm_benchmark"}

    # 1. compute_naive on square cases.
    sq = {}
    for n, M, seed in SQUARE_CASES:
        A, B = oracle.operands(n, M, M, seed)
        sq[f"n{n}_M{M}_s{seed}"] = ref_naive(R, np.ascontiguousarray(A), np.ascontiguousarray(B))
    np.savez_compressed(os.path.join(OUT, "ref_square_cases.npz"), **sq)
    meta["square_cases"] = SQUARE_CASES

    # 2. The first benchmark configuration with main.cc's own inputs.
    n, M = MAIN_CC_SHAPE["n"], MAIN_CC_SHAPE["M"]
    A = np.empty(n * M)
    B = np.empty(n * M)
    R.ref_fill_main_cc_f64(p(A), p(B), n * M, 123)
    A = A.reshape(n, M)
    B = B.reshape(n, M)
    out = {"C_naive": ref_naive(R, A, B)}
    for v in (4, 6, 9):
        C = np.zeros(M * M)
        ns = ctypes.c_uint64()
        rc = R.ref_tsmttsm_f64(v, M, MAIN_CC_SHAPE["stride"], MAIN_CC_SHAPE["tile"], n, p(A), p(B), p(C),
                               ctypes.byref(ns))
        assert rc == 0, (v, rc)
        out[f"C_v{v}"] = C.reshape(M, M)
        out[f"is_correct_v{v}"] = np.array(R.ref_is_correct_f64(p(out["C_naive"]), p(C), M, 1e-6, 1e-10))
    out["A_head"], out["B_head"] = A[:4].copy(), B[:4].copy()
    out["A_tail"], out["B_tail"] = A[-4:].copy(), B[-4:].copy()
    np.savez_compressed(os.path.join(OUT, "ref_config0.npz"), **out)
    meta["config0"] = MAIN_CC_SHAPE

    # 3. Every reference kernel on one small case.
    n, M, seed = VARIANTS_SHAPE["n"], VARIANTS_SHAPE["M"], VARIANTS_SHAPE["seed"]
    A, B = oracle.operands(n, M, M, seed)
    A = np.ascontiguousarray(A)
    B = np.ascontiguousarray(B)
    var = {"C_naive": ref_naive(R, A, B)}
    for v in range(1, 10):
        C = np.zeros(M * M)
        assert R.ref_tsmttsm_f64(v, M, 4096, 4, n, p(A), p(B), p(C), None) == 0
        var[f"tsmttsm{'' if v == 1 else v}"] = C.reshape(M, M)
    for name in ("tsmttsm_8_8_4_4", "tsmttsm_8_8_4_4_lf", "tsmttsm_8_8_4_4_sg", "tsmttsm_8_8_4_4_sg_lf",
                 "tsmttsm_8_8_2_2_sg", "tsmttsm_gen_8_8_4_4_tr", "tsmttsm_gen_8_8_4_4_lf_tr",
                 "tsmttsm_gen_8_8_4_4_2l_tr", "tsmttsm_gen_8_8_4_4_lf_2l_tr"):
        C = np.zeros(M * M)
        assert R.ref_generated_f64(name.encode(), n, p(A), p(B), p(C), None) == 0, name
        var[name] = C.reshape(M, M)
    np.savez_compressed(os.path.join(OUT, "ref_variants.npz"), **var)
    meta["variants"] = VARIANTS_SHAPE

    # 4. The generators' command lines (sycl_codegen.py, sycl_codegen_new.py
    #    run as scripts): for each flag set, the exit code, the kernel names
    #    in order, the stride the v2 script prints, and whether run_all_benchmarks
    #    is emitted.
    codegen = []
    for style, script in (("v2", "sycl_codegen_new.py"), ("v1", "sycl_codegen.py")):
        for flags in CODEGEN_FLAG_SETS:
            r = subprocess.run([sys.executable, os.path.join(oracle.reference_dir(), script), *flags],
                               capture_output=True, text=True)
            names = re.findall(r"sycl::event (tsmttsm_[0-9a-z_]+)\(", r.stdout)
            m = re.search(r"stride=(\d+)\s+local_size=(\d+)", r.stdout)
            codegen.append({"style": style, "flags": flags, "rc": r.returncode, "names": names,
                            "stride": int(m.group(1)) if m else None,
                            "benchmark": "run_all_benchmarks" in r.stdout})
    with open(os.path.join(OUT, "ref_codegen.json"), "w") as f:
        json.dump(codegen, f, indent=0)
        f.write("\n")

    with open(os.path.join(OUT, "golden_meta.json"), "w") as f:
        json.dump(meta, f, indent=1)
        f.write("\n")
    print("wrote", sorted(os.listdir(OUT)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
