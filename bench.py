#!/usr/bin/env python3
"""Benchmark: plain FP64 TSMTTSM (C = A^T B) on B200, one JSON line.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the width sweep (A, B row-major, uniform[-1, 1) from a fixed seed),
headline shape n = 2^26 rows, m = k = 8 columns; ``by_width`` reports every
shape of the sweep (square widths 1..64 at n = 2^26, 2^23 for 64, and
(4,32), (32,4), (1,64)).  A step is one call of ``tsm_gemm_tn_f64`` over the
whole headline input (8 GiB, larger than L2, so no flush is needed).

* ``value``: GB/s of algorithmic bytes 8 n (m + k) + 8 m k per step, with the
  inputs resident in HBM; for N > 1 (torchrun) each rank holds its own 2^26
  rows (weak scaling), ends each step with the deterministic cross-rank
  reduction of its partial C, and value = all rows' bytes / max-over-ranks time.
* ``e2e``: the same metric through the C ABI from pinned HOST buffers (H2D of A
  and B, the call, D2H of C inside the timed region).
* ``roofline``: the dominant kernel against the measured HBM copy bandwidth.
* ``cpu_baseline``: the reference's own tsmttsm4 (tsmttsm.hh:125-166, main.cc's
  launch shape) run on the host cores through the oracle's host SYCL subset,
  on a bounded sample of the same workload.

``--impl reference`` times that CPU implementation alone as the reference arm.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "TSMTTSM GB/s (% of HBM peak) by width; fast-form speedup vs FP64 at stated err"
HEAD_N, HEAD_M, HEAD_K = 1 << 26, 8, 8
SWEEP = [(1 << 26, 1, 1), (1 << 26, 2, 2), (1 << 26, 4, 4), (1 << 26, 8, 8), (1 << 26, 16, 16),
         (1 << 26, 32, 32), (1 << 23, 64, 64), (1 << 26, 4, 32), (1 << 26, 32, 4), (1 << 26, 1, 64)]
SEED = 123
REF_STRIDE, REF_TILE = 16384, 4  # main.cc:183 launch shape for M = 8


def algo_bytes(n: int, m: int, k: int) -> int:
    return 8 * n * (m + k) + 8 * m * k


def load_peaks() -> dict:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured (MEASURED_PEAKS.json)"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def profile_traffic(kernel_tag: str):
    """DRAM bytes per launch from the committed ncu summary, if present."""
    for name in sorted(os.listdir(os.path.join(ROOT, "profiles"))) if os.path.isdir(os.path.join(ROOT, "profiles")) else []:
        if kernel_tag not in name:
            continue
        with open(os.path.join(ROOT, "profiles", name)) as f:
            for line in f:
                if line.strip().startswith("traffic_bytes_per_launch"):
                    try:
                        return int(float(line.split("=")[1].split()[0]))
                    except (ValueError, IndexError):
                        return None
    return None


# --------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.1)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
                power.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[4:8]):
                if val.lower() in ("active", "1"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "power_w_max": max(power) if power else None, "samples": len(sm), "reasons": sorted(reasons)}


# ------------------------------------------------------------- reference arm
def reference_cpu(n_sample: int, steps: int, warmup: int, budget_s: float) -> dict:
    """The reference's tsmttsm4<double, 8, 16384, 4> on host threads (kind
    "reference"), or the oracle's OpenMP restatement (kind "port") when
    oracle/_ref was not built.  Returns GB/s over `steps` timed runs."""
    from oracle import oracle
    R = oracle.ref()
    A, B = oracle.operands(n_sample, HEAD_M, HEAD_K, SEED)
    C = __import__("numpy").zeros(HEAD_M * HEAD_K)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    if R is not None:
        kind, cores = "reference", R.ref_num_threads()

        def run():
            C[:] = 0
            ns = ctypes.c_uint64()
            rc = R.ref_tsmttsm_f64(4, HEAD_M, REF_STRIDE, REF_TILE, n_sample, p(A), p(B), p(C), ctypes.byref(ns))
            if rc != 0:
                raise RuntimeError(f"reference kernel refused the shape ({rc})")
            return ns.value * 1e-9
    else:
        kind, cores = "port", oracle.lib().tsm_oracle_num_threads()

        def run():
            t0 = time.perf_counter()
            oracle.v4_port(A, B, REF_STRIDE, REF_TILE)
            return time.perf_counter() - t0
    for _ in range(warmup):
        run()
    times = []
    t_start = time.perf_counter()
    for _ in range(steps):
        times.append(run())
        if time.perf_counter() - t_start > budget_s and len(times) >= 1:
            break
    t = sum(times) / len(times)
    gbs = algo_bytes(n_sample, HEAD_M, HEAD_K) / t / 1e9
    # The reference's own FP64 oracle, compute_naive (main.cc:14-27), one
    # thread, on the first 2^20 rows (one run).
    naive = None
    if R is not None:
        nn = min(n_sample, 1 << 20)
        Cn = __import__("numpy").zeros(HEAD_M * HEAD_K)
        t0 = time.perf_counter()
        R.ref_compute_naive_f64(nn, HEAD_M, p(A), p(B), p(Cn))
        tn = time.perf_counter() - t0
        naive = {"value": algo_bytes(nn, HEAD_M, HEAD_K) / tn / 1e9, "unit": "GB/s", "cores": 1,
                 "sample": f"compute_naive, n={nn} rows x m=k=8, one run of {tn * 1e3:.1f} ms"}
    return {"value": gbs, "unit": "GB/s", "cores": cores, "kind": kind, "steps_timed": len(times),
            "sample": (f"n={n_sample} rows x m=k=8 ("
                       + ("the headline shape, all of its rows" if n_sample == HEAD_N
                          else f"the headline shape at {n_sample / HEAD_N:.4g} of its rows") + "), "
                       f"tsmttsm4 stride {REF_STRIDE} tile {REF_TILE}, mean of {len(times)} runs "
                       f"of {t * 1e3:.1f} ms"),
            "naive_single_core": naive}


def run_reference_arm(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n_sample = args.ref_rows
    res = reference_cpu(n_sample, args.steps, args.warmup, budget_s=args.ref_budget)
    line = {"metric": METRIC, "impl": "reference", "value": res["value"], "unit": "GB/s",
            "n_gpus": args.gpus, "steps": res["steps_timed"], "warmup": args.warmup,
            "ms_per_step": algo_bytes(n_sample, HEAD_M, HEAD_K) / res["value"] / 1e6,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload_config(args.gpus),
            "cpu_baseline": {k: res[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": res["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def workload_config(n_gpus: int) -> dict:
    return {"workload": "plain FP64 TSMTTSM C=A^T B, width sweep; headline n=2^26 rows x m=k=8 per GPU",
            "n": HEAD_N, "m": HEAD_M, "k": HEAD_K, "inputs": "uniform[-1,1) SplitMix64 seed 123, row-major",
            "l2": "inputs (8 GiB) larger than L2, no flush", "parallelism": f"rows sharded, {n_gpus} GPU(s)"}


# -------------------------------------------------------------- the forms
def _time(fn, reps: int, warmup: int = 3) -> float:
    """Milliseconds per call, CUDA events on the current stream."""
    import torch
    for _ in range(warmup):
        fn()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def fp64_gemm_peak(dev) -> dict:
    """FP64 compute roof for the wide shapes: cuBLAS DGEMM (torch.matmul,
    8192^3, 2 N^3 flops), best of 5 after one warm-up, CUDA events."""
    import torch
    n = 8192
    a = torch.rand((n, n), dtype=torch.float64, device=dev)
    b = torch.rand((n, n), dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    best = None
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    del a, b
    torch.cuda.empty_cache()
    return {"tflops": round(2.0 * n**3 / (best * 1e-3) / 1e12, 2), "source": "cuBLAS DGEMM 8192^3 in this run"}


def forms(dev) -> dict:
    """The forms beside the plain FP64 path, each against FP64 on the same
    GPU: split precision (n = 2^25, m = k = 32, FP32 storage, column scaled
    normal data; TF32 hi/lo, BF16 hi/lo and BF16 hi/mid/lo parts), batched (512 problems, one launch under a CUDA graph vs one
    plain launch per problem), the Gram product C = A^T A (vs the
    two-operand call on a copy of A), column-major operands (vs the
    row-major call on the same values) and differentiation (n = 2^22,
    m = k = 16: fused backward vs forward time, FP64 and FP32)."""
    import numpy as np
    import torch

    import tsm_benchmark_b200 as tsm
    out = {}

    # --- precision: TF32 hi/lo split on tcgen05 vs plain FP64 on FP64 copies
    n, w = 1 << 25, 32
    g = torch.Generator(device=dev).manual_seed(3)
    sa = 10.0 ** (torch.rand(w, device=dev, generator=g) * 6 - 3)
    sb = 10.0 ** (torch.rand(w, device=dev, generator=g) * 6 - 3)
    A32 = (torch.randn((n, w), device=dev, generator=g) * sa).float()
    B32 = (torch.randn((n, w), device=dev, generator=g) * sb).float()
    A64, B64 = A32.double(), B32.double()
    C_split = torch.empty((w, w), dtype=torch.float64, device=dev)
    C_ref = torch.empty((w, w), dtype=torch.float64, device=dev)
    ms_split = _time(lambda: tsm.tsmttsm_split(A32, B32, C_split), 20)
    ms_f64 = _time(lambda: tsm.tsmttsm(A64, B64, C_ref), 20)
    # Sustained: 300 calls, long enough for the power cap to set the clock.
    ms_f64_sus = _time(lambda: tsm.tsmttsm(A64, B64, C_ref), 300)
    ms_split_sus = _time(lambda: tsm.tsmttsm_split(A32, B32, C_split), 300)
    scale = tsm.tsmttsm(A64.abs(), B64.abs())
    nw = float(torch.linalg.norm(C_split - C_ref) / torch.linalg.norm(C_ref))
    pe = float(((C_split - C_ref).abs() / scale).max())
    out["split_tf32"] = {"n": n, "m": w, "k": w, "ms": round(ms_split, 4), "fp64_ms": round(ms_f64, 4),
                         "speedup_vs_fp64": round(ms_f64 / ms_split, 3),
                         "GB/s": round(4 * n * 2 * w / (ms_split * 1e-3) / 1e9, 1),
                         "err_normwise_rel": nw, "err_entry_max_rel": pe, "stated_err": 1e-6,
                         "meets_stated_err": bool(nw <= 1e-6 and pe <= 1e-6),
                         "sustained_300_calls": {"ms": round(ms_split_sus, 4), "fp64_ms": round(ms_f64_sus, 4),
                                                 "speedup_vs_fp64": round(ms_f64_sus / ms_split_sus, 3)}}
    # the same inputs with BF16 parts: hi/lo (stated error 4e-5 per entry, above
    # the 1e-6 target by design) and hi/mid/lo
    for kind, stated in (("bf16x2", 4e-5), ("bf16x3", 1e-6)):
        ms_k = _time(lambda: tsm.tsmttsm_split(A32, B32, C_split, kind=kind), 20)
        ms_k_sus = _time(lambda: tsm.tsmttsm_split(A32, B32, C_split, kind=kind), 300)
        nwk = float(torch.linalg.norm(C_split - C_ref) / torch.linalg.norm(C_ref))
        pek = float(((C_split - C_ref).abs() / scale).max())
        out[f"split_{kind}"] = {"n": n, "m": w, "k": w, "ms": round(ms_k, 4), "fp64_ms": round(ms_f64, 4),
                                "speedup_vs_fp64": round(ms_f64 / ms_k, 3),
                                "GB/s": round(4 * n * 2 * w / (ms_k * 1e-3) / 1e9, 1),
                                "err_normwise_rel": nwk, "err_entry_max_rel": pek, "stated_err": stated,
                                "meets_stated_err": bool(nwk <= stated and pek <= stated),
                                "meets_1e-6": bool(nwk <= 1e-6 and pek <= 1e-6),
                                "sustained_300_calls": {"ms": round(ms_k_sus, 4), "fp64_ms": round(ms_f64_sus, 4),
                                                        "speedup_vs_fp64": round(ms_f64_sus / ms_k_sus, 3)}}
    del A32, B32, A64, B64, scale
    torch.cuda.empty_cache()

    # --- batching: one persistent launch (graph replay) vs one launch per problem
    rng = np.random.default_rng(5)
    ns = np.exp(rng.uniform(np.log(1e3), np.log(1e6), size=512)).astype(np.int64)
    ms_ = rng.choice((4, 8, 16, 32), size=512)
    ks_ = rng.choice((4, 8, 16, 32), size=512)
    As, Bs = [], []
    for i, (nn, mm, kk) in enumerate(zip(ns, ms_, ks_)):
        a = torch.empty((int(nn), int(mm)), dtype=torch.float64, device=dev)
        b = torch.empty((int(nn), int(kk)), dtype=torch.float64, device=dev)
        tsm.fill_uniform(a, 1000 + i, 0)
        tsm.fill_uniform(b, 1000 + i, 1)
        As.append(a)
        Bs.append(b)
    bt = tsm.BatchedTSMTTSM(As, Bs)
    graph = bt.capture_graph()
    ms_batched = _time(graph.replay, 20)
    Cp = [torch.empty((a.shape[1], b.shape[1]), dtype=torch.float64, device=dev) for a, b in zip(As, Bs)]
    lib = __import__("tsm_benchmark_b200._capi", fromlist=["load"]).load()
    sh = int(torch.cuda.current_stream(dev).cuda_stream)
    wsb = torch.zeros(lib.tsm_gemm_tn_workspace_size(1, 32, 32), dtype=torch.uint8, device=dev)

    def plain_all():
        for a, b, c in zip(As, Bs, Cp):
            lib.tsm_gemm_tn_f64(sh, a.shape[0], a.shape[1], b.shape[1], a.data_ptr(), a.shape[1], b.data_ptr(),
                                b.shape[1], c.data_ptr(), b.shape[1], 0, wsb.data_ptr(), wsb.numel())
    ms_plain = _time(plain_all, 5, warmup=1)
    err = max(float(torch.linalg.norm(c - p) / max(float(torch.linalg.norm(p)), 1e-300)) for c, p in zip(bt.Cs, Cp))
    total_bytes = int(sum(8 * a.shape[0] * (a.shape[1] + b.shape[1]) for a, b in zip(As, Bs)))
    out["batched"] = {"problems": 512, "bytes": total_bytes, "segments": bt.segments, "ms": round(ms_batched, 4),
                      "plain_launches_ms": round(ms_plain, 4), "speedup_vs_fp64_plain": round(ms_plain / ms_batched, 3),
                      "GB/s": round(total_bytes / (ms_batched * 1e-3) / 1e9, 1),
                      "err_vs_plain_max_rel": err, "launches": 1, "cuda_graph": True}
    del As, Bs, bt, graph, Cp
    torch.cuda.empty_cache()

    # --- Gram C = A^T A (A streamed once, upper triangle) vs the two-operand
    #     call on a copy of A
    rows = []
    for gm, gn in ((8, 1 << 26), (16, 1 << 26), (32, 1 << 26), (64, 1 << 23)):
        A = torch.empty((gn, gm), dtype=torch.float64, device=dev)
        tsm.fill_uniform(A, 77, 0)
        A2 = A.clone()
        Cg = torch.empty((gm, gm), dtype=torch.float64, device=dev)
        ms_g = _time(lambda: tsm.gram(A, Cg), 10)
        ms_p = _time(lambda: tsm.tsmttsm(A, A2, Cg), 10)
        sym = bool(torch.equal(tsm.gram(A), tsm.gram(A).T))
        rows.append({"n": gn, "m": gm, "gram_ms": round(ms_g, 4), "two_operand_ms": round(ms_p, 4),
                     "speedup": round(ms_p / ms_g, 3), "GB/s_of_A": round(8 * gn * gm / (ms_g * 1e-3) / 1e9, 1),
                     "symmetric": sym})
        del A, A2
        torch.cuda.empty_cache()
    out["gram"] = rows

    # --- block orthogonalisation B <- B - A (A^T B): C = A^T B, then the TSMM
    #     (two passes: A and B read twice, B written once).  A's columns are
    #     scaled to about unit norm, so repeated steps keep B bounded.
    rows = []
    for om, on in ((8, 1 << 25), (16, 1 << 24), (32, 1 << 23)):
        A = torch.empty((on, om), dtype=torch.float64, device=dev)
        B = torch.empty((on, om), dtype=torch.float64, device=dev)
        tsm.fill_uniform(A, 78, 0)
        tsm.fill_uniform(B, 78, 1)
        A.mul_((3.0 / on) ** 0.5)
        Co = torch.empty((om, om), dtype=torch.float64, device=dev)
        ms_o = _time(lambda: tsm.block_orthogonalize(A, B, Co), 10)
        ms_f = _time(lambda: tsm.tsmttsm(A, B, Co), 10)
        nbytes = 8 * on * (2 * om + 3 * om)
        rows.append({"n": on, "m": om, "k": om, "orth_ms": round(ms_o, 4), "tsmttsm_ms": round(ms_f, 4),
                     "over_tsmttsm": round(ms_o / ms_f, 3), "algorithmic_bytes": nbytes,
                     "GB/s": round(nbytes / (ms_o * 1e-3) / 1e9, 1), "finite": bool(torch.isfinite(B).all())})
        del A, B
        torch.cuda.empty_cache()
    out["block_orth"] = rows

    # --- column-major operands (A^T, B^T stored row-major, through
    #     tsm_gemm_tn_strided_f64) vs the row-major call on the same values
    rows = []
    for cm, ck, cn in ((8, 8, 1 << 26), (4, 32, 1 << 25), (32, 32, 1 << 25), (64, 64, 1 << 23)):
        At = torch.empty((cm, cn), dtype=torch.float64, device=dev)
        Bt = torch.empty((ck, cn), dtype=torch.float64, device=dev)
        tsm.fill_uniform(At, 91, 0)
        tsm.fill_uniform(Bt, 91, 1)
        Ar, Br = At.t().contiguous(), Bt.t().contiguous()
        Cc = torch.empty((cm, ck), dtype=torch.float64, device=dev)
        Cr = torch.empty((cm, ck), dtype=torch.float64, device=dev)
        ms_c = _time(lambda: tsm.tsmttsm(At.t(), Bt.t(), Cc), 10)
        ms_r = _time(lambda: tsm.tsmttsm(Ar, Br, Cr), 10)
        nbytes = 8 * cn * (cm + ck)
        rows.append({"n": cn, "m": cm, "k": ck, "column_major_ms": round(ms_c, 4), "row_major_ms": round(ms_r, 4),
                     "column_major_GB/s": round(nbytes / (ms_c * 1e-3) / 1e9, 1),
                     "row_major_GB/s": round(nbytes / (ms_r * 1e-3) / 1e9, 1),
                     "max_rel_diff": float((Cc - Cr).abs().max() / Cr.abs().max())})
        del At, Bt, Ar, Br
        torch.cuda.empty_cache()
    out["column_major"] = rows

    # --- differentiation: fused backward vs forward
    n, w = 1 << 22, 16
    for dt, name in ((torch.float64, "autograd_f64"), (torch.float32, "autograd_f32")):
        A = (torch.rand((n, w), device=dev, generator=g, dtype=torch.float64) * 2 - 1).to(dt)
        B = (torch.rand((n, w), device=dev, generator=g, dtype=torch.float64) * 2 - 1).to(dt)
        Wl = torch.randn((w, w), device=dev, generator=g, dtype=torch.float64).to(dt)
        C = torch.empty((w, w), dtype=dt, device=dev)
        ms_fwd = _time(lambda: tsm.tsmttsm(A, B, C), 50, warmup=20)
        ms_bwd = _time(lambda: tsm.tsmttsm_backward(A, B, Wl), 50, warmup=20)
        # The backward's read + write roof: a device-to-device copy of the
        # same bytes (A -> dA-sized, B -> dB-sized buffers).
        dA_, dB_ = torch.empty_like(A), torch.empty_like(B)
        ms_copy = _time(lambda: (dA_.copy_(A), dB_.copy_(B)), 50, warmup=20)
        esz = A.element_size()
        out[name] = {"n": n, "m": w, "k": w, "fwd_ms": round(ms_fwd, 4), "bwd_ms": round(ms_bwd, 4),
                     "bwd_over_fwd": round(ms_bwd / ms_fwd, 3),
                     "fwd_GB/s": round(esz * n * 2 * w / (ms_fwd * 1e-3) / 1e9, 1),
                     "bwd_GB/s": round(2 * esz * n * 2 * w / (ms_bwd * 1e-3) / 1e9, 1),
                     "d2d_copy_same_bytes_ms": round(ms_copy, 4),
                     "bwd_over_copy": round(ms_bwd / ms_copy, 3)}
        del A, B, dA_, dB_
        torch.cuda.empty_cache()
    return out


# ------------------------------------------------------------------ our arm
def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--sweep-steps", type=int, default=20)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-sweep", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true")
    ap.add_argument("--ref-rows", type=int, default=HEAD_N)
    ap.add_argument("--ref-budget", type=float, default=150.0)
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3

    if args.impl == "reference":
        run_reference_arm(args)
        return 0

    import numpy as np
    import torch
    import torch.distributed as dist

    import tsm_benchmark_b200 as tsm
    from tsm_benchmark_b200 import _capi, distributed as tsmdist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    lib = _capi.load()
    peaks = load_peaks()

    def barrier():
        if world > 1:
            dist.barrier()

    # Inputs: the largest sweep shape decides the buffer sizes.
    max_a = max(n * m for n, m, k in SWEEP)
    max_b = max(n * k for n, m, k in SWEEP)
    bufA = torch.empty(max_a, dtype=torch.float64, device=dev)
    bufB = torch.empty(max_b, dtype=torch.float64, device=dev)
    tsm.fill_uniform(bufA, SEED + rank, 0)
    tsm.fill_uniform(bufB, SEED + rank, 1)
    stream = torch.cuda.current_stream(dev)
    sh = int(stream.cuda_stream)

    def views(n, m, k):
        return bufA[: n * m].view(n, m), bufB[: n * k].view(n, k)

    A, B = views(HEAD_N, HEAD_M, HEAD_K)
    C = torch.zeros((HEAD_M, HEAD_K), dtype=torch.float64, device=dev)
    need = lib.tsm_gemm_tn_workspace_size(HEAD_N, 64, 64)
    ws = torch.zeros(need, dtype=torch.uint8, device=dev)

    def call(a, b, c, n, m, k):
        st = lib.tsm_gemm_tn_f64(sh, n, m, k, a.data_ptr(), m, b.data_ptr(), k, c.data_ptr(), k, 0,
                                 ws.data_ptr(), ws.numel())
        if st != 0:
            _capi.check(st, "tsm_gemm_tn_f64")

    def step():
        call(A, B, C, HEAD_N, HEAD_M, HEAD_K)
        if world > 1:
            tsmdist.reduce_partials_(C)

    # ---------------- headline: warmup, then K timed steps.  The clock
    # sampler starts (and takes its start-up pause) before the warm-up, so
    # the timed steps follow the warm-up with the GPU already at speed.
    sampler = ClockSampler(local)
    sampler.start()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms_total = ev0.elapsed_time(ev1)
    if world > 1:
        t = torch.tensor([ms_total], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_total = float(t.item())
    ms_step = ms_total / args.steps
    bytes_step = algo_bytes(HEAD_N, HEAD_M, HEAD_K)
    value = bytes_step * world / (ms_step * 1e-3) / 1e9

    # correctness guard on the timed inputs (a checksum identity, no oracle)
    chk = float((A.sum(1) * B.sum(1)).sum())
    cs = float(C.sum()) if world == 1 else None
    bound = 4 * math.sqrt(HEAD_N) * 2.0**-53 * float(torch.linalg.norm(A)) * float(torch.linalg.norm(B)) * 8
    checksum_ok = (cs is None) or abs(cs - chk) <= bound
    bits = ctypes.c_uint(0)
    lib.tsm_workspace_check(sh, ws.data_ptr(), ctypes.byref(bits))
    dev_err = int(bits.value)

    # ---------------- the dominant kernel's roofline (the only kernel here)
    vidx = lib.tsm_gemm_tn_default_variant(0, HEAD_N, HEAD_M, HEAD_K, A.data_ptr(), HEAD_M, B.data_ptr(), HEAD_K)
    vname = tsm.variants()[vidx]["name"] if vidx >= 0 else None
    # time the kernel alone (no reduction step) for the roofline figure
    kev0 = torch.cuda.Event(enable_timing=True)
    kev1 = torch.cuda.Event(enable_timing=True)
    kn = max(20, min(args.steps, 100))
    kev0.record(stream)
    for _ in range(kn):
        call(A, B, C, HEAD_N, HEAD_M, HEAD_K)
    kev1.record(stream)
    torch.cuda.synchronize()
    k_ms = kev0.elapsed_time(kev1) / kn
    achieved = bytes_step / (k_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": vname, "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"],
                "frac_of_8tbs_spec": achieved / 8000.0,
                "bytes_per_launch": bytes_step, "launch_ms": k_ms,
                "traffic": profile_traffic("bulk_8x8")}

    # ---------------- by width (each shape: warmup + timed launches)
    by_width = []
    fp64_peak = None
    if not args.no_sweep and world == 1:
        sweep_rows = []
        for n, m, k in SWEEP:
            a, b = views(n, m, k)
            c = torch.zeros((m, k), dtype=torch.float64, device=dev)
            # One second at rest before each shape: every shape starts from the
            # same power state, as the best-of-5 DGEMM roof does (the FP64-bound
            # 64 x 64 otherwise inherits the clock the shapes before it left).
            torch.cuda.synchronize()
            time.sleep(1.0)
            for _ in range(3):
                call(a, b, c, n, m, k)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.sweep_steps):
                call(a, b, c, n, m, k)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / args.sweep_steps
            vi = lib.tsm_gemm_tn_default_variant(0, n, m, k, a.data_ptr(), m, b.data_ptr(), k)
            sweep_rows.append((n, m, k, ms, tsm.variants()[vi]["name"] if vi >= 0 else None))
        # The FP64 roof after the sweep: timed before it, the DGEMM loop left
        # the clock lowered by the power cap for the first shapes.
        fp64_peak = fp64_gemm_peak(dev)
        for n, m, k, ms, vname in sweep_rows:
            gbs = algo_bytes(n, m, k) / (ms * 1e-3) / 1e9
            # the binding roof: HBM bytes at the measured copy rate, or FP64
            # FMAs at the measured DGEMM rate, whichever takes longer
            t_hbm = algo_bytes(n, m, k) / (peaks["hbm_gbs"] * 1e9)
            t_fp64 = 2.0 * n * m * k / (fp64_peak["tflops"] * 1e12)
            by_width.append({"n": n, "m": m, "k": k, "ms": round(ms, 4), "GB/s": round(gbs, 1),
                             "frac_hbm": round(gbs / peaks["hbm_gbs"], 4),
                             "GFLOP/s": round(2.0 * n * m * k / (ms * 1e-3) / 1e9, 1),
                             "bound": "hbm" if t_hbm >= t_fp64 else "fp64",
                             "frac_roof": round(max(t_hbm, t_fp64) / (ms * 1e-3), 4),
                             "variant": vname})

    # ---------------- e2e through the C ABI from pinned host buffers: every
    # rank copies its rows in, computes, joins the cross-rank sum (N > 1) and
    # copies C out; max over ranks, bytes of the whole job.
    e2e = None
    if args.e2e_steps > 0:
        Ah = torch.empty((HEAD_N, HEAD_M), dtype=torch.float64, pin_memory=True)
        Bh = torch.empty((HEAD_N, HEAD_K), dtype=torch.float64, pin_memory=True)
        Ah.copy_(A, non_blocking=False)
        Bh.copy_(B, non_blocking=False)
        Ch = torch.empty((HEAD_M, HEAD_K), dtype=torch.float64, pin_memory=True)

        def e2e_step():
            A.copy_(Ah, non_blocking=True)
            B.copy_(Bh, non_blocking=True)
            step()
            Ch.copy_(C, non_blocking=True)

        e2e_step()
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.e2e_steps):
            e2e_step()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.e2e_steps
        if world > 1:
            t = torch.tensor([ms], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        # The bound of the end-to-end step: the host-to-device link, measured
        # here as one pinned copy of A alone (several streams measured the same).
        l0 = torch.cuda.Event(enable_timing=True)
        l1 = torch.cuda.Event(enable_timing=True)
        l0.record(stream)
        A.copy_(Ah, non_blocking=True)
        l1.record(stream)
        torch.cuda.synchronize()
        link = Ah.numel() * 8 / (l0.elapsed_time(l1) * 1e-3) / 1e9
        h2d = (Ah.numel() * 8 + Bh.numel() * 8) * world
        e2e = {"value": bytes_step * world / (ms * 1e-3) / 1e9, "unit": "GB/s", "ms_per_step": ms,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": Ch.numel() * 8 * world,
               "h2d_link_GB/s": round(link, 2), "frac_of_h2d_link": round(h2d / world / (ms * 1e-3) / 1e9 / link, 4)}
        del Ah, Bh

    # ---------------- the precision, batching and differentiation forms
    forms_out = None
    if world == 1 and not args.no_forms:
        del bufA, bufB, A, B
        torch.cuda.empty_cache()
        forms_out = forms(dev)

    # ---------------- CPU baseline (rank 0, N = 1)
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        res = reference_cpu(args.ref_rows, steps=50, warmup=1, budget_s=20.0)
        cpu = {k: res[k] for k in ("value", "unit", "cores", "kind", "sample", "naive_single_core")}
        # the same kernel on 1/8 of the rows: GB/s does not depend on n
        small = reference_cpu(max(1, args.ref_rows // 8), steps=20, warmup=1, budget_s=5.0)
        cpu["at_eighth_rows"] = {k: small[k] for k in ("value", "unit", "sample")}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload_config(world),
                "frac_hbm": value / world / peaks["hbm_gbs"], "roofline": roofline, "cpu_baseline": cpu,
                "e2e": e2e, "gpu_launches": args.steps, "clocks": clocks, "by_width": by_width,
                "fp64_peak": fp64_peak,
                "checksum_ok": checksum_ok, "device_error_bits": dev_err, "forms": forms_out}
        # the sweep, compactly, inside the roofline object: shape -> GB/s,
        # binding roof and fraction of it
        roofline["by_width"] = [{"shape": f"{r['n'].bit_length() - 1}:{r['m']}x{r['k']}", "GB/s": r["GB/s"],
                                 "bound": r["bound"], "frac_roof": r["frac_roof"]} for r in by_width]
        print(json.dumps(line), flush=True)
        print(summary(line), file=sys.stderr, flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def summary(line: dict) -> str:
    """A short human-readable digest of the JSON line (stderr)."""
    out = [f"headline {line['value']:.1f} GB/s ({line['ms_per_step']:.4f} ms/step), kernel alone "
           f"{line['roofline']['achieved']:.1f} GB/s = {line['roofline']['frac']:.3f} of {line['roofline']['peak']} "
           f"({line['roofline']['peak_source']})"]
    if line.get("e2e"):
        out.append(f"e2e {line['e2e']['value']:.2f} GB/s ({line['e2e']['frac_of_h2d_link']:.3f} of the "
                   f"{line['e2e']['h2d_link_GB/s']} GB/s host-to-device link)")
    for r in line.get("by_width") or []:
        out.append(f"  n=2^{r['n'].bit_length() - 1} {r['m']}x{r['k']}: {r['GB/s']} GB/s, {r['GFLOP/s']} GFLOP/s, "
                   f"{r['bound']} {r['frac_roof']}, {r['variant']}")
    f = line.get("forms") or {}
    for key in ("split_tf32", "split_bf16x2", "split_bf16x3"):
        if key in f:
            x = f[key]
            out.append(f"  {key}: {x['ms']} ms vs FP64 {x['fp64_ms']} ms ({x['speedup_vs_fp64']}x; sustained "
                       f"{x['sustained_300_calls']['speedup_vs_fp64']}x), err {x['err_normwise_rel']:.2e}")
    if "batched" in f:
        x = f["batched"]
        out.append(f"  batched: {x['ms']} ms, {x['GB/s']} GB/s, {x['speedup_vs_fp64_plain']}x per-problem launches")
    for key in ("autograd_f64", "autograd_f32"):
        if key in f:
            x = f[key]
            out.append(f"  {key}: fwd {x['fwd_ms']} ms, bwd {x['bwd_ms']} ms ({x['bwd_over_fwd']}x; "
                       f"{x['bwd_over_copy']}x a D2D copy of the same bytes)")
    for x in f.get("gram") or []:
        out.append(f"  gram {x['m']} at n={x['n']}: {x['gram_ms']} ms, {x['GB/s_of_A']} GB/s of A, "
                   f"{x['speedup']}x the two-operand call")
    for x in f.get("block_orth") or []:
        out.append(f"  block_orth {x['m']}x{x['k']} at n={x['n']}: {x['orth_ms']} ms, {x['GB/s']} GB/s, "
                   f"{x['over_tsmttsm']}x one TSMTTSM")
    if line.get("cpu_baseline"):
        c = line["cpu_baseline"]
        out.append(f"cpu baseline ({c['kind']}, {c['cores']} cores): {c['value']:.3f} GB/s; {c['sample']}")
    return "\n".join(out)


if __name__ == "__main__":
    sys.exit(main())
