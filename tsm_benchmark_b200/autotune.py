#!/usr/bin/env python3
"""Autotuner: picks the fastest compiled variant per (m, k, n-bucket, dtype).

    python -m tsm_benchmark_b200.autotune [--shapes sweep|batched|all] [--out tuned.json]
    python -m tsm_benchmark_b200.autotune --shapes batched-paths   (the batched kernel's path per class)
    python -m tsm_benchmark_b200.autotune --pairs 8x8 --merge        (re-tune one shape, keep the rest)
    python -m tsm_benchmark_b200.autotune --shapes gram              (the Gram variant per width, C = A^T A)

For every width pair and row bucket it times each applicable variant of the
table (CUDA events, warm-up then repeated launches, inputs larger than L2
where the bucket allows), checks every candidate against the first one's
result (the checksum identity and a normwise bound), re-times the best
three (those within 5 % of the fastest) in interleaved rounds and records
the one with the best median.
The result, ``tsm_benchmark_b200/tuned.json``, is baked into the library's
default choice by the next build (codegen.py reads it); until then the API's
``variant=`` argument can use it directly.

Replaces the reference's manual search over launch shapes (main.cc:171-192:
M x stride x tile) and its generator's stride helpers (suggest_stride /
validate_stride, sycl_codegen_new.py:530-580).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "tuned.json")

SWEEP_PAIRS = [(1, 1), (2, 2), (4, 4), (8, 8), (16, 16), (32, 32), (64, 64), (4, 32), (32, 4), (1, 64)]
GRAM_WIDTHS = [1, 2, 4, 8, 16, 32, 48, 64]
# Sections of tuned.json that one mode writes and the others keep.
KEPT_SECTIONS = ("batched_paths", "gram_choices", "gram_timings")
BATCHED_PAIRS = [(a, b) for a in (4, 8, 16, 32) for b in (4, 8, 16, 32)]
# (nmin, n to time at): the largest nmin <= n selects the entry at run time.
BUCKETS = [(0, 1 << 15), (1 << 18, 1 << 20), (1 << 23, 1 << 26)]
MAX_BYTES = 24 << 30  # per operand pair while tuning


def _cap(w: int) -> int:
    c = 1
    while c < w:
        c *= 2
    return c


def candidates(variants: list[dict], m: int, k: int, dtype: str = "f64") -> list[dict]:
    """Variants of `dtype` that accept (m, k) for distinct A and B: every
    exact one, and the capacity ones no more than twice the smallest capacity
    per side (larger ones only add masked work).  Gram variants (B is A)
    are not candidates."""
    out = []
    cm, ck = _cap(m), _cap(k)
    for v in variants:
        if v["dtype"] != dtype or v.get("gram"):
            continue
        if v["exact"]:
            if m == v["wa"] and k == v["wb"]:
                out.append(v)
        elif m <= v["wa"] <= 2 * cm and k <= v["wb"] <= 2 * ck:
            out.append(v)
    return out


def gram_candidates(variants: list[dict], w: int, dtype: str = "f64") -> list[dict]:
    """Gram variants (C = A^T A, A streamed once) of `dtype` that take width
    `w`: the exact ones of that width, and capacity ones no more than twice
    the smallest capacity."""
    cw = _cap(w)
    return [v for v in variants if v.get("gram") and v["dtype"] == dtype and
            (v["wa"] == w if v["exact"] else w <= v["wa"] <= 2 * cw)]


def refinement_set(row: dict, within: float = 1.05, top_n: int = 3) -> list[str]:
    """Names of the fastest correct candidates of one shape, fastest first:
    at most `top_n`, each within `within` times the fastest single timing.
    `row` maps a variant name to {"ms": ..., "ok": ...}."""
    top = sorted((r["ms"], name) for name, r in row.items() if r["ok"])
    return [name for ms_, name in top[:top_n] if ms_ <= top[0][0] * within] if top else []


def median_winner(samples: dict) -> tuple[str, dict]:
    """The candidate with the smallest median over its interleaved timings
    (ties go to the one listed first), and every candidate's median."""
    med = {name: statistics.median(t) for name, t in samples.items()}
    return min(med, key=med.get), med


def keep_sections(res: dict, old: dict) -> dict:
    """`res` with the sections of an earlier file `old` that this mode did not
    write (KEPT_SECTIONS: another mode's tuning) carried over."""
    out = dict(res)
    for key in KEPT_SECTIONS:
        if key not in out and key in old:
            out[key] = old[key]
    return out


def merge_results(old: dict, res: dict, pairs) -> dict:
    """`res` (a tuning of `pairs`) with the other pairs' choices and timings
    of an earlier result `old` kept; choices sorted by (m, k, nmin)."""
    tuned = {(int(m), int(k)) for m, k in pairs}
    out = dict(res)
    out["choices"] = [c for c in old.get("choices", []) if (int(c["m"]), int(c["k"])) not in tuned] + \
        list(res["choices"])
    out["choices"].sort(key=lambda c: (int(c["m"]), int(c["k"]), int(c.get("nmin", 0))))
    kept = {key: val for key, val in old.get("timings", {}).items()
            if tuple(int(x) for x in key.split("@")[0].split("x")) not in tuned}
    out["timings"] = {**kept, **res["timings"]}
    return out


def time_variant(call, reps: int, warmup: int = 3) -> float:
    import torch
    for _ in range(warmup):
        call()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        call()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def refine(row: dict, make_call, nbytes: int, reps_time_ms: float, rounds: int):
    """The top candidates of `row` (within 5 % of the fastest single timing),
    timed in interleaved rounds (A B C A B C ...) and decided by the median --
    single timings of near-equal kernels differ by a few percent from run to
    run, more than the kernels do.  Records each one's median in `row` and
    returns (name, ms, GB/s) of the winner, or None with fewer than two."""
    top = refinement_set(row)
    if len(top) < 2:
        return None
    reps = max(3, min(100, int(reps_time_ms / 3 / max(row[top[0]]["ms"], 1e-3))))
    samples = {name: [] for name in top}
    for _ in range(rounds):
        for name in top:
            samples[name].append(time_variant(make_call(name), reps, warmup=1))
    win, med = median_winner(samples)
    for name in top:
        row[name]["median_ms_interleaved"] = round(med[name], 5)
    return (win, med[win], nbytes / (med[win] * 1e-3) / 1e9)


def tune(pairs, buckets=BUCKETS, reps_time_ms: float = 150.0, verbose: bool = True, rounds: int = 5) -> dict:
    import torch

    from . import variants as list_variants
    from .api import fill_uniform, tsmttsm

    dev = torch.device("cuda", 0)
    vs = list_variants()
    choices, timings = [], {}
    for m, k in pairs:
        for nmin, n in buckets:
            while n > 1 << 12 and 8 * n * (m + k) > MAX_BYTES:
                n //= 2
            A = torch.empty((n, m), dtype=torch.float64, device=dev)
            B = torch.empty((n, k), dtype=torch.float64, device=dev)
            fill_uniform(A, 3, 0)
            fill_uniform(B, 3, 1)
            chk = float((A.sum(1) * B.sum(1)).sum())
            bound = 8 * math.sqrt(n) * 2.0**-53 * float(torch.linalg.norm(A)) * float(torch.linalg.norm(B))
            C = torch.empty((m, k), dtype=torch.float64, device=dev)
            ref = None
            best = None
            row = {}
            for v in candidates(vs, m, k):
                call = lambda: tsmttsm(A, B, C, variant=v["index"])  # noqa: E731
                t0 = time_variant(call, 1, warmup=1)
                reps = max(3, min(200, int(reps_time_ms / max(t0, 1e-3))))
                ms = time_variant(call, reps)
                got = C.clone()
                if ref is None:
                    ref = got
                ok = abs(float(got.sum()) - chk) <= bound * math.sqrt(m * k) and \
                    float(torch.linalg.norm(got - ref)) <= 2 * bound
                gbs = 8 * n * (m + k) / (ms * 1e-3) / 1e9
                row[v["name"]] = {"ms": round(ms, 5), "GB/s": round(gbs, 1), "ok": ok}
                if ok and (best is None or ms < best[1]):
                    best = (v["name"], ms, gbs)
            idx = {v["name"]: v["index"] for v in vs}
            best = refine(row, lambda name: (lambda: tsmttsm(A, B, C, variant=idx[name])), 8 * n * (m + k),
                          reps_time_ms, rounds) or best
            timings[f"{m}x{k}@{n}"] = row
            if best:
                choices.append({"m": m, "k": k, "nmin": nmin, "n_timed": n, "variant": best[0],
                                "ms": round(best[1], 5), "GB/s": round(best[2], 1)})
                if verbose:
                    print(f"{m:>2}x{k:<2} n={n:>9}: {best[0]:<40} {best[2]:8.1f} GB/s "
                          f"({len(row)} candidates)", flush=True)
            del A, B
            torch.cuda.empty_cache()
    return {"device": torch.cuda.get_device_name(dev), "dtype": "f64", "when": time.strftime("%Y-%m-%d %H:%M:%S"),
            "choices": choices, "timings": timings}


def tune_gram(widths=GRAM_WIDTHS, buckets=BUCKETS, reps_time_ms: float = 150.0, verbose: bool = True,
              rounds: int = 5) -> dict:
    """For each width and row bucket, every Gram variant that takes the width
    (C = A^T A through tsmttsm(A, A)), timed like the plain variants; each
    result must be exactly symmetric and within the normwise bound of the
    first one's.  Returns {"gram_choices": [...], "gram_timings": {...}}."""
    import torch

    from . import variants as list_variants
    from .api import fill_uniform, tsmttsm

    dev = torch.device("cuda", 0)
    vs = list_variants()
    idx = {v["name"]: v["index"] for v in vs}
    choices, timings = [], {}
    for w in widths:
        for nmin, n in buckets:
            while n > 1 << 12 and 8 * n * w > MAX_BYTES:
                n //= 2
            A = torch.empty((n, w), dtype=torch.float64, device=dev)
            fill_uniform(A, 3, 0)
            bound = 8 * math.sqrt(n) * 2.0**-53 * float(torch.linalg.norm(A)) ** 2
            C = torch.empty((w, w), dtype=torch.float64, device=dev)
            ref, best, row = None, None, {}
            for v in gram_candidates(vs, w):
                call = lambda: tsmttsm(A, A, C, variant=v["index"])  # noqa: E731
                t0 = time_variant(call, 1, warmup=1)
                reps = max(3, min(200, int(reps_time_ms / max(t0, 1e-3))))
                ms = time_variant(call, reps)
                got = C.clone()
                if ref is None:
                    ref = got
                ok = bool(torch.equal(got, got.T)) and float(torch.linalg.norm(got - ref)) <= 2 * bound
                gbs = 8 * n * w / (ms * 1e-3) / 1e9
                row[v["name"]] = {"ms": round(ms, 5), "GB/s": round(gbs, 1), "ok": ok}
                if ok and (best is None or ms < best[1]):
                    best = (v["name"], ms, gbs)
            best = refine(row, lambda name: (lambda: tsmttsm(A, A, C, variant=idx[name])), 8 * n * w,
                          reps_time_ms, rounds) or best
            timings[f"gram{w}@{n}"] = row
            if best:
                choices.append({"w": w, "nmin": nmin, "n_timed": n, "variant": best[0],
                                "ms": round(best[1], 5), "GB/s": round(best[2], 1)})
                if verbose:
                    print(f"gram {w:>2} n={n:>9}: {best[0]:<40} {best[2]:8.1f} GB/s ({len(row)} candidates)",
                          flush=True)
            del A
            torch.cuda.empty_cache()
    return {"gram_choices": choices, "gram_timings": timings}


# Width classes of the batched kernel with two compiled consumer paths.
BATCHED_TC_CLASSES = [(16, 16), (16, 32), (32, 16), (32, 32)]


def tune_batched_paths(count: int = 96, rounds: int = 5, reps: int = 10, seed: int = 11,
                       verbose: bool = True) -> list[dict]:
    """For each tensor-core class of the batched kernel, both consumer paths
    (FP64 tensor cores, SIMT register tiles) timed inside the batched launch
    on `count` problems of that class (n log-uniform in [10^4, 10^6], the
    upper part of the batched configuration's range), in interleaved rounds;
    the path with the smaller median wins.  Both paths' results must agree
    within the normwise bound first."""
    import numpy as np
    import torch

    from .api import fill_uniform
    from .batched import BatchedTSMTTSM

    dev = torch.device("cuda", 0)
    out = []
    for m, k in BATCHED_TC_CLASSES:
        rng = np.random.default_rng(seed + m + 3 * k)
        ns = np.exp(rng.uniform(np.log(1e4), np.log(1e6), size=count)).astype(np.int64)
        As, Bs = [], []
        for i, n in enumerate(ns):
            a = torch.empty((int(n), m), dtype=torch.float64, device=dev)
            b = torch.empty((int(n), k), dtype=torch.float64, device=dev)
            fill_uniform(a, 100 + i, 0)
            fill_uniform(b, 100 + i, 1)
            As.append(a)
            Bs.append(b)
        plans = {path: BatchedTSMTTSM(As, Bs, class_paths={(m, k): path}) for path in ("dmma", "simt")}
        res = {path: [c.clone() for c in p.run()] for path, p in plans.items()}
        for a, b, c0, c1 in zip(As, Bs, res["dmma"], res["simt"]):
            bound = 8 * math.sqrt(a.shape[0]) * 2.0**-53 * float(torch.linalg.norm(a)) * float(torch.linalg.norm(b))
            if float(torch.linalg.norm(c0 - c1)) > bound:
                raise RuntimeError(f"batched paths disagree for class {m}x{k}")
        samples = {path: [] for path in plans}
        for _ in range(rounds):
            for path, p in plans.items():
                samples[path].append(time_variant(p.run, reps, warmup=1))
        win, med = median_winner(samples)
        nbytes = int(sum(8 * int(n) * (m + k) for n in ns))
        out.append({"m": m, "k": k, "path": win, "problems": count, "bytes": nbytes,
                    "median_ms": {path: round(t, 5) for path, t in med.items()}})
        if verbose:
            print(f"batched {m:>2}x{k:<2}: {win:<5} " + ", ".join(
                f"{path} {t:.4f} ms ({nbytes / (t * 1e-3) / 1e9:.0f} GB/s)" for path, t in med.items()), flush=True)
        del As, Bs, plans, res
        torch.cuda.empty_cache()
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--shapes", choices=["sweep", "batched", "batched-paths", "gram", "all"], default="all",
                    help="batched-paths: the batched kernel's consumer path per tensor-core class; "
                         "gram: the Gram variant per width (each kept beside the other choices of --out)")
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--budget-ms", type=float, default=150.0, help="timed milliseconds per candidate")
    ap.add_argument("--pairs", default=None, help="only these width pairs, e.g. 8x8,16x16 (overrides --shapes)")
    ap.add_argument("--merge", action="store_true",
                    help="keep the other pairs' choices and timings of an existing --out file")
    args = ap.parse_args(argv)
    if args.shapes in ("batched-paths", "gram"):
        old = {}
        if os.path.exists(args.out):
            with open(args.out) as f:
                old = json.load(f)
        if args.shapes == "gram":
            old.update(tune_gram(reps_time_ms=args.budget_ms))
            what = f"{len(old['gram_choices'])} Gram choices"
        else:
            old["batched_paths"] = tune_batched_paths()
            what = f"{len(old['batched_paths'])} batched paths"
        with open(args.out, "w") as f:
            json.dump(old, f, indent=1)
            f.write("\n")
        print(f"wrote {args.out}: {what}")
        return 0
    pairs = {"sweep": SWEEP_PAIRS, "batched": BATCHED_PAIRS,
             "all": sorted(set(SWEEP_PAIRS + BATCHED_PAIRS))}[args.shapes]
    if args.pairs:
        pairs = [tuple(int(x) for x in p.split("x")) for p in args.pairs.split(",")]
    res = tune(pairs, reps_time_ms=args.budget_ms)
    if args.merge and os.path.exists(args.out):
        with open(args.out) as f:
            res = merge_results(json.load(f), res, pairs)
    if os.path.exists(args.out):
        with open(args.out) as f:
            res = keep_sections(res, json.load(f))
    with open(args.out, "w") as f:
        json.dump(res, f, indent=1)
        f.write("\n")
    print(f"wrote {args.out}: {len(res['choices'])} choices")
    return 0


if __name__ == "__main__":
    sys.exit(main())
