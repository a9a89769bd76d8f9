#!/usr/bin/env python3
"""Runs one TSMTTSM shape a few times -- a small, self-contained case to put
under a profiler (ncu) or to time one variant.

    python -m tsm_benchmark_b200.profile_case --n 4194304 --m 8 --k 8 --reps 4 [--variant NAME]
    python -m tsm_benchmark_b200.profile_case --form split|backward|gram|batched|block_orth --n ... --m ... --k ...
    python -m tsm_benchmark_b200.profile_case --layout col --n ... --m ... --k ...   (A^T, B^T row-major)

One untimed call comes first (library setup); a profiler capture of the k-th
timed launch therefore skips k launches (`ncu -s k`).

Inputs are generated on the device (the library's uniform generator); the
last result is checked against the checksum identity
sum_ij C_ij = sum_r (sum_i A_ri)(sum_j B_rj).
"""
from __future__ import annotations

import argparse
import math
import sys

import torch


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1 << 22)
    ap.add_argument("--m", type=int, default=8)
    ap.add_argument("--k", type=int, default=8)
    ap.add_argument("--reps", type=int, default=4)
    ap.add_argument("--variant", default=None, help="variant name (default: the library's choice)")
    ap.add_argument("--form", choices=["plain", "split", "backward", "gram", "batched", "block_orth"],
                    default="plain",
                    help="plain FP64, FP32 TF32-split on tensor cores, the fused backward, the Gram product "
                         "C = A^T A, a batch of --count products of n rows and widths m x k in one launch, or "
                         "block orthogonalisation B <- B - A (A^T B) (two launches: the product, then the TSMM)")
    ap.add_argument("--count", type=int, default=64, help="problems in the batch (--form batched)")
    ap.add_argument("--dtype", choices=["f64", "f32"], default="f64", help="storage type of the backward")
    ap.add_argument("--split-kind", choices=["tf32", "bf16x2", "bf16x3"], default="tf32",
                    help="parts of the split form (--form split)")
    ap.add_argument("--layout", choices=["row", "col"], default="row",
                    help="plain form: row-major operands, or column-major ones (A^T, B^T stored row-major, "
                         "through tsm_gemm_tn_strided_f64)")
    args = ap.parse_args(argv)

    from tsm_benchmark_b200 import (BatchedTSMTTSM, block_orthogonalize, fill_uniform, gram, tsmttsm,
                                    tsmttsm_backward, tsmttsm_split, variants)
    dev = torch.device("cuda", 0)
    if args.form in ("gram", "batched", "block_orth"):
        if args.form == "gram":
            A = torch.empty((args.n, args.m), dtype=torch.float64, device=dev)
            fill_uniform(A, 1, 0)
            run = lambda: gram(A)  # noqa: E731
            nbytes = 8 * args.n * args.m
        elif args.form == "block_orth":
            # A's columns scaled to about unit norm, so repeated steps keep B bounded.
            A = torch.empty((args.n, args.m), dtype=torch.float64, device=dev)
            B = torch.empty((args.n, args.k), dtype=torch.float64, device=dev)
            fill_uniform(A, 1, 0)
            fill_uniform(B, 1, 1)
            A.mul_(math.sqrt(3.0 / max(args.n, 1)))
            C = torch.empty((args.m, args.k), dtype=torch.float64, device=dev)
            run = lambda: block_orthogonalize(A, B, C)  # noqa: E731
            nbytes = 8 * args.n * (2 * args.m + 3 * args.k)  # A and B read twice, B written once
        else:
            As, Bs = [], []
            for i in range(args.count):
                a = torch.empty((args.n, args.m), dtype=torch.float64, device=dev)
                b = torch.empty((args.n, args.k), dtype=torch.float64, device=dev)
                fill_uniform(a, 10 + i, 0)
                fill_uniform(b, 10 + i, 1)
                As.append(a)
                Bs.append(b)
            bt = BatchedTSMTTSM(As, Bs)
            run = bt.run
            nbytes = 8 * args.count * args.n * (args.m + args.k)
        run()  # first call: library setup, not timed
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for _ in range(args.reps):
            run()
        ev1.record()
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / args.reps
        print(f"{args.form} n={args.n} m={args.m} k={args.k}: {ms:.4f} ms/call, {nbytes / (ms * 1e-3) / 1e9:.1f} GB/s")
        return 0
    if args.form != "plain":
        A = torch.empty((args.n, args.m), dtype=torch.float64, device=dev)
        B = torch.empty((args.n, args.k), dtype=torch.float64, device=dev)
        fill_uniform(A, 1, 0)
        fill_uniform(B, 1, 1)
        if args.form == "split":
            A, B = A.float(), B.float()
            run = lambda: tsmttsm_split(A, B, kind=args.split_kind)  # noqa: E731
            nbytes = 4 * args.n * (args.m + args.k)
        else:
            dt = torch.float64 if args.dtype == "f64" else torch.float32
            A, B = A.to(dt), B.to(dt)
            dC = torch.ones((args.m, args.k), dtype=dt, device=dev)
            run = lambda: tsmttsm_backward(A, B, dC)  # noqa: E731
            nbytes = 2 * A.element_size() * args.n * (args.m + args.k)
        run()  # first call: library setup, not timed
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for _ in range(args.reps):
            run()
        ev1.record()
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / args.reps
        print(f"{args.form} {args.dtype if args.form == 'backward' else args.split_kind} n={args.n} m={args.m} k={args.k}: {ms:.4f} ms/call, {nbytes / (ms * 1e-3) / 1e9:.1f} GB/s")
        return 0
    if args.layout == "col":
        At = torch.empty((args.m, args.n), dtype=torch.float64, device=dev)
        Bt = torch.empty((args.k, args.n), dtype=torch.float64, device=dev)
        fill_uniform(At, 1, 0)
        fill_uniform(Bt, 1, 1)
        A, B = At.t(), Bt.t()
    else:
        A = torch.empty((args.n, args.m), dtype=torch.float64, device=dev)
        B = torch.empty((args.n, args.k), dtype=torch.float64, device=dev)
        fill_uniform(A, 1, 0)
        fill_uniform(B, 1, 1)
    vidx = -1
    if args.variant:
        names = {v["name"]: v["index"] for v in variants()}
        vidx = names[args.variant]
    C = tsmttsm(A, B, variant=vidx)  # first call: library setup, not timed
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.reps):
        C = tsmttsm(A, B, variant=vidx)
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.reps
    gbs = 8 * args.n * (args.m + args.k) / (ms * 1e-3) / 1e9
    chk = float((A.sum(1) * B.sum(1)).sum())
    bound = 32 * math.sqrt(args.n) * 2.0**-53 * float(torch.linalg.norm(A)) * float(torch.linalg.norm(B))
    ok = abs(float(C.sum()) - chk) <= bound * math.sqrt(args.m * args.k)
    print(f"{'column-major ' if args.layout == 'col' else ''}n={args.n} m={args.m} k={args.k} reps={args.reps}: "
          f"{ms:.4f} ms/call, {gbs:.1f} GB/s, checksum "
          f"{'ok' if ok else 'MISMATCH'}")
    return 0 if ok else 1


if __name__ == "__main__":
    sys.exit(main())
