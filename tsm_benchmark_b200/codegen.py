#!/usr/bin/env python3
"""CUDA variant generator for the TSMTTSM kernels (C = A^T * B).

Rewrite of the reference's SYCL generators (sycl_codegen.py:16-263,
sycl_codegen_new.py:142-363).  Those emit one SYCL kernel per
(M, N, TM, TN, stride, local_size, leap_frog, reduction, unroll) with scalar
accumulators, a grid-stride row loop and FP64 atomics.  This generator emits
rows of the kernel table in ``csrc/generated/``: explicit instantiations of
the sm_100a templates in ``csrc/tsm_plain.cuh`` (SIMT register tiles) and
``csrc/tsm_dmma.cuh`` (FP64 tensor cores, exact widths 16..64) over the axes

    width pair      (wa, wb)        -- exact widths or width capacities
    tile            (ta, tb)        -- per-thread register tile of C
                                       (the reference's TM x TN)
    consumer warps  cw              -- CTA size (the reference's local_size)
    prefetch depth  stages          -- shared-memory ring depth (the
                                       reference's leap-frog is depth 2 in
                                       registers)
    chunk rows      rows            -- rows per TMA bulk copy
    unroll          unroll          -- row-loop unroll (the reference's
                                       --unroll)
    reduction       two-level       -- warp shuffle + fixed-order CTA sum +
                                       last-CTA fixed-order sum (the only
                                       scheme: deterministic; replaces
                                       "global" / "twolevel" / "sg")

plus a tuned-defaults table (from ``tuned.json``, written by the autotuner)
that the library consults before falling back to table order.

Usage::

    python -m tsm_benchmark_b200.codegen            # write csrc/generated/
    python -m tsm_benchmark_b200.codegen --check    # exit 1 if out of date
    python -m tsm_benchmark_b200.codegen --list     # print the variant names

    # the reference generators' command line: the drop-in header on stdout
    python -m tsm_benchmark_b200.codegen --M 4 8 16 32 --tile-sizes 2 4 \\
        [--stride S] [--local-size L] [--sg-size 32] [--unroll U] \\
        [--with-benchmark] [--style v1|v2] > tsmttsm_kernels.hh

The emitted files are committed; tests check that regenerating reproduces
them byte for byte.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import math
import os
import sys
from typing import Iterable

HERE = os.path.dirname(os.path.abspath(__file__))
GEN_DIR = os.path.join(HERE, "csrc", "generated")
TUNED_JSON = os.path.join(HERE, "tuned.json")

SMEM_LIMIT = 227 * 1024  # dynamic shared memory per CTA on sm_100a
WIDTH_CAPS = (1, 2, 4, 8, 16, 32, 64)


@dataclasses.dataclass(frozen=True)
class BulkVariant:
    """One TMA-bulk pipelined kernel (tsm_tn_bulk_kernel)."""

    wa: int
    wb: int
    ta: int
    tb: int
    cw: int = 8
    stages: int = 6
    rows: int = 0  # 0: sized for ~32 KB stages
    unroll: int = 1
    exact: bool = True
    dtype: str = "f64"
    gram: bool = False  # C = A^T A only: streams A once

    @property
    def esize(self) -> int:
        return 8 if self.dtype == "f64" else 4

    @property
    def epc(self) -> int:  # elements per 16-byte chunk
        return 16 // self.esize

    def resolved(self) -> "BulkVariant":
        if self.rows:
            return self
        rg = self.cw * 32 // self.num_tiles
        e = self.epc
        width = self.wa if self.gram else self.wa + self.wb
        rows = max(e, (32768 // (self.esize * width)) // e * e)
        # Round to whole passes of the row groups, keeping every bulk copy a
        # multiple of 16 bytes.
        if rows >= rg:
            rows = rows // rg * rg
        rows = max(e, rows // e * e)
        return dataclasses.replace(self, rows=rows)

    @property
    def num_tiles(self) -> int:
        return (self.wa // self.ta) * (self.wb // self.tb)

    @property
    def name(self) -> str:
        v = self.resolved()
        kind = "bulk" if v.dtype == "f64" else "bulkf32"
        s = (f"{kind}_{v.wa}x{v.wb}_t{v.ta}x{v.tb}_w{v.cw}_s{v.stages}"
             f"_r{v.rows}_u{v.unroll}")
        s = s if v.exact else s + "_cap"
        return s + "_gram" if v.gram else s

    def smem_bytes(self) -> int:
        v = self.resolved()
        ct = v.cw * 32
        nt = v.num_tiles
        slots = v.cw if nt < 32 else ct // nt
        ring = v.stages * v.rows * (v.wa if v.gram else v.wa + v.wb) * v.esize
        red = slots * v.wa * v.wb * 8
        data = max(ring, red)
        return (data + 127) // 128 * 128 + 2 * v.stages * 8 + 16

    def validate(self) -> list[str]:
        v = self.resolved()
        errs = []
        if v.wa % v.ta or v.wb % v.tb:
            errs.append("tile must divide the width")
        nt = v.num_tiles
        if nt & (nt - 1):
            errs.append("tile count must be a power of two")
        if (v.cw * 32) % nt:
            errs.append("consumer threads must cover whole tiles")
        if v.rows % v.epc:
            errs.append("chunk rows must keep bulk copies a multiple of 16 bytes")
        if v.dtype not in ("f64", "f32"):
            errs.append("dtype must be f64 or f32")
        rg = v.cw * 32 // max(nt, 1)
        if v.rows >= rg and (v.rows // rg) % v.unroll:
            errs.append("unroll must divide the rows per thread")
        if v.ta * v.tb > 64:
            errs.append("register tile above 64 accumulators")
        if v.gram and not (v.exact and v.wa == v.wb):
            errs.append("Gram variants are exact and square")
        if self.smem_bytes() > SMEM_LIMIT:
            errs.append(f"shared memory {self.smem_bytes()} above {SMEM_LIMIT}")
        return errs

    def emit(self) -> str:
        v = self.resolved()
        ctype = "double" if v.dtype == "f64" else "float"
        return (f'TSM_BULK_VARIANT("{self.name}", {ctype}, {v.wa}, {v.wb}, {v.ta}, {v.tb}, '
                f'{v.cw}, {v.stages}, {v.rows}, {v.unroll}, '
                f'{"true" if v.exact else "false"}, {"true" if v.gram else "false"})')


@dataclasses.dataclass(frozen=True)
class DirectVariant:
    """One direct-load kernel (tsm_tn_direct_kernel)."""

    wa: int
    wb: int
    ta: int
    tb: int
    threads: int = 256
    exact: bool = False
    dtype: str = "f64"

    @property
    def num_tiles(self) -> int:
        return (self.wa // self.ta) * (self.wb // self.tb)

    @property
    def name(self) -> str:
        kind = "direct" if self.dtype == "f64" else "directf32"
        s = f"{kind}_{self.wa}x{self.wb}_t{self.ta}x{self.tb}_th{self.threads}"
        return s if self.exact else s + "_cap"

    def validate(self) -> list[str]:
        errs = []
        if self.wa % self.ta or self.wb % self.tb:
            errs.append("tile must divide the width")
        nt = self.num_tiles
        if nt & (nt - 1):
            errs.append("tile count must be a power of two")
        if self.threads % nt or self.threads % 32:
            errs.append("threads must cover whole tiles")
        if self.ta * self.tb > 64:
            errs.append("register tile above 64 accumulators")
        return errs

    def emit(self) -> str:
        ctype = "double" if self.dtype == "f64" else "float"
        return (f'TSM_DIRECT_VARIANT("{self.name}", {ctype}, {self.wa}, {self.wb}, {self.ta}, '
                f'{self.tb}, {self.threads}, {"true" if self.exact else "false"})')


@dataclasses.dataclass(frozen=True)
class DmmaVariant:
    """One FP64 tensor-core kernel (tsm_tn_dmma_kernel, csrc/tsm_dmma.cuh):
    exact widths, multiples of 16 up to 64; 2-D swizzled TMA loads."""

    wa: int
    wb: int
    mt: int = 0      # 8x8 tiles of C per warp along m (0: best loads-per-DMMA ratio)
    nt: int = 0      # ... along k
    cw: int = 0      # 0: regions x row slots, 8..12 warps
    stages: int = 0  # 0: as many ~64 KB stages as fit, at most 4
    rows: int = 0    # 0: ~64 KB stages
    dtype: str = "f64"
    exact: bool = True
    gram: bool = False  # C = A^T A only: streams A once

    @staticmethod
    def best_region(wa: int, wb: int) -> tuple[int, int]:
        """(mt, nt): even tile counts dividing wa/8 and wb/8, at most 16 tiles,
        maximising DMMAs per shared load (mt nt / (mt/2 + nt/2)); ties go to
        the larger region, then to mt >= nt."""
        best = None
        for mt in range(2, wa // 8 + 1, 2):
            for nt in range(2, wb // 8 + 1, 2):
                if (wa // 8) % mt or (wb // 8) % nt or mt * nt > 16:
                    continue
                key = (mt * nt / (mt + nt), mt * nt, mt >= nt)
                if best is None or key > best[0]:
                    best = (key, mt, nt)
        return best[1], best[2]

    @property
    def regions(self) -> int:
        if self.gram:  # upper-triangle block-pair regions of tsm_gram_dmma_kernel
            return {16: 1, 32: 1, 48: 2, 64: 2}[self.wa]
        mt, nt = (self.mt, self.nt) if self.mt else self.best_region(self.wa, self.wb)
        return ((self.wa // 8) // mt) * ((self.wb // 8) // nt)

    def resolved(self) -> "DmmaVariant":
        v = self
        if not v.mt and not v.gram:
            mt, nt = self.best_region(v.wa, v.wb)
            v = dataclasses.replace(v, mt=mt, nt=nt)
        if not v.cw:
            r = v.regions
            v = dataclasses.replace(v, cw=r * max(1, -(-8 // r)))
        blocks = v.wa // 16 + (0 if v.gram else v.wb // 16)
        if not v.rows:
            # whole 8-row swizzle groups and an equal number of 4-row k-steps
            # for every row slot
            slots = v.cw // v.regions
            unit = 8 * 4 * slots // math.gcd(8, 4 * slots)
            v = dataclasses.replace(v, rows=max(unit, min(256, 512 // blocks) // unit * unit))
        if not v.stages:
            stage = blocks * v.rows * 128
            v = dataclasses.replace(v, stages=max(2, min(4, (SMEM_LIMIT - 2048) // stage)))
        return v

    @property
    def name(self) -> str:
        v = self.resolved()
        if v.gram:
            return f"dmma_{v.wa}x{v.wb}_gram_w{v.cw}_s{v.stages}_r{v.rows}"
        return f"dmma_{v.wa}x{v.wb}_t{8 * v.mt}x{8 * v.nt}_w{v.cw}_s{v.stages}_r{v.rows}"

    def smem_bytes(self) -> int:
        v = self.resolved()
        slots = v.cw // v.regions
        ring = v.stages * (v.wa // 16 + (0 if v.gram else v.wb // 16)) * v.rows * 128
        red = slots * v.wa * v.wb * 8
        return 1024 + (max(ring, red) + 127) // 128 * 128 + 2 * v.stages * 8 + 16

    def validate(self) -> list[str]:
        v = self.resolved()
        errs = []
        if v.wa % 16 or v.wb % 16 or not (16 <= v.wa <= 64 and 16 <= v.wb <= 64):
            errs.append("widths must be multiples of 16 in 16..64")
        if not v.gram and (v.mt % 2 or v.nt % 2 or (v.wa // 8) % v.mt or (v.wb // 8) % v.nt or v.mt * v.nt > 16):
            errs.append("region: even tile counts dividing the widths, at most 16 tiles")
        if v.cw % v.regions:
            errs.append("consumer warps must cover whole regions")
        if v.cw > 12:
            errs.append("more than 12 consumer warps (register cap)")
        boxes = -(-v.rows // 256)  # tensor boxes of at most 256 rows per 16-column block
        if v.rows <= 0 or v.rows % 8 or v.rows > 1024 or v.rows % boxes or (v.rows // boxes) % 8:
            errs.append("chunk rows: equal boxes of whole 8-row groups, at most 256 rows each")
        if (v.rows // 4) % (v.cw // v.regions):
            errs.append("chunk k-steps must split evenly over the row slots")
        if v.dtype != "f64":
            errs.append("FP64 only")
        if v.gram and v.wa != v.wb:
            errs.append("Gram variants are square")
        if self.smem_bytes() > SMEM_LIMIT:
            errs.append(f"shared memory {self.smem_bytes()} above {SMEM_LIMIT}")
        return errs

    def emit(self) -> str:
        v = self.resolved()
        if v.gram:
            return f'TSM_GRAM_DMMA_VARIANT("{self.name}", {v.wa}, {v.cw}, {v.stages}, {v.rows})'
        return f'TSM_DMMA_VARIANT("{self.name}", {v.wa}, {v.wb}, {v.mt}, {v.nt}, {v.cw}, {v.stages}, {v.rows})'


DMMA_WIDTHS = (16, 32, 48, 64)


def default_tile(w: int) -> int:
    """Per-thread tile extent for a width (capacity)."""
    return {1: 1, 2: 2, 4: 4, 8: 4, 16: 8, 32: 8, 64: 8}[w]


# Width pairs with exact (fully specialised) bulk variants: every shape of the
# plain sweep (square 1..64, (4,32), (32,4), (1,64)) and the widths of the
# batched problems ({4,8,16,32}^2).
EXACT_PAIRS = sorted(set(
    [(w, w) for w in WIDTH_CAPS] + [(4, 32), (32, 4), (1, 64)]
    + [(a, b) for a in (4, 8, 16, 32) for b in (4, 8, 16, 32)]))

# Extra tile / launch candidates the autotuner may pick for the sweep shapes.
EXTRA_CANDIDATES: dict[tuple[int, int], list[dict]] = {
    (1, 1): [dict(unroll=2), dict(unroll=4)],
    (2, 2): [dict(unroll=2)],
    (4, 4): [dict(ta=2, tb=2), dict(unroll=2)],
    (8, 8): [dict(ta=8, tb=8), dict(unroll=2), dict(ta=2, tb=8),
             # the headline shape: the 2 x 8 tile with other ring shapes
             dict(ta=2, tb=8, stages=3, rows=512), dict(ta=2, tb=8, stages=4, rows=384),
             dict(ta=2, tb=8, stages=10, rows=128), dict(ta=2, tb=8, stages=2, rows=768)],
    (16, 16): [dict(ta=4, tb=4), dict(ta=4, tb=8)],
    (32, 32): [dict(ta=8, tb=4), dict(cw=16)],
    (64, 64): [dict(unroll=2), dict(stages=4)],
}


def _round_rows(v) -> int:
    """Rows per chunk rounded down the way the default sizing rounds: whole
    passes of the row groups, every bulk copy a multiple of 16 bytes."""
    rg = v.cw * 32 // v.num_tiles
    e = v.epc
    rows = v.rows
    if rows >= rg:
        rows = rows // rg * rg
    return max(e, rows // e * e)


def default_variants() -> list:
    out: list = []
    # FP64 tensor-core kernels first: exact widths, contiguous or strided
    # operands with 16-byte row pitches.
    for wa in DMMA_WIDTHS:
        for wb in DMMA_WIDTHS:
            out.append(DmmaVariant(wa, wb))
    for wa, wb in EXACT_PAIRS:
        base = BulkVariant(wa, wb, default_tile(wa), default_tile(wb))
        out.append(base)
        for extra in EXTRA_CANDIDATES.get((wa, wb), []):
            out.append(dataclasses.replace(base, **extra))
        # Larger ring stages: 3 x ~64 KB, 4 x ~48 KB, 2 x ~96 KB instead of 6 x ~32 KB
        # (longer contiguous bulk copies; the 8 x 8 headline streamed 6.5 %
        # faster with 3 x 64 KB).
        rows = base.resolved().rows
        for stages, mult in ((3, 2.0), (4, 1.5), (2, 3.0)):
            v = dataclasses.replace(base, stages=stages, rows=int(rows * mult))
            v = dataclasses.replace(v, rows=_round_rows(v))
            if not v.validate() and v.name not in {u.name for u in out}:
                out.append(v)
    for wa in WIDTH_CAPS:
        for wb in WIDTH_CAPS:
            out.append(BulkVariant(wa, wb, default_tile(wa), default_tile(wb), exact=False))
    for wa in WIDTH_CAPS:
        for wb in WIDTH_CAPS:
            out.append(DirectVariant(wa, wb, default_tile(wa), default_tile(wb)))
    # FP32 storage (FP32 per-thread accumulation, FP64 reductions): exact
    # squares, then capacities, then direct loads, in the same order.
    # FP32 exact squares: 2 stages of three times the rows first, then 3
    # stages of twice the rows, then the 6-stage ones (the FP32 default is
    # the first applicable variant; in interleaved timings at n = 2^22-2^25,
    # 3 stages streamed 2-9 % faster than 6 and 2 stages up to 7 % faster
    # than 3).
    for stages, mult in ((2, 3), (3, 2)):
        for w in WIDTH_CAPS:
            g = BulkVariant(w, w, default_tile(w), default_tile(w), dtype="f32")
            v = dataclasses.replace(g, stages=stages, rows=mult * g.resolved().rows)
            v = dataclasses.replace(v, rows=_round_rows(v))
            if not v.validate():
                out.append(v)
    for w in WIDTH_CAPS:
        out.append(BulkVariant(w, w, default_tile(w), default_tile(w), dtype="f32"))
    for wa in WIDTH_CAPS:
        for wb in WIDTH_CAPS:
            out.append(BulkVariant(wa, wb, default_tile(wa), default_tile(wb), exact=False, dtype="f32"))
    for wa in WIDTH_CAPS:
        for wb in WIDTH_CAPS:
            out.append(DirectVariant(wa, wb, default_tile(wa), default_tile(wb), dtype="f32"))
    # Gram C = A^T A (A streamed once), last so that earlier indices stay put:
    # tensor cores for the DMMA widths, SIMT register tiles below 16.
    for w in DMMA_WIDTHS:
        out.append(DmmaVariant(w, w, gram=True))
    # SIMT Gram kernels, 2 stages of ~96 KB first, then 3 of ~64 KB, the
    # 6-stage ones last (the default takes the first applicable Gram variant;
    # in interleaved timings at n = 2^26, 3 stages streamed A 3-11 % faster
    # than 6 and 2 stages 1.5-8 % faster than 3).
    for stages, mult in ((2, 3), (3, 2)):
        for w in (1, 2, 4, 8):
            g = BulkVariant(w, w, default_tile(w), default_tile(w), gram=True)
            v = dataclasses.replace(g, stages=stages, rows=mult * g.resolved().rows)
            v = dataclasses.replace(v, rows=_round_rows(v))
            if not v.validate():
                out.append(v)
    for w in (1, 2, 4, 8):
        out.append(BulkVariant(w, w, default_tile(w), default_tile(w), gram=True))
    # FP64 tensor-core kernels with other ring shapes (autotuner candidates)
    for wa, rows, stages in ((16, 192, 4), (16, 128, 6), (32, 96, 4), (32, 192, 2), (32, 64, 6)):
        out.append(DmmaVariant(wa, wa, rows=rows, stages=stages))
    # Longer chunks for 16 x 16 (two tensor boxes per block and chunk): 2 x 96 KB
    # and 3 x 72 KB; the Gram kernel of width 16 with 2 x 96 KB and 3 x 64 KB.
    for rows, stages in ((384, 2), (288, 3)):
        out.append(DmmaVariant(16, 16, rows=rows, stages=stages))
    for rows, stages in ((768, 2), (512, 3)):
        out.append(DmmaVariant(16, 16, rows=rows, stages=stages, gram=True))
    # 64 x 64 (FP64-bound) on 2 x 96 KB as well as 3 x 64 KB.
    out.append(DmmaVariant(64, 64, rows=96, stages=2))
    # More consumer warps on the 2 x 96 KB rings (the Gram kernel of width 32
    # gained from 12): 32 x 32, 16 x 16 and 64 x 64 with 12.
    for w, rows, cw in ((32, 192, 12), (16, 384, 12), (64, 96, 12)):
        out.append(DmmaVariant(w, w, rows=rows, stages=2, cw=cw))
    # The wider Gram kernels (FP64- and HBM-bound at once) with 2 x 96 KB rings;
    # width 32 also with 12 consumer warps.
    for w, rows, cw in ((32, 384, 8), (32, 384, 12), (48, 256, 0), (64, 192, 0), (48, 240, 12), (64, 192, 12)):
        out.append(DmmaVariant(w, w, rows=rows, stages=2, cw=cw, gram=True))
    return out


def check_variants(vs: Iterable) -> None:
    names = set()
    for v in vs:
        errs = v.validate()
        if errs:
            raise ValueError(f"{v.name}: {'; '.join(errs)}")
        if v.name in names:
            raise ValueError(f"duplicate variant {v.name}")
        names.add(v.name)


BATCHED_PATHS = {"dmma": 0, "simt": 1}


def load_tuned_batched(path: str = TUNED_JSON) -> list[tuple[int, int, int]]:
    """Tuned consumer path per width class of the batched kernel: list of
    (m, k, path), path 0 = the class's default (FP64 tensor cores for m, k
    >= 16), 1 = SIMT register tiles."""
    if not os.path.exists(path):
        return []
    with open(path) as f:
        doc = json.load(f)
    return sorted((int(e["m"]), int(e["k"]), BATCHED_PATHS[e["path"]]) for e in doc.get("batched_paths", []))


def load_tuned_gram(path: str = TUNED_JSON) -> list[tuple[int, int, str]]:
    """Tuned Gram variants (C = A^T A): list of (width, nmin, variant name)."""
    if not os.path.exists(path):
        return []
    with open(path) as f:
        doc = json.load(f)
    return sorted((int(e["w"]), int(e.get("nmin", 0)), str(e["variant"])) for e in doc.get("gram_choices", []))


def load_tuned(path: str = TUNED_JSON) -> list[tuple[int, int, int, str]]:
    """Tuned defaults: list of (m, k, nmin, variant name)."""
    if not os.path.exists(path):
        return []
    with open(path) as f:
        doc = json.load(f)
    rows = []
    for e in doc.get("choices", []):
        rows.append((int(e["m"]), int(e["k"]), int(e.get("nmin", 0)), str(e["variant"])))
    return sorted(rows)


HEADER = ("// Generated by tsm_benchmark_b200/codegen.py -- do not edit.\n"
          "// Regenerate with: python -m tsm_benchmark_b200.codegen\n")


def render(vs: list, tuned: list, parts: int = 8, batched_paths: list | None = None,
           gram: list | None = None) -> dict[str, str]:
    """Returns {file name: contents} for csrc/generated/."""
    if batched_paths is None:
        batched_paths = load_tuned_batched()
    if gram is None:
        gram = load_tuned_gram()
    check_variants(vs)
    known = {v.name for v in vs}
    for m, k, nmin, name in tuned:
        if name not in known:
            raise ValueError(f"tuned choice {name} for ({m},{k}) is not a variant")
    grams = {v.name for v in vs if getattr(v, "gram", False)}
    for w, nmin, name in gram:
        if name not in grams:
            raise ValueError(f"tuned Gram choice {name} for width {w} is not a Gram variant")
    files: dict[str, str] = {}
    chunks = [vs[i::parts] for i in range(parts)]
    # Keep table order global: part i holds rows i, i+parts, ...; the index
    # below re-interleaves them so the library sees the list order above.
    for i, chunk in enumerate(chunks):
        body = [HEADER, '#include "../tsm_registry.cuh"', "", "namespace tsm {", ""]
        body.append(f"extern const Variant kGenPart{i}[];")
        body.append(f"const Variant kGenPart{i}[] = {{")
        for v in chunk:
            body.append(f"    {v.emit()},")
        body.append("};")
        body.append(f"extern const int kGenPart{i}Count;")
        body.append(f"const int kGenPart{i}Count = {len(chunk)};")
        body.append("")
        body.append("}  // namespace tsm")
        files[f"variants_p{i}.cu"] = "\n".join(body) + "\n"

    idx = [HEADER, '#include "../tsm_registry.cuh"', "", "namespace tsm {", ""]
    for i in range(parts):
        idx.append(f"extern const Variant kGenPart{i}[];")
    idx.append("")
    # One single-row part per variant, in list order.
    idx.append("const VariantPart kVariantParts[] = {")
    for j in range(len(vs)):
        idx.append(f"    {{kGenPart{j % parts} + {j // parts}, 1}},")
    idx.append("};")
    idx.append(f"const int kVariantPartCount = {len(vs)};")
    idx.append("")
    idx.append("// Tuned defaults: \"m k nmin variant\" (largest nmin <= n wins).")
    idx.append("extern const char* const kTunedDefaults[];")
    idx.append("const char* const kTunedDefaults[] = {")
    for m, k, nmin, name in tuned:
        idx.append(f'    "{m} {k} {nmin} {name}",')
    idx.append("    nullptr};")
    idx.append("extern const int kTunedDefaultCount;")
    idx.append(f"const int kTunedDefaultCount = {len(tuned)};")
    idx.append("")
    idx.append("// Tuned consumer paths of the batched kernel: \"m k path\" (0 tensor cores, 1 SIMT).")
    idx.append("extern const char* const kTunedBatchedPaths[];")
    idx.append("const char* const kTunedBatchedPaths[] = {")
    for m, k, path in batched_paths:
        idx.append(f'    "{m} {k} {path}",')
    idx.append("    nullptr};")
    idx.append("extern const int kTunedBatchedPathCount;")
    idx.append(f"const int kTunedBatchedPathCount = {len(batched_paths)};")
    idx.append("")
    idx.append("// Tuned Gram variants (C = A^T A): \"w nmin variant\" (largest nmin <= n wins).")
    idx.append("extern const char* const kTunedGram[];")
    idx.append("const char* const kTunedGram[] = {")
    for w, nmin, name in gram:
        idx.append(f'    "{w} {nmin} {name}",')
    idx.append("    nullptr};")
    idx.append("extern const int kTunedGramCount;")
    idx.append(f"const int kTunedGramCount = {len(gram)};")
    idx.append("")
    idx.append("}  // namespace tsm")
    files["variants_index.cu"] = "\n".join(idx) + "\n"
    return files


COMPAT_HEADER = os.path.join(HERE, "compat", "tsmttsm_kernels.hh")

# The four kernel names the reference generators emit per (M, TM), as
# (prefetch, reduction-optimised) options, with the benchmark labels their
# harnesses print: v2 sycl_codegen_new.py:153,257 (basic, _lf, _sg, _sg_lf);
# v1 sycl_codegen.py:38-44 (_tr, _lf_tr, _2l_tr, _lf_2l_tr).
DROPIN_STYLES = {
    "v2": [("", False, False, "basic"), ("_lf", True, False, "lf"), ("_sg", False, True, "sg"),
           ("_sg_lf", True, True, "sg_lf")],
    "v1": [("_tr", False, False, "basic"), ("_lf_tr", True, False, "leapfrog"), ("_2l_tr", False, True, "2level"),
           ("_lf_2l_tr", True, True, "all")],
}


def dropin_name(style: str, m: int, tm: int, suffix: str) -> str:
    base = f"tsmttsm_gen_{m}_{m}_{tm}_{tm}" if style == "v1" else f"tsmttsm_{m}_{m}_{tm}_{tm}"
    return base + suffix


def _covers(v, m: int) -> bool:
    return (v.wa, v.wb) == (m, m) if v.exact else (v.wa >= m and v.wb >= m)


def pick_dropin_variant(vs: list, m: int, tm: int, prefetch: bool, reduce_opt: bool, local_size: int = 256,
                        unroll: int = 1, tuned: list | None = None) -> tuple[str | None, str]:
    """The compiled FP64 variant a generated drop-in kernel runs, and why.

    The reference's options map onto this library's axes as follows:
      * TM -> the SIMT register tile TM x TM (the nearest compiled tile);
      * leap-frog prefetch (_lf) -> the shared-memory ring: without it the
        deepest compiled ring (many short bulk copies in flight), with it the
        shallowest (a double buffer of long copies, the leap-frog's analogue);
      * the reduction-optimised kernels (_sg / _2l) -> the autotuned choice
        for (M, M, K) (FP64 tensor cores for widths 16..64), and with _lf the
        tensor-core kernel's shallowest ring that is not one of the tuned
        choices for (M, M) (so the two names time different kernels), or
        the SIMT tile's middle ring below width 16;
      * local_size -> consumer warps (local_size / 32) and --unroll -> the
        row-loop unroll, where such a variant is compiled.
    None means the library's autotuned default at run time."""
    if reduce_opt and not prefetch:
        return None, "chosen per (M, M, K) at run time; every kernel reduces with the two-level sum"
    simt = [v for v in vs if isinstance(v, BulkVariant) and v.dtype == "f64" and not v.gram and _covers(v, m)
            and v.ta == v.tb]
    if reduce_opt and prefetch:
        dm = [v.resolved() for v in vs if isinstance(v, DmmaVariant) and not v.gram and (v.wa, v.wb) == (m, m)]
        if dm:
            tuned_names = {name for tm_, tk_, _, name in (load_tuned() if tuned is None else tuned)
                           if (tm_, tk_) == (m, m)}
            order = sorted(dm, key=lambda d: (d.stages, -d.rows))
            v = next((d for d in order if d.name not in tuned_names), order[0])
            why = "FP64 tensor cores, shallowest ring"
            if v is not order[0]:
                why += " other than the autotuned choice"
            elif v.name in tuned_names:
                why += " (an autotuned choice too: every ring compiled for this width is one for some row count)"
            return v.name, why
    if not simt:
        return None, "no SIMT tile compiled for this width: the autotuned default"
    exact = [v for v in simt if v.exact]
    if exact:
        pool = exact
    else:  # the smallest capacity that covers the width
        cap = min(v.wa for v in simt)
        pool = [v for v in simt if v.wa == cap and v.wb == cap]

    def tile_gap(v):
        return abs(math.log2(v.ta) - math.log2(tm))

    best_gap = min(tile_gap(v) for v in pool)
    pool = [v for v in pool if tile_gap(v) == best_gap]
    notes = []
    if best_gap:
        notes.append(f"no {tm}x{tm} tile compiled for width {m}: nearest tile {pool[0].ta}x{pool[0].ta}")
    for axis, want, label in (("cw", local_size // 32, "local_size"), ("unroll", unroll, "unroll")):
        hit = [v for v in pool if getattr(v, axis) == want]
        if hit:
            pool = hit
        elif (axis == "cw" and want != 8) or (axis == "unroll" and want != 1):
            notes.append(f"{label} {want * 32 if axis == 'cw' else want} not compiled for this tile")
    if reduce_opt and prefetch:  # below width 16: the middle ring of the SIMT tile
        depths = sorted({v.resolved().stages for v in pool})
        want = depths[len(depths) // 2]
        v = [u for u in pool if u.resolved().stages == want][0]
        notes.insert(0, "SIMT tile, middle ring depth")
    else:
        key = (lambda u: (u.resolved().stages, -u.resolved().rows))
        v = min(pool, key=key) if prefetch else max(pool, key=key)
        notes.insert(0, "shallowest ring (double buffer)" if prefetch else "deepest ring")
    return v.name, "; ".join(notes)


def suggest_stride(widths, tiles, local_size: int, sg_size: int, target_groups: int = 2048) -> int:
    """The work-item count the v2 generator picks when --stride is omitted
    (sycl_codegen_new.py:561-580): the least common multiple of local_size
    and, per (M, TM), the tile count and sg_size x tile count, scaled to
    about `target_groups` work-groups."""
    req = local_size
    for m in widths:
        for tm in tiles:
            if m % tm:
                continue
            nt = (m // tm) ** 2
            req = math.lcm(req, nt, sg_size * nt)
    req = math.lcm(req, local_size)
    return max(1, -(-local_size * target_groups // req)) * req


def validate_launch(style: str, widths, tiles, stride: int, local_size: int, sg_size: int) -> list[str]:
    """The reference generators' launch checks (sycl_codegen.py:475-491,
    sycl_codegen_new.py:530-558, :609-611): returns the error lines; v1
    only warns about uneven tile distribution (printed, not returned)."""
    errs = []
    if sg_size != 32:
        errs.append(f"Error: --sg-size {sg_size}: the sub-group on B200 is the 32-thread warp")
    if local_size % 32:
        errs.append(f"Error: --local-size ({local_size}) must be a multiple of --sg-size (32)")
    if stride % local_size:
        errs.append(f"Error: --stride {stride} must be divisible by --local-size {local_size}")
        return errs
    for m in widths:
        if not 1 <= m <= 64:
            errs.append(f"Error: --M {m}: widths are 1..64")
            continue
        for tm in tiles:
            if m % tm:
                continue
            nt = (m // tm) ** 2
            if style == "v1":
                if stride % (nt * local_size):
                    print(f"Warning: --stride ({stride}) is not a multiple of num_tiles*local_size="
                          f"{nt * local_size} for M={m}, TM={tm}.", file=sys.stderr)
                continue
            if stride % nt:
                errs.append(f"Warning: stride ({stride}) not divisible by num_tiles ({nt}) for M={m}, TM={tm}"
                            "  [basic/lf kernels]")
            if (stride // sg_size) % nt:
                errs.append(f"Warning: stride/sg_size ({stride // sg_size}) not divisible by num_tiles ({nt}) "
                            f"for M={m}, TM={tm}  [sg kernels]")
    return errs


def render_dropin_header(vs: list, widths=(4, 8, 16), tiles=(2, 4), style: str = "v2", stride: int | None = None,
                         local_size: int | None = None, sg_size: int = 32, unroll: int = 1,
                         with_benchmark: bool = True) -> str:
    """The header the reference generators print, for this library:
    `sycl_codegen_new.py` (style v2: tsmttsm_{M}_{N}_{TM}_{TN}{,_lf,_sg,_sg_lf}
    (q, int K, const T* A, const T* B, T* C), :153-159,257-264) or
    `sycl_codegen.py` (style v1: tsmttsm_gen_{M}_{N}_{TM}_{TN}[_lf][_2l]_tr
    (q, int K, T* A, T* B, T* C), :38-63), plus run_all_benchmarks<T>(q, K,
    warmup, runs) (v2 :417-419, defaults 1 << 20, 10, 30; v1 :319, defaults
    1024 * 1024, 50, 100) with --with-benchmark.  Each kernel adds A^T B into
    C through tsm_gemm_tn_f64_launch: the variant pick_dropin_variant chose,
    on at most stride / local_size CTAs (the reference's work-groups)."""
    if local_size is None:
        local_size = 32 if style == "v1" else 256
    if stride is None:
        stride = 16384 if style == "v1" else suggest_stride(widths, tiles, local_size, sg_size)
    groups = stride // local_size
    const = "const " if style == "v2" else ""
    gen = "sycl_codegen.py" if style == "v1" else "sycl_codegen_new.py"
    out = [HEADER.rstrip("\n"), "//",
           f"// Drop-in for the header `{gen}` emits, on libtsm_b200.so.",
           "// Kernel names and signatures are the reference generator's; every kernel adds",
           "// A^T B into C through tsm_gemm_tn_f64_launch on the queue's stream, with a",
           "// compiled variant of this library (named above each kernel) on at most",
           "// stride / local_size CTAs.",
           f"//   widths {' '.join(map(str, widths))}; tiles {' '.join(map(str, tiles))}; stride={stride} "
           f"local_size={local_size} sg_size={sg_size} unroll={unroll}",
           "#pragma once", "", "#include <sycl/sycl.hpp>", "", "#include <vector>", "",
           '#include "tsm_compat_bench.hh"', '#include "tsmttsm.hh"', ""]
    for m in widths:
        out.append(f"// {'=' * 60}")
        out.append(f"// M = {m}")
        out.append(f"// {'=' * 60}")
        out.append("")
        for tm in tiles:
            if m % tm:
                continue
            picked = {}
            for suffix, prefetch, reduce_opt, _label in DROPIN_STYLES[style]:
                vname, why = pick_dropin_variant(vs, m, tm, prefetch, reduce_opt, local_size, unroll)
                fname = dropin_name(style, m, tm, suffix)
                if vname is not None and vname in picked:
                    why += f" (the same kernel as {picked[vname]}: no other ring compiled for this tile)"
                picked.setdefault(vname, fname)
                out.append(f"// runs {vname or 'the autotuned default'}: {why}")
                out.append("template <typename T>")
                out.append(f"sycl::event {fname}(sycl::queue& q, int K, {const}T* A, {const}T* B, T* C) {{")
                if vname:
                    out.append(f'  static const int variant = tsm_compat::variant_by_name("{vname}");')
                else:
                    out.append("  static const int variant = -1;")
                out.append(f"  return tsm_compat::accumulate_tn<T>(q, K, {m}, {m}, A, B, C, variant, {groups});")
                out.append("}")
                out.append("")
    if with_benchmark:
        k_default, warm, runs, rel = ("1024 * 1024", 50, 100, "1e-8") if style == "v1" else ("1 << 20", 10, 30, "1e-6")
        out.append("template <typename T>")
        out.append(f"void run_all_benchmarks(sycl::queue& q, int K = {k_default}, int warmup = {warm}, "
                   f"int runs = {runs}) {{")
        out.append('  std::cout << "Device: " << q.get_device().get_info<sycl::info::device::name>() << "\\n\\n";')
        out.append("  std::vector<tsm_compat::BenchResult> results;")
        for m in widths:
            out.append("  {")
            out.append(f"    tsm_compat::Problem<T> p(q, K, {m}, 123, {rel});")
            for tm in tiles:
                if m % tm:
                    continue
                for suffix, _p, _r, label in DROPIN_STYLES[style]:
                    fname = dropin_name(style, m, tm, suffix)
                    out.append(f'    results.push_back(p.bench("M{m}_T{tm}_{label}", '
                               f"[&](int k) {{ return {fname}<T>(q, k, p.A, p.B, p.C); }}, warmup, runs));")
            out.append("  }")
        out.append("  tsm_compat::print_results(results);")
        out.append("}")
        out.append("")
    out.append("// End of generated code")
    return "\n".join(out) + "\n"


def render_compat_header(vs: list) -> str:
    """compat/tsmttsm_kernels.hh: the v2 header with the reference
    generator's defaults (--M 4 8 16 --tile-sizes 2 4 --with-benchmark)."""
    return render_dropin_header(vs)


def write(files: dict[str, str], out_dir: str = GEN_DIR) -> None:
    os.makedirs(out_dir, exist_ok=True)
    for name, text in files.items():
        path = os.path.join(out_dir, name)
        old = open(path).read() if os.path.exists(path) else None
        if old != text:
            with open(path, "w") as f:
                f.write(text)
    for name in os.listdir(out_dir):
        if name.endswith(".cu") and name not in files:
            os.remove(os.path.join(out_dir, name))


def is_current(files: dict[str, str], out_dir: str = GEN_DIR) -> bool:
    for name, text in files.items():
        path = os.path.join(out_dir, name)
        if not os.path.exists(path) or open(path).read() != text:
            return False
    return True


REFERENCE_FLAGS = ("--M", "--tile-sizes", "--stride", "--local-size", "--sg-size", "--unroll", "--with-benchmark",
                   "--style")


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else list(argv)
    if any(a.split("=")[0] in REFERENCE_FLAGS for a in argv):
        return main_dropin(argv)
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--check", action="store_true", help="exit 1 if csrc/generated is stale")
    ap.add_argument("--list", action="store_true", help="print the variant names")
    ap.add_argument("--out", default=GEN_DIR, help="output directory")
    args = ap.parse_args(argv)
    vs = default_variants()
    files = render(vs, load_tuned())
    compat = render_compat_header(vs)
    if args.list:
        for v in vs:
            print(v.name)
        return 0
    if args.check:
        ok = is_current(files, args.out) and os.path.exists(COMPAT_HEADER) and open(COMPAT_HEADER).read() == compat
        print("generated kernels are", "current" if ok else "STALE")
        return 0 if ok else 1
    write(files, args.out)
    if not os.path.exists(COMPAT_HEADER) or open(COMPAT_HEADER).read() != compat:
        with open(COMPAT_HEADER, "w") as f:
            f.write(compat)
    print(f"wrote {len(files)} files, {len(vs)} variants, {len(load_tuned())} tuned choices, "
          f"{len(load_tuned_gram())} tuned Gram choices to {args.out}")
    return 0


def main_dropin(argv) -> int:
    """The reference generators' command line: prints the drop-in header on
    stdout, e.g. ``python -m tsm_benchmark_b200.codegen --M 4 8 16 32
    --tile-sizes 2 4 --with-benchmark > tsmttsm_kernels.hh`` (v2 names) or
    the same with ``--style v1``.  Flags and defaults as in
    sycl_codegen_new.py:587-603 (v2) and sycl_codegen.py:461-473 (v1)."""
    ap = argparse.ArgumentParser(description="Generate the drop-in tsmttsm_kernels.hh for libtsm_b200.so")
    ap.add_argument("--style", choices=("v1", "v2"), default="v2",
                    help="v2: sycl_codegen_new.py names (default); v1: sycl_codegen.py names")
    ap.add_argument("--M", type=int, nargs="+", default=[4, 8, 16], help="Matrix sizes (default: 4 8 16)")
    ap.add_argument("--tile-sizes", type=int, nargs="+", default=[2, 4], help="Tile sizes TM=TN (default: 2 4)")
    ap.add_argument("--stride", type=int, default=None,
                    help="Total work-item count (v1 default 16384; v2: auto-computed if omitted)")
    ap.add_argument("--local-size", type=int, default=None, help="Work-group size (v1 default 32, v2 256)")
    ap.add_argument("--sg-size", type=int, default=32, help="Sub-group size: the warp, 32")
    ap.add_argument("--unroll", type=int, default=1, help="Row-loop unroll factor (default: 1)")
    ap.add_argument("--with-benchmark", action="store_true", help="Append run_all_benchmarks<T>")
    args = ap.parse_args(argv)
    local = args.local_size if args.local_size is not None else (32 if args.style == "v1" else 256)
    stride = args.stride
    if stride is None:
        stride = 16384 if args.style == "v1" else suggest_stride(args.M, args.tile_sizes, local, args.sg_size)
    errs = validate_launch(args.style, args.M, args.tile_sizes, stride, local, args.sg_size)
    if errs:
        for e in errs:
            print(e, file=sys.stderr)
        return 1
    sys.stdout.write(render_dropin_header(default_variants(), args.M, args.tile_sizes, args.style, stride, local,
                                          args.sg_size, args.unroll, args.with_benchmark))
    return 0


if __name__ == "__main__":
    sys.exit(main())
