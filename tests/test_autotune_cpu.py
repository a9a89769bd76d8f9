"""Host logic of the autotuner (no GPU): which variants are candidates for a
shape, which candidates go to the interleaved refinement, how the winner is
decided and how a partial re-tune merges into an earlier table; and that the
committed tuned table names, for every shape, a variant that accepts it."""
import json
import os

from tests.conftest import ROOT


def test_candidates_follow_widths_and_dtype():
    from tsm_benchmark_b200 import variants
    from tsm_benchmark_b200.autotune import candidates
    vs = variants()
    for m, k in [(8, 8), (3, 5), (1, 64), (64, 64), (16, 16)]:
        got = candidates(vs, m, k)
        assert got, (m, k)
        for v in got:
            assert v["dtype"] == "f64" and not v["gram"], v["name"]
            if v["exact"]:
                assert (v["wa"], v["wb"]) == (m, k), v["name"]
            else:
                assert m <= v["wa"] and k <= v["wb"], v["name"]
        names = {v["name"] for v in got}
        # every exact variant of the pair, none of another width pair
        exact = {v["name"] for v in vs if v["exact"] and v["dtype"] == "f64" and not v["gram"]
                 and (v["wa"], v["wb"]) == (m, k)}
        assert exact <= names
    # capacities at most twice the smallest power of two per side: 3 x 5 takes
    # 4..8 x 8..16, never 64-wide capacity kernels
    for v in candidates(vs, 3, 5):
        assert not v["exact"] and v["wa"] in (4, 8) and v["wb"] in (8, 16), v["name"]
    assert all(v["dtype"] == "f32" for v in candidates(vs, 16, 16, dtype="f32"))


def test_refinement_set_and_median_winner():
    from tsm_benchmark_b200.autotune import median_winner, refinement_set
    row = {"a": {"ms": 1.00, "ok": True}, "b": {"ms": 1.04, "ok": True}, "c": {"ms": 1.049, "ok": True},
           "d": {"ms": 1.03, "ok": True}, "e": {"ms": 0.50, "ok": False}, "f": {"ms": 1.20, "ok": True}}
    # the wrong result is never a candidate, however fast; at most three, within 5 %
    assert refinement_set(row) == ["a", "d", "b"]
    assert refinement_set({"x": {"ms": 1.0, "ok": True}, "y": {"ms": 1.06, "ok": True}}) == ["x"]
    assert refinement_set({"x": {"ms": 1.0, "ok": False}}) == []
    assert refinement_set({}) == []
    # decided by the median, not by the single best sample
    win, med = median_winner({"a": [1.00, 1.30, 1.31], "b": [1.10, 1.11, 1.12]})
    assert win == "b" and med["a"] == 1.30
    win, _ = median_winner({"a": [1.0, 2.0], "b": [1.5, 1.5]})
    assert win == "a"  # equal medians: the first listed


def test_merge_keeps_other_pairs():
    from tsm_benchmark_b200.autotune import merge_results
    old = {"choices": [{"m": 8, "k": 8, "nmin": 0, "variant": "old8"},
                       {"m": 8, "k": 8, "nmin": 8388608, "variant": "old8big"},
                       {"m": 1, "k": 1, "nmin": 0, "variant": "old1"}],
           "timings": {"8x8@32768": {"old8": {}}, "1x1@32768": {"old1": {}}}}
    res = {"device": "d", "choices": [{"m": 8, "k": 8, "nmin": 8388608, "variant": "new8big"},
                                      {"m": 8, "k": 8, "nmin": 0, "variant": "new8"}],
           "timings": {"8x8@67108864": {"new8big": {}}}}
    out = merge_results(old, res, [(8, 8)])
    assert [c["variant"] for c in out["choices"]] == ["old1", "new8", "new8big"]
    assert set(out["timings"]) == {"1x1@32768", "8x8@67108864"}  # the re-tuned pair's old timings go
    assert out["device"] == "d" and res["choices"][0]["variant"] == "new8big"  # inputs untouched


def test_committed_tuned_table_is_consistent():
    from tsm_benchmark_b200 import variants
    from tsm_benchmark_b200.autotune import BUCKETS, candidates
    with open(os.path.join(ROOT, "tsm_benchmark_b200", "tuned.json")) as f:
        doc = json.load(f)
    vs = variants()
    seen = set()
    nmins = {b[0] for b in BUCKETS}
    for c in doc["choices"]:
        m, k, nmin = int(c["m"]), int(c["k"]), int(c["nmin"])
        assert (m, k, nmin) not in seen, c
        seen.add((m, k, nmin))
        assert nmin in nmins, c
        assert c["variant"] in {v["name"] for v in candidates(vs, m, k)}, c
    # every sweep shape has an entry for the headline bucket
    from tsm_benchmark_b200.autotune import SWEEP_PAIRS
    for m, k in SWEEP_PAIRS:
        assert (m, k, BUCKETS[-1][0]) in seen, (m, k)


def test_batched_paths_reach_the_generated_table(tmp_path):
    """tuned.json's batched_paths become the library's per-class table
    (kTunedBatchedPaths in csrc/generated/variants_index.cu): 0 for the
    tensor cores, 1 for SIMT register tiles."""
    import json

    from tsm_benchmark_b200 import codegen
    doc = {"choices": [], "batched_paths": [{"m": 16, "k": 16, "path": "simt"}, {"m": 32, "k": 32, "path": "dmma"}]}
    path = tmp_path / "tuned.json"
    path.write_text(json.dumps(doc))
    assert codegen.load_tuned_batched(str(path)) == [(16, 16, 1), (32, 32, 0)]
    files = codegen.render(codegen.default_variants(), [], batched_paths=codegen.load_tuned_batched(str(path)))
    idx = files["variants_index.cu"]
    assert '"16 16 1",' in idx and '"32 32 0",' in idx and "kTunedBatchedPathCount = 2;" in idx


def test_gram_choices_reach_the_generated_table(tmp_path):
    """tuned.json's gram_choices become the library's Gram table (kTunedGram
    in csrc/generated/variants_index.cu); a name that is not a Gram variant
    is rejected."""
    import json

    import pytest

    from tsm_benchmark_b200 import codegen
    doc = {"choices": [], "gram_choices": [{"w": 16, "nmin": 8388608, "variant": "dmma_16x16_gram_w8_s2_r768"},
                                           {"w": 16, "nmin": 0, "variant": "dmma_16x16_gram_w8_s4_r256"}]}
    path = tmp_path / "tuned.json"
    path.write_text(json.dumps(doc))
    gram = codegen.load_tuned_gram(str(path))
    assert gram == [(16, 0, "dmma_16x16_gram_w8_s4_r256"), (16, 8388608, "dmma_16x16_gram_w8_s2_r768")]
    files = codegen.render(codegen.default_variants(), [], batched_paths=[], gram=gram)
    idx = files["variants_index.cu"]
    assert '"16 8388608 dmma_16x16_gram_w8_s2_r768",' in idx and "kTunedGramCount = 2;" in idx
    with pytest.raises(ValueError, match="not a Gram variant"):
        codegen.render(codegen.default_variants(), [], batched_paths=[], gram=[(16, 0, "dmma_16x16_t16x16_w8_s2_r384")])


def test_gram_candidates():
    """Gram candidates: Gram variants only, exact ones of the width, capacity
    ones up to twice the smallest capacity; every width of the tuner has one."""
    from tsm_benchmark_b200.autotune import GRAM_WIDTHS, gram_candidates
    vs = [
        {"name": "g16a", "gram": True, "dtype": "f64", "exact": True, "wa": 16, "wb": 16},
        {"name": "g16b", "gram": True, "dtype": "f64", "exact": True, "wa": 16, "wb": 16},
        {"name": "p16", "gram": False, "dtype": "f64", "exact": True, "wa": 16, "wb": 16},
        {"name": "c8", "gram": True, "dtype": "f64", "exact": False, "wa": 8, "wb": 8},
        {"name": "c32", "gram": True, "dtype": "f64", "exact": False, "wa": 32, "wb": 32},
        {"name": "f16", "gram": True, "dtype": "f32", "exact": True, "wa": 16, "wb": 16},
    ]
    assert [v["name"] for v in gram_candidates(vs, 16)] == ["g16a", "g16b", "c32"]
    assert [v["name"] for v in gram_candidates(vs, 5)] == ["c8"]
    from tsm_benchmark_b200 import codegen
    real = [{"name": v.name, "gram": getattr(v, "gram", False), "dtype": v.dtype, "exact": v.exact,
             "wa": v.wa, "wb": v.wb} for v in codegen.default_variants()]
    for w in GRAM_WIDTHS:
        assert gram_candidates(real, w), w


def test_dmma_chunk_rows_rule():
    """DMMA chunks of more than 256 rows are split into equal tensor boxes of
    at most 256 rows, each a whole number of 8-row swizzle groups (the kernel's
    dmma_rows_ok); other row counts are rejected by the generator."""
    from tsm_benchmark_b200.codegen import DmmaVariant
    ok = [DmmaVariant(16, 16, rows=384, stages=2), DmmaVariant(16, 16, rows=288, stages=3),
          DmmaVariant(16, 16, rows=768, stages=2, gram=True), DmmaVariant(32, 32, rows=192, stages=2)]
    for v in ok:
        assert v.validate() == [], v.name
    bad = [DmmaVariant(16, 16, rows=264, stages=2),   # two boxes of 132 rows: not whole 8-row groups
           DmmaVariant(16, 16, rows=300, stages=2),   # not a multiple of 8
           DmmaVariant(16, 16, rows=1032, stages=1)]  # above 1024
    for v in bad:
        assert any("chunk rows" in e for e in v.validate()), v.rows


def test_modes_keep_each_others_sections():
    """A plain tuning rewrites choices and timings and keeps the batched paths
    and the Gram table of the file it replaces; merging one pair keeps the
    other pairs' choices."""
    from tsm_benchmark_b200.autotune import keep_sections, merge_results
    old = {"choices": [{"m": 8, "k": 8, "nmin": 0, "variant": "a"}, {"m": 16, "k": 16, "nmin": 0, "variant": "b"}],
           "timings": {"8x8@1": {}, "16x16@1": {}},
           "batched_paths": [{"m": 16, "k": 16, "path": "dmma"}],
           "gram_choices": [{"w": 16, "nmin": 0, "variant": "g"}], "gram_timings": {"gram16@1": {}}}
    res = {"choices": [{"m": 16, "k": 16, "nmin": 0, "variant": "c"}], "timings": {"16x16@1": {"x": 1}}}
    merged = keep_sections(merge_results(old, res, [(16, 16)]), old)
    assert [(c["m"], c["variant"]) for c in merged["choices"]] == [(8, "a"), (16, "c")]
    assert merged["timings"]["16x16@1"] == {"x": 1} and "8x8@1" in merged["timings"]
    for key in ("batched_paths", "gram_choices", "gram_timings"):
        assert merged[key] == old[key], key
    # a section the new result carries is not overwritten by the old one
    assert keep_sections({"gram_choices": []}, old)["gram_choices"] == []
