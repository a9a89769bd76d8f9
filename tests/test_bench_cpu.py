"""The reference arm of bench.py (no GPU): `bench.py --impl reference` times
the reference's own tsmttsm4 on host threads and prints one JSON line with the
same metric, unit and workload as the GPU arm; under a multi-rank launch only
rank 0 prints it.  Run on a small row sample so the test takes seconds."""
import json
import os
import subprocess
import sys

from tests.conftest import ROOT

KEYS = {"metric", "impl", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
        "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"}


def _run(env_extra: dict) -> subprocess.CompletedProcess:
    env = dict(os.environ, **env_extra)
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2", "--warmup", "1",
           "--ref-rows", str(1 << 16), "--ref-budget", "5"]
    return subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)


def test_reference_arm_prints_one_contract_line():
    import bench
    p = _run({"RANK": "0", "WORLD_SIZE": "1"})
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, p.stdout
    line = json.loads(lines[0])
    assert KEYS <= set(line), KEYS - set(line)
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC
    assert line["unit"] == "GB/s" and line["higher_is_better"] is True and line["dtype"] == "f64"
    assert line["config"] == bench.workload_config(1)
    assert line["value"] > 0 and 1 <= line["steps"] <= 2
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert f"n={1 << 16} rows" in cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    # ms_per_step is the sample's bytes over the measured rate
    expect_ms = bench.algo_bytes(1 << 16, bench.HEAD_M, bench.HEAD_K) / line["value"] / 1e6
    assert abs(line["ms_per_step"] - expect_ms) <= 1e-9 * expect_ms


def test_reference_arm_other_ranks_exit_quietly():
    p = _run({"RANK": "1", "WORLD_SIZE": "2"})
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""


def test_algorithmic_bytes():
    import bench
    # A and B read once, C written once: 8 GiB + 512 B at the headline shape
    assert bench.algo_bytes(bench.HEAD_N, bench.HEAD_M, bench.HEAD_K) == (8 << 30) + 512
    assert bench.algo_bytes(0, 64, 64) == 8 * 64 * 64
