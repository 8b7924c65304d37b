"""bench.py's reference arm on the host cores: the JSON line the driver
reads (keys, units, impl) and the multi-rank rule (ranks other than 0 exit
0 without work).  CPU only; needs the reference's CPU path built into
oracle/_ref (skipped otherwise)."""
import json
import os
import subprocess
import sys

import pytest
from conftest import ROOT

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "ref_N5_B0")
needs_ref = pytest.mark.skipif(not os.path.exists(REF_BIN), reason="oracle/_ref not built")


def run_bench(*args, env=None):
    e = dict(os.environ, **(env or {}))
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT,
                          env=e, capture_output=True, text=True, timeout=600)


@needs_ref
def test_reference_arm_prints_one_contract_line():
    r = run_bench("--impl", "reference", "--steps", "1", "--warmup", "0")
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
    assert d["config"]["workload"].startswith("acoustic WADG LSRK45 step, N=5")


def test_reference_arm_other_ranks_exit_without_work():
    r = run_bench("--impl", "reference", "--steps", "1", "--warmup", "0",
                  env={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""


@pytest.mark.gpu
def test_bench_line_on_the_gpu(cuda):
    """A small run of the product arm: one JSON line with the roofline,
    end-to-end, launch-count and clock records."""
    r = run_bench("--steps", "2", "--warmup", "3", "--extra", "none", "--no-cpu-baseline",
                  "--hex", "8", "--variants", "nodal")
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    d = json.loads(lines[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config", "roofline",
              "e2e", "gpu_launches", "clocks"):
        assert k in d, k
    assert d["n_gpus"] == 1 and d["steps"] == 2 and d["warmup"] == 3 and d["value"] > 0
    assert d["gpu_launches"] == 6 * 2
    for k in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert k in d["roofline"], k
    assert d["e2e"]["h2d_bytes_per_step"] > 0 and d["e2e"]["d2h_bytes_per_step"] > 0
    assert "sm_mhz" in d["clocks"] and "reasons" in d["clocks"]
    assert d["precision"]["state"] == "fp32" and "contractions" in d["precision"]
