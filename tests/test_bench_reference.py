"""bench.py's reference arm on the host cores: the JSON line it prints.

`bench.py --impl reference` times the reference's own CPU matcher (the TBB
matchers of src/matchtbb.cu built from the reference sources, or the oracle's
restatement where that build is absent) on the same workload, metric and unit
as the GPU arm.  It needs no GPU, so its output contract is checked here on a
small workload; under torchrun only rank 0 runs and prints.  The GPU arm's
clocks object is checked on given nvidia-smi lines.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _run(extra_env=None):
    env = {**os.environ, **(extra_env or {})}
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--workload",
                           "grid512_random_maximal", "--steps", "2", "--warmup", "3"],
                          cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_one_line():
    p = _run()
    assert p.returncode == 0, p.stderr
    lines = [x for x in p.stdout.splitlines() if x.strip()]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["unit"] == "edges/s" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["steps"] == 2 and line["warmup"] == 3 and line["n_gpus"] == 1
    assert line["config"]["workload"] == "grid512_random_maximal" and line["config"]["type"] == 7
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert cb["matcher"] == "GraphMatchingTBBRandom"
    assert line["e2e"] == {"value": line["value"], "unit": "edges/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    p = _run({"WORLD_SIZE": "2", "RANK": "1", "LOCAL_RANK": "1"})
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""


def test_clock_summary_reads_nvidia_smi_lines():
    """The bench line's clocks object from nvidia-smi's CSV samples: median SM
    clock, the maximum, and every throttle reason seen active."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    c = bench.ClockSampler(0)
    c.lines = ["0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
               "0, 1800, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
               "0, 1965, 1965, 710.0, 0x0, Not Active, Not Active, Not Active, Not Active",
               "[N/A]", ""]
    s = c.summary()
    assert s["samples"] == 3 and s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
    c.lines.append("0, 1200, 1965, 500.0, 0x48, Active, Not Active, Active, Not Active")
    assert c.summary()["reasons"] == ["hw_slowdown", "sw_power_cap", "sw_thermal_slowdown"]
    assert bench.ClockSampler(0).summary()["sm_mhz"] is None
