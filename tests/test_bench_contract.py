"""bench.py's reference arm on the CPU: it times the reference's own CPU
generator (extras/mcmcCPUgenThreaded.c, built into oracle/_ref) and prints
exactly one JSON line with the benchmark's keys; under torchrun only rank 0
runs it, the other ranks exit 0 without work."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _bench(args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([sys.executable, str(ROOT / "bench.py")] + args, capture_output=True, text=True,
                          timeout=600, cwd=ROOT, env=e)


def _json_lines(out):
    return [json.loads(x) for x in out.splitlines() if x.startswith("{")]


def test_reference_arm_prints_one_contract_line():
    p = _bench(["--impl", "reference", "--steps", "1", "--warmup", "3", "--cpu-seconds", "1"])
    assert p.returncode == 0, p.stderr[-2000:]
    lines = _json_lines(p.stdout)
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference"
    if "unavailable" in d:
        pytest.skip(d["unavailable"])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["metric"] == d["unit"] == "site-updates/s" and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] == 3 and d["n_gpus"] == 1 and d["value"] > 0
    assert d["config"]["workload"] and d["config"]["L"] == 232 and d["config"]["q"] == 21
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert "mcmcCPUgenThreaded.c" in cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_runs_on_rank_0_only():
    p = _bench(["--impl", "reference", "--steps", "1", "--warmup", "3", "--cpu-seconds", "1"],
               env={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert p.returncode == 0, p.stderr[-2000:]
    assert _json_lines(p.stdout) == []


def test_clock_summary_parses_nvidia_smi_rows():
    """The clocks record of the bench line: median SM clock under load, the
    maximum, and every throttle reason seen Active (rows as nvidia-smi
    prints them with --format=csv,noheader,nounits)."""
    sys.path.insert(0, str(ROOT))
    import bench
    cs = bench.ClockSampler(0)
    assert cs.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
    row = "0, {}, 1965, 812.40, 0x{}, {}, Not Active, Not Active, {}"
    for text in [row.format(1965, "0000000000000000", "Not Active", "Not Active"),
                 row.format(1950, "0000000000000004", "Not Active", "Active"),
                 row.format(1890, "0000000000000004", "Not Active", "Active"),
                 "0, [N/A], 1965, [N/A], [N/A], [N/A], [N/A], [N/A], [N/A]"]:
        cs.rows.append([x.strip() for x in text.split(",")])
    s = cs.summary()
    assert s["sm_mhz"] == 1950.0 and s["sm_max_mhz"] == 1965.0 and s["samples"] == 3
    assert s["reasons"] == ["sw_power_cap"]
    cs.rows.append([x.strip() for x in row.format(1500, "0000000000000048", "Active", "Not Active").split(",")])
    assert cs.summary()["reasons"] == ["hw_slowdown", "sw_power_cap"]
