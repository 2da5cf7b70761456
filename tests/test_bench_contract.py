"""bench.py's reference arm on the CPU: one JSON line with the contract's keys.

`python bench.py --impl reference` times the reference's CPU path (the
oracle's restatement of NttTables::forward_fast / inverse_fast,
lattice-ring/src/ntt.rs:118-216) on the headline workload's metric and unit;
the driver compares it with the GPU arm's line, so both must name the same
metric, unit and direction.
"""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "1"], capture_output=True, text=True, cwd=ROOT, timeout=600, check=True).stdout
    lines = [l for l in out.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out
    line = json.loads(lines[0])
    sys.path.insert(0, ROOT)
    import bench
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["higher_is_better"] is True and line["steps"] == 1 and line["warmup"] == 1
    assert line["value"] > 0 and line["ms_per_step"] > 0
    assert line["vs_baseline"] is None
    assert isinstance(line["config"]["workload"], str) and line["config"]["workload"]
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == line["value"] and cb["unit"] == line["unit"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_do_no_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "1", "--gpus", "2"], capture_output=True, text=True, cwd=ROOT, env=env,
                         timeout=300, check=True).stdout
    assert not [l for l in out.splitlines() if l.startswith("{")]
