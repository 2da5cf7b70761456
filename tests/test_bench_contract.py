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


def test_short_summaries_fit_the_kept_tail():
    """The JSON line ends with the short summaries of configs 1, 3, 4 and 5;
    with full-precision inputs they must fit well inside the last 1500
    characters of the line, which is what a log tail keeps."""
    sys.path.insert(0, ROOT)
    import json as _json

    import bench
    f = 1234567.891234567
    e2e = {"value": f, "unit": "u", "h2d_bytes_per_step": 536870912, "d2h_bytes_per_step": 268435456}
    cpu = {"value": f, "unit": "u", "cores": 128, "kind": "port", "sample": "x" * 200,
           "single_thread": {"value": f, "cores": 1, "sample": "y" * 100}}
    commit = {"bit_exact": True, "bit_exact_vs_oracle_sample": True,
              "speedup_tensor_vs_plain": f, "speedup_ntt_tensor_products_vs_plain": f, "cpu_baseline": cpu,
              **{k: {"ms_per_batch": f, "value": f, "e2e": e2e} for k in ("plain", "tensor", "ntt_tensor_products")}}
    commit["tensor"]["roofline"] = {"frac": f, "achieved": f, "peak": f}
    fold = {"m": 1048576, "forms_agree": True, "cpu_baseline": cpu,
            "graph": {"ms_per_step": f, "value": f, "e2e": e2e}, "eager": {"ms_per_step": f},
            "graph_int64_products": {"ms_per_step": f}}
    uneven = {"jobs": 512, "sum_n": 24000000, "speedup_batch_vs_one_by_one": f, "cpu_baseline": cpu,
              "one_by_one": {"ms": f}, "batch": {"ms": f, "value": f, "bit_exact_vs_one_by_one": True, "e2e": e2e}}
    single = {"device_us_per_commit": f, "e2e_us_per_commit": f, "cpu_baseline": {"value": f}}
    tail = {"single_commit": bench.compact_single(single), "uneven_batch": bench.compact_uneven(uneven),
            "fold": bench.compact_fold(fold), "commit": bench.compact_commit(commit)}
    s = _json.dumps(tail)
    assert len(s) < 1400, len(s)
    c = tail["commit"]
    assert c["plain"]["v"] == 1235000.0 and c["int8_roofline"]["frac"] == 1230000.0
    assert c["cpu"]["1t"] and c["cpu"]["all"] and tail["fold"]["cpu"]["1t"] and tail["uneven_batch"]["cpu"]["1t"]
    assert bench.compact_commit(None) is None and bench.compact_fold({}) is None


def test_compact_summaries_close_the_line():
    """The short summaries of configs 1, 3, 4 and 5 that end the GPU arm's
    line keep their keys with a leg missing or partly filled, and round the
    figures to a few significant digits."""
    sys.path.insert(0, ROOT)
    import bench
    for fn in (bench.compact_commit, bench.compact_fold, bench.compact_uneven, bench.compact_single):
        assert fn(None) is None
    c = bench.compact_commit({"bit_exact": True, "plain": {"ms_per_batch": 7.531234, "value": 1.114e9,
                                                            "e2e": {"value": 4.838e8, "h2d_bytes_per_step": 1,
                                                                    "d2h_bytes_per_step": 2}},
                              "speedup_ntt_tensor_products_vs_plain": 4.2543})
    assert c["plain"] == {"ms": 7.531, "v": 1.114e9, "e2e": 4.838e8}
    assert c["ntt_tensor"] == {"ms": None, "v": None, "e2e": None}
    assert c["ntt_tensor_vs_plain"] == 4.25 and c["e2e_bytes"] == {"h2d": 1, "d2h": 2} and c["cpu"] is None
    f = bench.compact_fold({"m": 1 << 20, "graph": {"ms_per_step": 3.66412}, "forms_agree": True})
    assert f["ms"] == 3.664 and f["eager_ms"] is None and f["forms_agree"] is True
    u = bench.compact_uneven({"jobs": 512, "batch": {"ms": 48.5512, "bit_exact_vs_one_by_one": True}})
    assert u["batch_ms"] == 48.55 and u["bit_exact"] is True and u["one_by_one_ms"] is None
    s = bench.compact_single({"device_us_per_commit": 13.61, "e2e_us_per_commit": 30.64})
    assert s == {"device_us": 13.6, "e2e_us": 30.6, "cpu_1t_us": None}
    assert len(json.dumps({"commit": c, "fold": f, "uneven_batch": u, "single_commit": s})) < 1500
