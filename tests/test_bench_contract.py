"""The benchmark's output contract, checked on the CPU through its reference arm (the crate's CG
loop on the oracle's operator; no GPU code runs in that arm): one JSON line with the metric, unit,
step counts, the CPU baseline and the end-to-end block, `unavailable` for the depth-12 workload,
and silence on ranks other than 0."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench(*args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True,
                       env=e, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    return [json.loads(line) for line in r.stdout.splitlines() if line.startswith("{")]


def test_reference_arm_line():
    sys.path.insert(0, ROOT)
    import bench
    lines = _bench("--impl", "reference", "--points", "20000", "--depth", "5", "--steps", "2", "--warmup", "1")
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC
    assert d["unit"] == "points/s" and d["higher_is_better"] is True and d["value"] > 0
    assert d["steps"] == 2 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["config"]["depth"] == 5 and d["config"]["points"] == 20000
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and "extrapolat" not in cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_large_workload_is_unavailable():
    lines = _bench("--impl", "reference", "--config", "5")
    assert len(lines) == 1 and lines[0]["impl"] == "reference" and "unavailable" in lines[0]


def test_reference_arm_other_ranks_print_nothing():
    env = {"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"}
    assert _bench("--impl", "reference", "--points", "20000", "--depth", "5", "--steps", "1", "--warmup", "1",
                  env=env) == []
