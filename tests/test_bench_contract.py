"""The bench's reference arm runs on the host cores only, so its contract is
checked here on the CPU: one JSON line with the metric, the timing keys, a
cpu_baseline describing the run and an e2e block without host<->device bytes;
ranks other than 0 of a multi-process launch exit quietly; the forest's
reference run is reported unavailable."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench(args, **env):
    e = dict(os.environ, **env)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, env=e,
                          capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_one_json_line():
    r = _bench(["--impl", "reference", "--config", "plain-small", "--steps", "1", "--warmup", "1"])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == d["unit"] == "Msamples/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["scaling"] == "weak"
    assert d["steps"] == 1 and d["warmup"] == 1 and d["ms_per_step"] > 0
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert "workload" in d["config"]


def test_reference_arm_other_ranks_exit_quietly():
    r = _bench(["--impl", "reference", "--config", "plain-small", "--steps", "1", "--warmup", "1"],
               RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_forest_reference_is_reported_unavailable():
    r = _bench(["--impl", "reference", "--config", "forest"])
    assert r.returncode == 0
    d = json.loads(r.stdout.strip().splitlines()[-1])
    assert d["impl"] == "reference" and "unavailable" in d
