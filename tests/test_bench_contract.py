"""bench.py's output contract, on the CPU: the reference arm (the oracle port
timed on the host cores) prints one JSON line with the keys the contract
names, only on rank 0; the clock sampler's summary of nvidia-smi rows."""
import json
import os
import subprocess
import sys
import threading

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _run(env_extra, *args):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], env=env, cwd=ROOT,
                          capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_one_contract_line():
    p = _run({}, "--impl", "reference", "--steps", "1", "--warmup", "1")
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "rays/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 1
    assert d["config"]["workload"] == "shapes-1M-800x800-100views"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert abs(d["ms_per_step"] - d["config"]["rays_per_step"] / d["value"] * 1e3) < 1e-6 * d["ms_per_step"]


def test_reference_arm_is_silent_on_other_ranks():
    p = _run({"RANK": "1", "WORLD_SIZE": "2"}, "--impl", "reference", "--steps", "1", "--warmup", "1")
    assert p.returncode == 0 and p.stdout.strip() == ""


def test_clock_sampler_summary():
    import bench
    cs = bench.ClockSampler(0)
    cs.proc = subprocess.Popen([sys.executable, "-c", "import time; time.sleep(30)"])
    cs.thread = threading.Thread(target=lambda: None)
    cs.thread.start()
    cs.rows = [["1965", "1965", "700.1", "0x0", "Not Active", "Not Active", "Not Active", "Not Active"],
               ["1800", "1965", "990.5", "0x4", "Not Active", "Not Active", "Not Active", "Active"],
               ["1900", "1965", "950.0", "0x4", "Not Active", "Not Active", "Not Active", "Active"],
               ["[N/A]", "1965", "950.0", "0x0", "Not Active", "Not Active", "Not Active", "Not Active"]]
    s = cs.stop()
    assert s["sm_mhz"] == 1900.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"] and s["samples"] == 4


def test_clock_sampler_without_nvidia_smi(monkeypatch):
    import bench

    def no_smi(*a, **k):
        raise OSError("no nvidia-smi")

    monkeypatch.setattr(bench.subprocess, "Popen", no_smi)
    cs = bench.ClockSampler(0)
    cs.start()
    assert cs.stop() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
