"""bench.py --impl reference: the CPU arm that times the reference's solver (the oracle port, since
the reference cannot be built here) on the host cores. It needs no GPU, so its output line is checked
here: the same metric, unit and config as the GPU arm, a cpu_baseline describing the run, and an e2e
entry with no host-device traffic. Under a multi-rank launch only rank 0 works and prints."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(extra_env=None):
    env = dict(os.environ)
    env.update(extra_env or {})
    # the 500-camera workload keeps the CPU sample short (the default workload is the 12M-observation one)
    return subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                           "--workload", "plane500"],
                          cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)


def test_reference_arm_prints_the_contract_line():
    r = _run()
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["unit"] == "LM iterations/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["ms_per_step"] > 0
    assert d["config"]["workload"].startswith("plane500")
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_without_work():
    r = _run({"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
