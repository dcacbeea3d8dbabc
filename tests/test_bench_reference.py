"""bench.py's reference arm runs on the host cores only (the oracle's FP64
integrators over a bounded sample of the served stream): its JSON line keeps
the benchmark contract, and under torchrun every rank but 0 exits without
work."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra):
    env = {**os.environ, **env_extra}
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "1", "--requests-per-step", "2", "--cpu-seconds", "1"],
                          capture_output=True, text=True, cwd=ROOT, env=env, timeout=600)


def test_reference_arm_prints_one_contract_line():
    r = _run({"WORLD_SIZE": "1", "RANK": "0"})
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "ray-steps/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 1
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["kind"] == "port"
    assert d["cpu_baseline"]["cores"] >= 1 and d["cpu_baseline"]["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "ray-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert d["metric"].startswith("ray-steps/s") and "workload" in d["config"]


def test_reference_arm_other_ranks_exit_quietly():
    r = _run({"WORLD_SIZE": "2", "RANK": "1"})
    assert r.returncode == 0 and r.stdout.strip() == ""
