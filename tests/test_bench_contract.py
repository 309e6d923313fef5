"""bench.py's reference arm on the host CPU: the JSON line the benchmark contract asks for, and
the silent exit of ranks other than 0."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(extra_env=None):
    env = dict(os.environ)
    env.update(extra_env or {})
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2", "--warmup", "1",
           "--cpu-seconds", "1"]
    return subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_the_contract_line():
    p = _run()
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    out = json.loads(lines[0])
    assert out["impl"] == "reference" and out["metric"] == "spectral path samples/sec at 1080p"
    assert out["unit"] == "path samples/s" and out["higher_is_better"] is True
    assert out["value"] > 0 and out["steps"] == 2 and out["warmup"] == 1
    assert out["config"]["workload"] == "c1_dispersive_metallic_fractal_1080p"
    cb = out["cpu_baseline"]
    assert cb["value"] == out["value"] and cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    assert out["e2e"] == {"value": out["value"], "unit": "path samples/s", "h2d_bytes_per_step": 0,
                          "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_do_nothing():
    p = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert p.returncode == 0, p.stderr[-2000:]
    assert not [l for l in p.stdout.splitlines() if l.startswith("{")]
