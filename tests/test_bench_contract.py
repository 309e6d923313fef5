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


def test_reference_arm_prints_the_gpu_arms_config_and_no_package_code():
    """Both arms print the same workload config (the GPU arm builds it with the same function),
    and the reference arm's process maps none of the package's own native libraries."""
    sys.path.insert(0, ROOT)
    import bench
    p = _run()
    assert p.returncode == 0, p.stderr[-2000:]
    out = json.loads([l for l in p.stdout.splitlines() if l.startswith("{")][0])
    import argparse
    ns = argparse.Namespace(gpus=1, spp_per_step=64)
    assert out["config"] == bench.workload_config(ns, 1920, 1080)
    if out["cpu_baseline"]["kind"] == "reference":
        assert out["impl_detail"]["package_native_code_loaded"] == []


def _best_rate(run, n, reps=3):
    return max(n / run(n) for _ in range(reps))


def test_cpu_baseline_keeps_every_core_after_the_flop_count():
    """The algorithmic FLOP count runs the counting oracle on one thread; the CPU baseline that
    follows it in the same process must still use every host core, at the rate a fresh process
    measures (within 20%)."""
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import bench
    from snelly_b200 import scenes
    from snelly_b200.testing import HostSnelly
    host = HostSnelly(scenes.DispersiveFractal())
    bench.flops_per_path(host)
    run, kind, team, keep = bench.cpu_sampler(host)
    n = 6000
    run(1000)
    after = _best_rate(run, n)
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    assert team() == cores, (team(), cores)
    code = ("import sys; sys.path.insert(0, %r); sys.path.insert(0, %r)\n"
            "import bench\nfrom snelly_b200 import scenes\nfrom snelly_b200.testing import HostSnelly\n"
            "run, kind, team, keep = bench.cpu_sampler(HostSnelly(scenes.DispersiveFractal()))\nrun(1000)\n"
            "print(max(%d / run(%d) for _ in range(3)))\n") % (ROOT, os.path.join(ROOT, "oracle"), n, n)
    p = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    fresh = float(p.stdout.strip().splitlines()[-1])
    assert after >= 0.8 * fresh, (after, fresh)
