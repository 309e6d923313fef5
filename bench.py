#!/usr/bin/env python
"""Benchmark: spectral path samples per second on the 1080p dispersive + metallic fractal workload.

Workload (one step = one full image: 64 progressive frames, i.e. 64 spectral path samples per
pixel, in one advance of the job; --spp-per-step changes it): a 5-iteration Menger sponge
(Cauchy dielectric, roughness 0.02), a tabulated-gold sphere and a diffuse ground plane under a
3-degree sun and a sky, 1920x1080, maxBounces 8, maxMarchSteps 512, dispersive, random-pose
camera drawn from seed 2.

Prints one JSON line (rank 0). `value`: path samples/s with all state resident on the device,
timed with CUDA events on the renderer's stream around each step, L2 flushed between steps,
max over ranks. `e2e`: the same through the public scene API with host buffers (per step:
parameter upload, the frame, and a device-to-host read of the whole mean image into page-locked
host memory, which overlaps the next step's frame), wall clock until every image is on the host.
`--impl reference` times the reference's own shader built for the host CPU
(oracle/_ref, else the oracle port) on a bounded pixel sample per step, all host threads.

`latency` (rank 0): the metric's second half, batched vs plain: the first --latency-jobs render
jobs of the heterogeneous batch draw (seed 4: 128^2..1024^2, four scenes, 4..64 spp), rendered
one after another through the single-job path and then all at once in batched launches, with
path samples/s and p50/p99 time to target spp (every job submitted at t = 0) for both.

Multi-GPU: replicas (one job per GPU, no collective): `value` sums all ranks' samples over the
slowest rank's time.
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "c1_dispersive_metallic_fractal_1080p"
METRIC = "spectral path samples/sec at 1080p"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=12)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", choices=["snelly", "reference"], default="snelly")
    ap.add_argument("--kernel", choices=["auto", "mega", "wavefront"], default="auto",
                    help="integrator (auto: the library's autotuner picks per scene and image size)")
    ap.add_argument("--spp-per-step", type=int, default=64,
                    help="frames (samples per pixel) rendered per step, as one advance of the job "
                         "(64: one full image of the workload)")
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="budget of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--latency-jobs", type=int, default=32,
                    help="jobs of the heterogeneous batch draw (seed 4) for the batched-vs-plain latency block "
                         "(0: skip it)")
    return ap.parse_args()


def workload_scene(args, seed_offset=0):
    from snelly_b200 import scenes
    return scenes.DispersiveFractal(args.width, args.height)


# ---------------------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------------------------
# CPU side: algorithmic FLOPs per path, CPU baseline
# ---------------------------------------------------------------------------------------------
def flops_per_path(host):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    return oracle.flops_per_path(host, pixels=1000, frames=2)


def cpu_sampler(host, prefer_reference=True):
    """A callable running `n` random pixels x `frames` frames of the workload on every host core
    (returns seconds), its kind ("reference": the reference's shader built for the CPU; "port":
    the oracle), and a callable giving the threads the last run used. With the prebuilt reference
    library nothing of the package's own native code is loaded: pixels are seeded by the numpy
    restatement."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    W, H = host.width, host.height
    rs = np.random.RandomState(11)
    ref = None
    if prefer_reference:
        try:
            import build_ref
            ref = build_ref.ref_for(host, name="bench_c1", prebuilt_only=not build_ref.have_reference())
        except Exception:
            ref = None
    if ref is not None:
        rlib, p, tables, keep = ref
        calls = host.scene_uniforms()

        def run(n, frames=1):
            pix = np.sort(rs.choice(W * H, n, replace=False))
            rng0 = oracle.seed_pixels(host.seed, pix)
            t = time.perf_counter()
            rlib.render(p, calls, tables, W, H, pix, frames, rng0, threads=0)
            return time.perf_counter() - t
        return run, "reference", rlib.last_team, (keep,)
    lib = oracle.OracleLib(host.sceneObj.shader(), host.scene_opts())
    p, keep = oracle.host_params(host)
    sh = host.scene_shader()
    ub = oracle.pack_uniforms(lib.cpp, sh.calls, sh.textures, params=p)

    def run(n, frames=1):
        pix = np.sort(rs.choice(W * H, n, replace=False))
        rng0 = oracle.seed_pixels(host.seed, pix)
        t = time.perf_counter()
        lib.render(p, ub, W, H, pix, frames, rng0, threads=0)
        return time.perf_counter() - t
    return run, "port", lib.last_team, (keep,)


def cpu_baseline(host, budget_s, frames=64):
    """The workload at its full spp (`frames` frames per pixel) on a random pixel sample sized to
    about `budget_s` seconds, every host core."""
    run, kind, team, keep = cpu_sampler(host)
    t = run(2000, frames)  # calibration at the full spp (a 1-frame sample runs faster per sample)
    rate = 2000 / max(t, 1e-6)
    n = int(min(host.width * host.height, max(64, rate * budget_s)))
    dt = run(n, frames)
    cores = team()
    return {"value": n * frames / dt, "unit": "path samples/s", "cores": cores, "kind": kind,
            "sample": f"{n} random pixels of the {host.width}x{host.height} workload, {frames} frames (its full spp) each "
                      f"({dt:.1f} s on {cores} host threads of {os.cpu_count()})"}


def workload_config(args, width, height):
    """The workload's definition, printed identically by both arms."""
    return {"workload": WORKLOAD, "width": width, "height": height, "spp_per_step": max(1, args.spp_per_step),
            "image_spp": 64, "max_bounces": 8, "max_march_steps": 512, "dispersive": True,
            "l2": "flushed between timed steps (256 MiB write); path state 0.77 GB > L2",
            "parallelism": f"replicas x{args.gpus}"}


def traffic_from_profiles(kernel_name):
    """DRAM bytes per launch of the frame kernel from the committed ncu summary, if any."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    for f in sorted(os.listdir(d)):
        if kernel_name in f and f.endswith(".md"):
            m = re.search(r"dram_bytes_per_launch_1080p:\s*([0-9.eE+]+)", open(os.path.join(d, f)).read())
            if m:
                return float(m.group(1))
    return None


# ---------------------------------------------------------------------------------------------
# the arms
# ---------------------------------------------------------------------------------------------
def reference_arm(args, rank):
    if rank != 0:
        return
    from snelly_b200.testing import HostSnelly
    host = HostSnelly(workload_scene(args))
    run, kind, team, keep = cpu_sampler(host)
    frames = max(1, args.spp_per_step)
    t = run(1000, frames)  # calibration at the step's spp
    rate = 1000 / max(t, 1e-6)  # pixels/s
    per_step = int(min(host.width * host.height, max(16, rate * args.cpu_seconds / max(1, args.steps))))
    for _ in range(args.warmup):
        run(min(per_step, 64), frames)
    times = [run(per_step, frames) for _ in range(args.steps)]
    value = per_step * frames * args.steps / sum(times)
    cores = team()
    sample = (f"{per_step} random pixels x {frames} frames (the step's full spp) per step of the {host.width}x{host.height} "
              f"workload (a bounded pixel sample of the step; {cores} host threads of {os.cpu_count()})")
    native = [l.split()[-1] for l in open("/proc/self/maps") if "libsnelly" in l] if os.path.exists("/proc/self/maps") else []
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "path samples/s", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * sum(times) / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (procedural SDF scene, seeded camera; no dataset)",
           "config": workload_config(args, host.width, host.height),
           "impl_detail": {"device": "host CPU", "program": "the reference's path tracer shader built for the CPU"
                           if kind == "reference" else "the oracle's restatement of the path tracer",
                           "package_native_code_loaded": sorted(set(native))},
           "cpu_baseline": {"value": value, "unit": "path samples/s", "cores": cores, "kind": kind,
                            "sample": sample},
           "e2e": {"value": value, "unit": "path samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def rank_max(dist, x):
    """The largest of every rank's x (each rank passes its own; dist None: one rank)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world, samples_per_step, steps, slowest_s):
    """Replicas (one job per GPU, no collective on the data path): every rank renders
    samples_per_step path samples per step, so the job renders world times that over the slowest
    rank's time."""
    return world * samples_per_step * steps / slowest_s


def gpu_arm(args, rank, world, local_rank):
    import ctypes

    import torch
    from snelly_b200 import _native as N
    from snelly_b200 import api
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()

    def allmax(x):
        return rank_max(dist, x)

    ctx = api.Context(local_rank)
    peak_tflops, _ = ctx.fp32_peak()
    s = api.Snelly(workload_scene(args), context=ctx)
    s.seed = 1 + rank
    s.pathtracer.maxSpp = 1 << 30  # progressive rendering never stops inside the benchmark
    s.pathtracer.kernelMode = {"auto": N.KERNEL_AUTO, "mega": N.KERNEL_MEGA, "wavefront": N.KERNEL_WAVEFRONT}[args.kernel]
    s.render(0)  # compile, allocate, seed (and, for --kernel auto, the autotuner's trial frames)
    kernel_used = "wavefront" if ctx.job_kernel(s.job_id()) == N.KERNEL_WAVEFRONT else "mega"
    wf_config = ctx.job_wavefront_config(s.job_id()) if kernel_used == "wavefront" else None
    W, H = s.width, s.height
    fps = max(1, args.spp_per_step)
    samples_per_step = W * H * int(round(s.pathtracer.maxSamplesPerFrame)) * fps
    stream = torch.cuda.ExternalStream(ctx.stream())
    jid = s.job_id()
    for _ in range(args.warmup):
        ctx.advance(jid, fps)
    ctx.sync()
    torch.cuda.synchronize()

    # ---- device-resident throughput ------------------------------------------------------------
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    launches0 = ctx.launch_count()
    for k in range(args.steps):
        ctx.flush_l2(256 << 20)  # evict L2 between timed steps (outside the events)
        starts[k].record(stream)
        ctx.advance(jid, fps)
        ends[k].record(stream)
    ctx.sync()
    torch.cuda.synchronize()
    barrier()
    launches = ctx.launch_count() - launches0 - args.steps  # minus the flushes
    clk = clocks.stop()
    step_ms = [a.elapsed_time(b) for a, b in zip(starts, ends)]
    total_ms = allmax(sum(step_ms))
    value = replica_throughput(world, samples_per_step, args.steps, total_ms / 1000.0)

    # ---- end to end through the public API ----------------------------------------------------
    # each step's image is read into one of two page-locked host buffers while the next step renders
    pinned = [torch.empty((H, W, 4), dtype=torch.float32, pin_memory=True).numpy() for _ in range(2)]
    h2d = ctypes.sizeof(N.SnellyParams) + max(4, len(s.scene_uniforms()) * 4)
    barrier()
    t0 = time.perf_counter()
    for k in range(args.steps):
        s.render(fps)
        s.readback(out=pinned[k % 2], wait=False)
    ctx.sync()  # every step's image is on the host
    e2e_s = allmax(time.perf_counter() - t0)
    e2e_value = replica_throughput(world, samples_per_step, args.steps, e2e_s)
    assert all(np.isfinite(p).all() for p in pinned)

    latency = None
    if rank == 0 and args.latency_jobs > 0:
        from snelly_b200 import batchbench
        jobs = batchbench.job_set(args.latency_jobs, 4)
        latency = {"workload": f"the first {args.latency_jobs} jobs of the heterogeneous batch draw (seed 4)"}
        latency.update(batchbench.measure(ctx, jobs))
    if rank == 0:
        from snelly_b200.testing import HostSnelly
        host = HostSnelly(workload_scene(args))
        fpp, spp_special, counted = flops_per_path(host)
        per_launch_ms = statistics.mean(step_ms)
        achieved = fpp * samples_per_step / (per_launch_ms / 1000.0) / 1e12
        kname = "pt_frame_mega" if kernel_used == "mega" else "pt_wavefront"
        frame_traffic = traffic_from_profiles(kname)  # DRAM bytes of one 1080p frame (ncu summary)
        cpu = None if args.no_cpu_baseline else cpu_baseline(host, args.cpu_seconds)
        out = {
            "metric": METRIC, "value": value, "unit": "path samples/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (procedural SDF scene, seeded camera; no dataset)",
            "config": workload_config(args, W, H),
            "impl_detail": {"device": "B200", "kernel": kernel_used, "kernel_choice": args.kernel, "math": "fast",
                            "wavefront_config": wf_config},
            "e2e": {"value": e2e_value, "unit": "path samples/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": W * H * 16},
            "gpu_launches": int(launches),
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak_tflops, "unit": "TFLOP/s",
                         "frac": achieved / peak_tflops, "traffic": frame_traffic * fps if frame_traffic else None,
                         "flops_per_path": fpp, "special_ops_per_path": spp_special,
                         "peak_source": "measured FFMA microbenchmark in this run (snelly_measure_fp32_peak)"},
            "clocks": clk,
            "cpu_baseline": cpu,
            "latency": latency,
        }
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        reference_arm(args, rank)
        return
    gpu_arm(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
