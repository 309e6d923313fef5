"""Heterogeneous batch benchmark: 256 render jobs, each run alone and then all in batched launches.

The job set is drawn from one seed: square resolutions log-uniform in [128, 1024], scenes uniform
over {plain sphere, dispersive fractal, volumetric/subsurface Mandelbox, mesh-like distance grid},
spp uniform in {4..64}, bounce limits uniform in {4..12}, camera poses on a sphere of radius
U(4, 8) looking at the origin.

* plain: the single-job path, one job after another: render(spp) then read the image back.
* batched: every job resident at once; each tick advances all unfinished jobs by up to 8 frames
  with snelly_advance_batch (the autotuner's wavefront jobs run concurrently as pixel ranges on
  their own streams; the rest share path-per-thread launches per scene module, modules on separate
  streams), and a job is read back when it reaches its spp.
Both use the autotuner's integrator and launch configuration per (scene, image-size class).

`python -m snelly_b200.batchbench` prints one JSON line: path samples per second of both, their
ratio, per-job time-to-target percentiles of both (every job submitted at t = 0), and a check that
the images are the same in both runs.
"""
import argparse
import json
import math
import time

import numpy as np

from . import _native as N
from . import api
from .serving import posed_scene

SCENE_NAMES = ("c0", "c1", "c2", "mesh")


def job_set(n=256, seed=4, res_range=(128, 1024), spp_range=(4, 64)):
    rs = np.random.RandomState(seed)
    jobs = []
    for k in range(n):
        res = int(round(math.exp(rs.uniform(math.log(res_range[0]), math.log(res_range[1])))))
        name = SCENE_NAMES[rs.randint(len(SCENE_NAMES))]
        scene = posed_scene(name, res, rs)
        spp = int(rs.randint(spp_range[0], spp_range[1] + 1))
        jobs.append({"id": k, "scene": scene, "name": name, "res": res, "spp": spp, "seed": 1000 + k})
    return jobs


def _snelly(ctx, job, kernel):
    s = api.Snelly(job["scene"], context=ctx)
    s.seed = job["seed"]
    s.pathtracer.kernelMode = kernel
    return s


def warm(ctx, jobs, kernel):
    """Compile every scene module and run the autotuner for every (scene, size class) before the
    clock starts, as a long-running renderer would have."""
    seen = set()
    for j in jobs:
        key = (j["name"], int(round(math.log2(j["res"] * j["res"]))))
        if key in seen:
            continue
        seen.add(key)
        s = _snelly(ctx, j, kernel)
        s.render(1)
        s.readback()
        ctx.destroy_job(s.job_id())


def run_plain(ctx, jobs, kernel, keep=None):
    """One job after another through the single-job path; returns (path samples, seconds, per-job
    times to target measured from the start)."""
    ctx.sync()
    t0 = time.perf_counter()
    samples, done_at = 0, []
    for j in jobs:
        s = _snelly(ctx, j, kernel)
        s.render(j["spp"])
        img = s.readback()
        samples += s.width * s.height * j["spp"]
        done_at.append(time.perf_counter() - t0)
        if keep is not None:
            keep[j["id"]] = img
        ctx.destroy_job(s.job_id())
    return samples, time.perf_counter() - t0, np.array(done_at)


def run_batched(ctx, jobs, kernel=N.KERNEL_AUTO, frames_per_tick=8, keep=None):
    """Every job resident at once. Each tick advances every unfinished job by up to
    `frames_per_tick` frames in one snelly_advance_batch call (the autotuner's wavefront jobs as
    concurrent pixel ranges on their own streams, the rest in shared path-per-thread launches per
    scene module); a job is read back once it reaches its spp. Returns (path samples, seconds,
    per-job times to target)."""
    ctx.sync()
    t0 = time.perf_counter()
    active = {}
    for j in jobs:
        s = _snelly(ctx, j, kernel)
        s.render(0)
        active[s.job_id()] = (j, s, [0])
    samples, done_at = 0, []
    while active:
        step = {jid: min(frames_per_tick, j["spp"] - n[0]) for jid, (j, s, n) in active.items()}
        ctx.advance_batch(step)
        finished = []
        for jid, (j, s, n) in active.items():
            n[0] += step[jid]
            if n[0] >= j["spp"]:
                finished.append(jid)
        for jid in finished:
            j, s, n = active.pop(jid)
            img = s.readback()
            samples += s.width * s.height * j["spp"]
            done_at.append(time.perf_counter() - t0)
            if keep is not None:
                keep[j["id"]] = img
            ctx.destroy_job(jid)
    return samples, time.perf_counter() - t0, np.array(done_at)


def measure(ctx, jobs, frames_per_tick=8, check_images=True):
    """Plain and batched runs of `jobs` (both with the autotuner's integrator per job): the dict
    the JSON line reports."""
    warm(ctx, jobs, N.KERNEL_AUTO)
    plain_imgs, batch_imgs = ({}, {}) if check_images else (None, None)
    ps, pt, pdone = run_plain(ctx, jobs, N.KERNEL_AUTO, plain_imgs)
    bs, bt, bdone = run_batched(ctx, jobs, N.KERNEL_AUTO, frames_per_tick, batch_imgs)
    out = {
        "jobs": len(jobs), "path_samples": bs, "pixels": int(sum(j["res"] ** 2 for j in jobs)),
        "plain": {"seconds": pt, "samples_per_s": ps / pt, "time_to_target_p50_s": float(np.percentile(pdone, 50)),
                  "time_to_target_p99_s": float(np.percentile(pdone, 99))},
        "batched": {"seconds": bt, "samples_per_s": bs / bt, "frames_per_tick": frames_per_tick,
                    "time_to_target_p50_s": float(np.percentile(bdone, 50)),
                    "time_to_target_p99_s": float(np.percentile(bdone, 99))},
        "batched_over_plain": (bs / bt) / (ps / pt),
        "scenes": {n: sum(1 for j in jobs if j["name"] == n) for n in SCENE_NAMES},
    }
    if check_images:
        same = sum(int(np.array_equal(plain_imgs[k], batch_imgs[k])) for k in plain_imgs)
        out["images_identical_plain_vs_batched"] = f"{same}/{len(plain_imgs)}"
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=256)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--max-res", type=int, default=1024)
    ap.add_argument("--frames-per-tick", type=int, default=8)
    args = ap.parse_args()
    ctx = api.Context(0)
    jobs = job_set(args.jobs, args.seed, res_range=(128, args.max_res))
    out = {"metric": "heterogeneous batch: path samples/s and time to target, batched vs plain"}
    out.update(measure(ctx, jobs, args.frames_per_tick))
    print(json.dumps(out))


if __name__ == "__main__":
    main()
