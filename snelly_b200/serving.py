"""Continuous-batching render server on one GPU.

Requests (a scene, a resolution, a target of spp or of relative noise on the mean luminance)
arrive over time. The server admits waiting requests in arrival order while its HBM budget
allows, keeps every admitted job's per-pixel state resident on the device, and on each tick
advances every active job in one batched call (snelly_advance_batch: the autotuner's wavefront
jobs run concurrently as pixel ranges on their own streams, the others share path-per-thread
launches per scene module, modules on separate streams): a fixed-spp job by up to
`frames_per_tick` frames, a noise-target job by one frame (its stopping rule reads the image
statistics after every frame). A job leaves when it reaches its target; its image is read back
and its memory returned to the budget, so requests that arrive while others render join as soon
as memory frees up.

Each pixel owns its RNG stream and its accumulation order, so a job's image does not depend on
what it was batched with (tests/test_gpu_batch.py checks this bit for bit).

`python -m snelly_b200.serving --rate 200 --duration 60` runs the Poisson request stream of the
serving configuration and prints one JSON line with p50 / p99 time-to-target and the aggregate
path samples per second.
"""
import argparse
import json
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import api, scenes

# per pixel: rng, Kahan sums + compensations, resolved image (80 B), and the wavefront's path
# record, parked-ray state and queues when the autotuner gives the job the wavefront (<= 420 B)
JOB_BYTES_PER_PIXEL = 80 + 420


@dataclass
class Request:
    rid: int
    arrival: float                 # seconds from the start of the stream
    scene: object                  # a scene object (reference scene API)
    target_spp: int = 0            # stop after this many frames (0: use the noise target)
    noise_target: float = 0.0      # stop when the relative standard error of the mean luminance <= this
    max_spp: int = 1024
    seed: int = 1


@dataclass
class Result:
    rid: int
    arrival: float
    admitted: float
    finished: float
    spp: int
    pixels: int
    noise: float
    image: np.ndarray = field(default=None, repr=False)

    @property
    def latency(self):
        return self.finished - self.arrival


class Server:
    def __init__(self, ctx, hbm_budget_bytes, keep_images=False, frames_per_tick=4):
        self.ctx = ctx
        self.budget = hbm_budget_bytes
        self.keep_images = keep_images
        self.frames_per_tick = frames_per_tick

    @staticmethod
    def job_bytes(req):
        return req.scene.width * req.scene.height * JOB_BYTES_PER_PIXEL

    def warm(self, requests):
        """Compile every distinct scene module and run the autotuner for every (module, image-size
        class) before the clock starts (a server knows its scenes and sizes)."""
        seen = set()
        for r in requests:
            s = api.Snelly(r.scene, context=self.ctx)
            key = (r.scene.shader(), bytes(s.scene_opts()), int(round(math.log2(r.scene.width * r.scene.height))))
            if key not in seen:
                seen.add(key)
                s.render(0)
                self.ctx.destroy_job(s.job_id())

    def run(self, requests, clock=time.perf_counter):
        pending = sorted(requests, key=lambda r: r.arrival)
        waiting, active, done = [], {}, []
        used = 0
        t0 = clock()
        samples = 0
        while pending or waiting or active:
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                waiting.append(pending.pop(0))
            while waiting and used + self.job_bytes(waiting[0]) <= self.budget:
                req = waiting.pop(0)
                s = api.Snelly(req.scene, context=self.ctx)
                s.seed = req.seed
                s.render(0)  # allocate + seed (the integrator the autotuner chose for this module and size)
                used += self.job_bytes(req)
                active[s.job_id()] = {"req": req, "snelly": s, "spp": 0, "admitted": clock() - t0, "means": []}
            if not active:
                if waiting and used == 0:
                    raise RuntimeError(f"request {waiting[0].rid} needs more memory than the whole budget")
                if pending:
                    time.sleep(max(0.0, min(0.01, pending[0].arrival - (clock() - t0))))
                continue
            step = {}
            for jid, a in active.items():
                req = a["req"]
                step[jid] = 1 if req.noise_target > 0 else max(1, min(self.frames_per_tick, req.target_spp - a["spp"]))
            self.ctx.advance_batch(step)
            self.ctx.sync()
            finished = []
            for jid, a in active.items():
                a["spp"] += step[jid]
                req = a["req"]
                s = a["snelly"]
                samples += s.width * s.height * step[jid]
                noise = float("nan")
                if req.noise_target > 0:
                    st = self.ctx.image_stats(jid)
                    npx = s.width * s.height
                    mean_y = st[1] / npx
                    # per-frame image means from successive running means give the spread
                    a["means"].append(mean_y)
                    k = len(a["means"])
                    if k >= 4:
                        m = np.array(a["means"])
                        frames = m * np.arange(1, k + 1) - np.concatenate([[0.0], m[:-1] * np.arange(1, k)])
                        noise = float(np.std(frames, ddof=1) / math.sqrt(k) / max(abs(m[-1]), 1e-30))
                    if (k >= 4 and noise <= req.noise_target) or a["spp"] >= req.max_spp:
                        finished.append((jid, noise))
                elif a["spp"] >= req.target_spp:
                    finished.append((jid, noise))
            for jid, noise in finished:
                a = active.pop(jid)
                s = a["snelly"]
                img = s.readback()
                t = clock() - t0
                done.append(Result(a["req"].rid, a["req"].arrival, a["admitted"], t, a["spp"], s.width * s.height, noise,
                                   img if self.keep_images else None))
                self.ctx.destroy_job(jid)
                used -= self.job_bytes(a["req"])
        elapsed = clock() - t0
        return done, samples, elapsed


def serving_requests(rate, duration, seed=5, noise_fraction=0.5, spp_range=(4, 64), res_range=(128, 1024),
                     scene_names=("c0", "c1", "c2", "mesh")):
    """A Poisson request stream: arrivals at `rate` per second for `duration` seconds; each request
    draws a scene (plain sphere, dispersive fractal, volumetric/subsurface Mandelbox, mesh-like
    distance grid), a square resolution (log-uniform), a camera pose on a sphere of radius U(4, 8), a
    bounce limit U{4..12}, and either a fixed spp U{spp_range} or a 2% relative-noise target."""
    rs = np.random.RandomState(seed)
    t, reqs, rid = 0.0, [], 0
    while True:
        t += rs.exponential(1.0 / rate)
        if t > duration:
            break
        res = int(round(math.exp(rs.uniform(math.log(res_range[0]), math.log(res_range[1])))))
        name = scene_names[rs.randint(len(scene_names))]
        sc = posed_scene(name, res, rs)
        if rs.uniform() < noise_fraction:
            reqs.append(Request(rid, t, sc, noise_target=0.02, max_spp=spp_range[1], seed=rid + 1))
        else:
            reqs.append(Request(rid, t, sc, target_spp=int(rs.randint(spp_range[0], spp_range[1] + 1)), seed=rid + 1))
        rid += 1
    return reqs


class _Posed:
    """A benchmark scene with a random camera pose and bounce limit (same scene module)."""

    def __init__(self, base, pos, target, bounces):
        self.base, self.pos, self.target, self.bounces = base, pos, target, bounces
        self.width, self.height = base.width, base.height

    def init(self, snelly):
        self.base.init(snelly)
        snelly.getCamera().position.set(*self.pos)
        snelly.getControls().target.set(*self.target)
        r = snelly.getRenderer()
        r.maxBounces = 12               # one module (MAX_BOUNCES = 12) per scene type ...
        r.jobMaxBounces = self.bounces  # ... and the request's own bound at run time

    def shader(self):
        return self.base.shader()

    def __getattr__(self, name):  # the other scene methods (syncShader, length scales, ...)
        if name == "base":
            raise AttributeError(name)
        return getattr(self.base, name)


def posed_scene(name, res, rs):
    base = scenes.SCENES[name](res, res)
    r = rs.uniform(4.0, 8.0)
    th = rs.uniform(0.15, 0.45 * math.pi)
    ph = rs.uniform(0.0, 2.0 * math.pi)
    pos = (r * math.sin(th) * math.cos(ph), r * math.cos(th), r * math.sin(th) * math.sin(ph))
    return _Posed(base, pos, (0.0, 0.0, 0.0), int(rs.randint(4, 13)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--duration", type=float, default=60.0)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--max-res", type=int, default=1024)
    ap.add_argument("--seed", type=int, default=5)
    args = ap.parse_args()
    ctx = api.Context(0)
    reqs = serving_requests(args.rate, args.duration, seed=args.seed, res_range=(128, args.max_res))
    srv = Server(ctx, int(args.budget_gb * 2 ** 30))
    srv.warm(reqs)
    done, samples, elapsed = srv.run(reqs)
    lat = np.array([r.latency for r in done])
    print(json.dumps({"metric": "serving time-to-target", "requests": len(done), "rate_per_s": args.rate,
                      "duration_s": args.duration, "elapsed_s": elapsed,
                      "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                      "path_samples_per_s": samples / elapsed, "hbm_budget_gb": args.budget_gb}))


if __name__ == "__main__":
    main()
