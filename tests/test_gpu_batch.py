"""Batched launches: many jobs of different scenes, sizes and frame counts in one call give the
same images as each job rendered alone (bit for bit: each pixel owns its RNG stream and its
accumulation order)."""
import numpy as np
import pytest

from helpers import gpu_render
from snelly_b200 import api, scenes

pytestmark = pytest.mark.gpu


def _mix():
    return [(lambda: scenes.PlainSphere(64, 64), 6, 1), (lambda: scenes.DispersiveFractal(80, 45), 3, 2),
            (lambda: scenes.HooksAndMaps(48, 48), 5, 3), (lambda: scenes.PlainSphere(96, 32), 2, 4),
            (lambda: scenes.AtmosphereLights(40, 30), 4, 5), (lambda: scenes.DispersiveFractal(33, 17), 7, 6)]


def test_same_alone_and_in_the_mix(gpu_ctx):
    alone = [gpu_render(gpu_ctx, f(), fr, seed=sd)[1] for f, fr, sd in _mix()]
    mixed = []
    for f, fr, sd in _mix():
        s = api.Snelly(f(), context=gpu_ctx)
        s.seed = sd
        s.render(0)
        mixed.append((s, fr))
    gpu_ctx.advance_batch({s.job_id(): fr for s, fr in mixed})
    for (s, fr), ref in zip(mixed, alone):
        img = s.readback()
        assert (img[..., 3] == fr).all()
        np.testing.assert_array_equal(img, ref)


def test_batches_larger_than_one_launch(gpu_ctx):
    """40 jobs of one scene module (more than the 32 parameter slots of a launch)."""
    rs = np.random.RandomState(0)
    jobs = []
    for k in range(40):
        w, h, fr = int(rs.randint(8, 40)), int(rs.randint(8, 40)), int(rs.randint(1, 5))
        s = api.Snelly(scenes.PlainSphere(w, h), context=gpu_ctx)
        s.seed = 100 + k
        s.render(0)
        jobs.append((s, fr, w, h))
    gpu_ctx.advance_batch({s.job_id(): fr for s, fr, w, h in jobs})
    for k, (s, fr, w, h) in enumerate(jobs):
        ref = gpu_render(gpu_ctx, scenes.PlainSphere(w, h), fr, seed=100 + k)[1]
        np.testing.assert_array_equal(s.readback(), ref)


def test_wavefront_jobs_in_a_batch(gpu_ctx):
    """Wavefront jobs in a batch run concurrently, each in its own constant-memory slot and pixel
    ranges: 36 of one scene module (more than the 32 slots: two waves), path-per-thread jobs of
    the same module (whose launch lane hands the slots over), other modules, and one image large
    enough for three concurrent pixel ranges. Every image equals the job rendered alone, bit for
    bit."""
    from snelly_b200 import _native as N
    rs = np.random.RandomState(3)
    spec = []
    for k in range(36):
        spec.append((scenes.PlainSphere, int(rs.randint(24, 120)), int(rs.randint(24, 120)), int(rs.randint(1, 4)),
                     N.KERNEL_WAVEFRONT))
    for k in range(4):
        spec.append((scenes.PlainSphere, int(rs.randint(24, 80)), int(rs.randint(24, 80)), 2, N.KERNEL_MEGA))
    spec += [(scenes.DispersiveFractal, 96, 54, 3, N.KERNEL_WAVEFRONT), (scenes.AtmosphereLights, 64, 48, 2, N.KERNEL_WAVEFRONT),
             (scenes.DispersiveFractal, 512, 400, 2, N.KERNEL_WAVEFRONT)]
    jobs = []
    for k, (cls, w, h, fr, km) in enumerate(spec):
        s = api.Snelly(cls(w, h), context=gpu_ctx)
        s.seed = 500 + k
        s.pathtracer.kernelMode = km
        s.render(0)
        assert gpu_ctx.job_kernel(s.job_id()) == km
        jobs.append((s, fr))
    gpu_ctx.advance_batch({s.job_id(): fr for s, fr in jobs})
    got = [s.readback().copy() for s, fr in jobs]
    for s, fr in jobs:
        gpu_ctx.destroy_job(s.job_id())
    for k, (cls, w, h, fr, km) in enumerate(spec):
        ref = gpu_render(gpu_ctx, cls(w, h), fr, seed=500 + k, kernel_mode=km)
        assert (got[k][..., 3] == fr).all(), k
        np.testing.assert_array_equal(got[k], ref[1], err_msg=f"job {k}")
        gpu_ctx.destroy_job(ref[0].job_id())


def test_single_wavefront_job_in_a_batch(gpu_ctx):
    """A batch whose only wavefront job shares the call with path-per-thread jobs (what a serving
    tick often is): the wavefront job's parameters go to its own slot like any batch job's, and its
    image equals the job rendered alone, bit for bit, over two calls."""
    from snelly_b200 import _native as N
    spec = [(scenes.DispersiveFractal, 80, 45, N.KERNEL_WAVEFRONT, 31), (scenes.PlainSphere, 40, 40, N.KERNEL_MEGA, 32),
            (scenes.HooksAndMaps, 32, 32, N.KERNEL_MEGA, 33)]
    jobs = []
    for cls, w, h, km, sd in spec:
        s = api.Snelly(cls(w, h), context=gpu_ctx)
        s.seed = sd
        s.pathtracer.kernelMode = km
        s.render(0)
        jobs.append(s)
    # another job's parameters in slot 0 of the fractal's module, as a solo render leaves them
    other = gpu_render(gpu_ctx, scenes.DispersiveFractal(64, 64), 1, seed=99, kernel_mode=N.KERNEL_WAVEFRONT)[0]
    for _ in range(2):
        gpu_ctx.advance_batch({s.job_id(): 2 for s in jobs})
    for (cls, w, h, km, sd), s in zip(spec, jobs):
        ref = gpu_render(gpu_ctx, cls(w, h), 4, seed=sd, kernel_mode=km)
        np.testing.assert_array_equal(s.readback(), ref[1])
        gpu_ctx.destroy_job(ref[0].job_id())
        gpu_ctx.destroy_job(s.job_id())
    gpu_ctx.destroy_job(other.job_id())
