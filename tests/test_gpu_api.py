"""C ABI behaviour on the GPU: progressive frames, checkpoint/resume, errors and budgets."""
import ctypes

import numpy as np
import pytest

from helpers import gpu_render
from snelly_b200 import _native as N
from snelly_b200 import api, scenes

pytestmark = pytest.mark.gpu


def test_progressive_frames_equal_single_render(gpu_ctx):
    a, img_a = gpu_render(gpu_ctx, scenes.PlainSphere(64, 64), 8)
    b = api.Snelly(scenes.PlainSphere(64, 64), context=gpu_ctx)
    b.render(3)
    b.render(5)
    img_b = b.readback()
    np.testing.assert_array_equal(img_a, img_b)


def test_checkpoint_resume_is_exact(gpu_ctx):
    a, _ = gpu_render(gpu_ctx, scenes.DispersiveFractal(64, 36), 6)
    full = a.readback()
    b, _ = gpu_render(gpu_ctx, scenes.DispersiveFractal(64, 36), 3)
    rng, acc, comp, _ = b.readback_state()
    sid = b.compileShaders()
    desc = b.render_desc(3)
    jid = gpu_ctx.restore(sid, desc, rng, acc, comp)
    resumed = gpu_ctx.readback(jid, 64, 36)
    np.testing.assert_array_equal(full, resumed)


def test_budget_refusal_leaves_context_usable():
    ctx = api.Context(0, hbm_budget=64 << 20)
    s = api.Snelly(scenes.PlainSphere(2048, 2048), context=ctx)
    with pytest.raises(N.SnellyError) as e:
        s.render(1)
    assert e.value.code == -3  # ENOMEM_BUDGET
    s2 = api.Snelly(scenes.PlainSphere(32, 32), context=ctx)
    s2.render(2)
    assert np.isfinite(s2.readback()).all()
    ctx.close()


def test_errors_are_reported(gpu_ctx):
    L = N.lib()
    with pytest.raises(N.SnellyError) as e:
        gpu_ctx.readback(987654, 4, 4)
    assert e.value.code == -7
    opts = N.SceneOpts(3, 64, 1, 1, 0, 0, 0, 0, 0, 0, 1)
    with pytest.raises(N.SnellyError) as e:
        gpu_ctx.create_scene("float SDF_SURFACE(vec3 X) { return length(X) - ; }", opts)
    assert e.value.code == -2 and "error" in str(e.value)
    with pytest.raises(N.SnellyError) as e:
        gpu_ctx.create_scene("float f(vec3 X) { return 1.0; }", opts)
    assert e.value.code == -2
    sid = gpu_ctx.create_scene("uniform float R; float SDF_SURFACE(vec3 X) { return length(X) - R; }", opts)
    with pytest.raises(N.SnellyError) as e:
        gpu_ctx.set_uniforms(sid, {"nope": (N.U_FLOAT, [1.0])})
    assert e.value.code == -7
    with pytest.raises(N.SnellyError) as e:
        gpu_ctx.set_uniforms(sid, {"R": (N.U_VEC3, [1.0, 2.0, 3.0])})
    assert e.value.code == -1
    d = N.RenderDesc()
    d.width, d.height, d.frames = 0, 4, 1
    with pytest.raises(N.SnellyError) as e:
        gpu_ctx.render(sid, d)
    assert e.value.code == -1


def test_cancel_and_poll(gpu_ctx):
    s = api.Snelly(scenes.PlainSphere(128, 128), context=gpu_ctx)
    s.render(4)
    jid = s.job_id()
    try:
        gpu_ctx.readback(jid, 128, 128, poll=True)
    except N.SnellyError as e:
        assert e.code == -4  # EBUSY while frames run
    gpu_ctx.sync()
    img = gpu_ctx.readback(jid, 128, 128, poll=True)
    assert (img[..., 3] == 4).all()
    gpu_ctx.cancel(jid)
    with pytest.raises(N.SnellyError) as e:
        gpu_ctx.readback(jid, 128, 128)
    assert e.value.code == -8


def test_native_kernels_ran(gpu_ctx):
    before = gpu_ctx.launch_count()
    gpu_render(gpu_ctx, scenes.PlainSphere(32, 32), 3)
    assert gpu_ctx.launch_count() >= before + 4  # seed + 3 frames + resolve


def test_autotuned_kernel_choice_leaves_no_trace(gpu_ctx):
    """A scene created with SNELLY_KERNEL_AUTO runs the autotuner's trial frames on the job's own
    buffers, then seeds the job again: its image equals a render with the chosen integrator set
    explicitly, bit for bit; the decision is cached per module and size class."""
    from snelly_b200 import api
    from snelly_b200 import _native as N

    def run(kmode):
        s = api.Snelly(scenes.DispersiveFractal(96, 54), context=gpu_ctx)
        s.seed = 9
        s.pathtracer.kernelMode = kmode
        s.render(3)
        img = s.readback().copy()
        k = gpu_ctx.job_kernel(s.job_id())
        gpu_ctx.destroy_job(s.job_id())
        return img, k

    img_auto, k = run(N.KERNEL_AUTO)
    assert k in (N.KERNEL_MEGA, N.KERNEL_WAVEFRONT)
    img_explicit, k2 = run(k)
    assert k2 == k
    np.testing.assert_array_equal(img_auto, img_explicit)
    img_again, k3 = run(N.KERNEL_AUTO)
    assert k3 == k
    np.testing.assert_array_equal(img_again, img_auto)


def test_async_readback_overlaps_and_matches(gpu_ctx):
    """SNELLY_READ_ASYNC: the copy is ordered after the frames enqueued before it and before the
    frames enqueued after it touch the mean image; page-locked and pageable outputs both hold the
    image of their moment once the context is synchronised."""
    import torch
    s = api.Snelly(scenes.PlainSphere(64, 48), context=gpu_ctx)
    pinned = [torch.empty((48, 64, 4), dtype=torch.float32, pin_memory=True).numpy() for _ in range(2)]
    pageable = np.full((48, 64, 4), -1.0, np.float32)
    s.render(2)
    s.readback(out=pinned[0], wait=False)
    s.render(3)
    s.readback(out=pinned[1], wait=False)
    s.readback(out=pageable, wait=False)
    gpu_ctx.sync()
    ref2 = api.Snelly(scenes.PlainSphere(64, 48), context=gpu_ctx)
    ref2.render(2)
    np.testing.assert_array_equal(pinned[0], ref2.readback())
    np.testing.assert_array_equal(pinned[1], s.readback())
    np.testing.assert_array_equal(pageable, pinned[1])
    assert (pinned[1][..., 3] == 5).all()
    # a job destroyed right after an asynchronous readback waits for the copy
    s.render(1)
    s.readback(out=pinned[0], wait=False)
    gpu_ctx.destroy_job(s.job_id())
    assert (pinned[0][..., 3] == 6).all()
