"""The scene API's per-frame behaviour on the GPU: parameter changes between frames of a live job
(snelly_update_job), animation through pre/post-frame callbacks, and dumpScene round trips."""
import numpy as np
import pytest

from snelly_b200 import _native as N
from snelly_b200 import api, scenes

pytestmark = pytest.mark.gpu

KERNELS = [N.KERNEL_MEGA, N.KERNEL_WAVEFRONT]


def turntable(ctx, kernel, frame=0, **kw):
    sc = scenes.Turntable(32, 32, target_spp=1 << 20, **kw)
    s = api.Snelly(sc, context=ctx)
    s.pathtracer.kernelMode = kernel
    sc.animFrame = frame
    return sc, s


@pytest.mark.parametrize("kernel", KERNELS)
def test_changed_parameters_reach_the_next_frames(gpu_ctx, kernel):
    """Two frames at animation pose 0, then two at pose 3 in the same job (camera, scene uniforms
    and the resulting uniform block all change) equal a job restored from the two-frame state with
    the pose-3 parameters: the accumulation continues, the new parameters apply from the next
    frame, as with the reference's per-frame uniform upload."""
    sc, a = turntable(gpu_ctx, kernel)
    a.render(2)
    sc.animFrame = 3
    a.render(2)
    got = a.readback()
    assert (got[..., 3] == 4).all()

    _, b = turntable(gpu_ctx, kernel)
    b.render(2)
    rng, acc, comp, _ = b.readback_state()
    sc3, c = turntable(gpu_ctx, kernel, frame=3)
    sc3.pose(c, 3)
    sid = c.compileShaders()
    c.sync_scene(sid)
    jid = gpu_ctx.restore(sid, c.render_desc(2), rng, acc, comp)
    want = gpu_ctx.readback(jid, 32, 32)
    gpu_ctx.destroy_job(jid)
    np.testing.assert_array_equal(got, want)
    # and the second pose did change the image
    _, d = turntable(gpu_ctx, kernel)
    d.render(4)
    assert not np.array_equal(d.readback(), got)


def test_update_without_change_is_identity(gpu_ctx):
    _, a = turntable(gpu_ctx, N.KERNEL_MEGA)
    a.render(2)
    gpu_ctx.update_job(a.job_id(), a.render_desc(0))
    a.render(2)
    _, b = turntable(gpu_ctx, N.KERNEL_MEGA)
    b.render(4)
    np.testing.assert_array_equal(a.readback(), b.readback())


def test_update_rejects_a_new_image_size(gpu_ctx):
    _, a = turntable(gpu_ctx, N.KERNEL_MEGA)
    a.render(1)
    d = a.render_desc(0)
    d.width += 1
    with pytest.raises(N.SnellyError) as e:
        gpu_ctx.update_job(a.job_id(), d)
    assert e.value.code == -1
    a.render(1)  # the job is untouched
    assert (a.readback()[..., 3] == 2).all()


def test_turntable_animation_frames(gpu_ctx):
    """The animation protocol of the reference's scene template: each animation frame accumulates
    target_spp samples, is handed to postframeCallback, and the next frame starts from a reset.
    Every handed-over frame equals a fresh render of that pose."""
    got = {}
    sc = scenes.Turntable(32, 32, frames=3, target_spp=3, on_frame=lambda i, s: got.__setitem__(i, s.readback()))
    s = api.Snelly(sc, context=gpu_ctx)
    s.pathtracer.kernelMode = N.KERNEL_MEGA
    s.render(3 * 3)
    assert sorted(got) == [0, 1, 2]
    for k in range(3):
        assert (got[k][..., 3] == 3).all()
        _, f = turntable(gpu_ctx, N.KERNEL_MEGA, frame=k)
        f.render(3)
        np.testing.assert_array_equal(got[k], f.readback())
    assert not np.array_equal(got[0], got[1]) and not np.array_equal(got[1], got[2])


def test_dump_scene_round_trip_renders_the_same_image(gpu_ctx):
    a = api.Snelly(scenes.HooksAndMaps(32, 32), context=gpu_ctx)
    a.pathtracer.kernelMode = N.KERNEL_MEGA
    a.getCamera().position.set(0.5, 1.5, 3.5)
    a.getRenderer().sunLatitude = 35.0
    a.getMaterials().getSurface().roughness = 0.45
    a.getMaterials().loadMetal("Copper").roughness = 0.2
    a.reset()
    a.render(2)
    code = a.dumpScene("python")
    b = api.Snelly(scenes.HooksAndMaps(32, 32), context=gpu_ctx)
    b.pathtracer.kernelMode = N.KERNEL_MEGA
    exec(code, {"snelly": b, "self": b.sceneObj})
    b.reset()
    b.render(2)
    np.testing.assert_array_equal(a.readback(), b.readback())
