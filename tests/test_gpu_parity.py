"""The CUDA path tracer against the reference (golden fixtures) and the oracle: per pixel with
matched seeds, and statistically with independent seeds. Tolerances are written in each test."""
import numpy as np
import pytest

from helpers import CASES, golden, gpu_render, host, oracle_render, welch_p
from snelly_b200 import _native as N
from snelly_b200 import scenes

pytestmark = pytest.mark.gpu


def _close(a, b, rtol):
    return np.abs(a - b).max(-1) <= rtol * np.maximum(1.0, np.abs(b).max(-1))


KERNELS = {"mega": N.KERNEL_MEGA, "wavefront": N.KERNEL_WAVEFRONT}


@pytest.mark.parametrize("kernel", sorted(KERNELS))
@pytest.mark.parametrize("name", sorted(CASES))
def test_strict_math_matches_reference_per_pixel(gpu_ctx, name, kernel):
    """IEEE-strict module vs the reference shader: same seeds, so paths agree pixel by pixel
    except where a transcendental's last-ulp difference (CUDA's vs glibc's sin/cos/exp/log/pow)
    flips a branch; the subsurface walk (up to 128 -log(u) steps per vertex) is the longest such
    chain. Bar: >= 93% of pixels within 1e-4 relative, image mean XYZ within 0.5%."""
    g = golden(name)
    s, img = gpu_render(gpu_ctx, CASES[name](), int(g["frames"]), seed=int(g["seed"]), math_mode=N.MATH_STRICT,
                        kernel_mode=KERNELS[kernel])
    got = img.reshape(-1, 4)
    ref = g["mean"]
    assert (got[:, 3] == ref[:, 3]).all()
    ok = _close(got[:, :3], ref[:, :3], 1e-4)
    assert ok.mean() >= 0.93, f"{name}: only {ok.mean():.4f} of pixels within 1e-4"
    rel = np.abs(got[:, :3].mean(0) - ref[:, :3].mean(0)) / np.abs(ref[:, :3].mean(0))
    assert rel.max() <= 5e-3, rel


# The C2 Mandelbox distance estimator amplifies last-bit differences (approximate division and
# contracted multiply-adds in fast-math builds) into different hit points within a few steps, so
# matched seeds give different paths at half the pixels: per-pixel agreement is not expected
# there, and C2 is checked in distribution (test_statistical_agreement_independent_seeds).
FAST_CASES = sorted(n for n in CASES if n != "c2")


@pytest.mark.parametrize("kernel", sorted(KERNELS))
@pytest.mark.parametrize("name", FAST_CASES)
def test_fast_math_matches_reference(gpu_ctx, name, kernel):
    """Production (fast-math) module vs the reference shader with matched seeds. Bar: >= 80% of
    pixels within 1e-3 relative (the rest diverged through ulp-level differences), image mean XYZ
    within 3% on these small, few-frame images (the 0.5% bar is tested at scale below)."""
    g = golden(name)
    s, img = gpu_render(gpu_ctx, CASES[name](), int(g["frames"]), seed=int(g["seed"]), math_mode=N.MATH_FAST,
                        kernel_mode=KERNELS[kernel])
    got = img.reshape(-1, 4)
    ref = g["mean"]
    assert np.isfinite(got).all()
    ok = _close(got[:, :3], ref[:, :3], 1e-3)
    assert ok.mean() >= 0.80, f"{name}: only {ok.mean():.4f} of pixels within 1e-3"
    rel = np.abs(got[:, :3].mean(0) - ref[:, :3].mean(0)) / np.abs(ref[:, :3].mean(0))
    assert rel.max() <= 3e-2, rel


def test_rng_seeding_matches_oracle(gpu_ctx):
    from snelly_b200 import api
    s = api.Snelly(scenes.PlainSphere(64, 64), context=gpu_ctx)
    s.seed = 12345
    s.render(0)
    rng, acc, comp, _ = s.readback_state()
    import oracle
    h = host("c0")
    lib = oracle.OracleLib(h.sceneObj.shader(), h.scene_opts())
    np.testing.assert_array_equal(rng, lib.seed(12345, np.arange(64 * 64)))
    assert (acc == 0).all() and (comp == 0).all()


STAT_SCENES = {
    "c1": lambda: scenes.DispersiveFractal(160, 92),
    "c0": lambda: scenes.PlainSphere(96, 96),
    "c2": lambda: scenes.VolumetricSubsurface(64, 64),
}


def _gpu_batches(ctx, factory, kernel, batches, frames, seed0):
    ys = []
    for b in range(batches):
        s, img = gpu_render(ctx, factory(), frames, seed=seed0 + b, kernel_mode=KERNELS[kernel])
        ys.append(img[..., 1].reshape(-1))
        ctx.destroy_job(s.job_id())
    return np.array(ys, np.float64)


def _oracle_batches(factory, batches, frames, seed0):
    from snelly_b200.testing import HostSnelly
    ys = []
    for b in range(batches):
        h = HostSnelly(factory(), seed=seed0 + b)
        xyz, _, _ = oracle_render(h, np.arange(h.width * h.height), frames)
        ys.append(xyz[:, 1] / frames)
    return np.array(ys, np.float64), h.height, h.width


def _welch(a, b):
    """|mean difference| / standard error per column (Welch), and the zero-variance mask."""
    se = np.sqrt(a.var(0, ddof=1) / len(a) + b.var(0, ddof=1) / len(b))
    m = se > 0
    return np.abs(a.mean(0) - b.mean(0))[m] / se[m], m


@pytest.mark.parametrize("kernel", sorted(KERNELS))
@pytest.mark.parametrize("scene", sorted(STAT_SCENES))
def test_statistical_agreement_independent_seeds(gpu_ctx, scene, kernel):
    """Production GPU module and the oracle with independent seeds agree within Monte Carlo error
    at matched spp: 16 batches of 4 frames on each side (64 spp), per-pixel luminance compared with
    Welch's two-sample t statistic as a two-sided p-value (Welch-Satterthwaite degrees of
    freedom, about 30). Bars: the image mean luminance within 4 standard errors of the difference
    (about 0.5-1% at these sizes); at most 0.8% of pixels with p < 0.0027 (0.27% expected when both
    sides estimate the same image) and 0.05% with p < 5.7e-7 (the Gaussian 3 and 5 standard-error
    levels); over 4x4-pixel tiles at most 1% with p < 0.0027 and none with p < 2e-9 (6 standard
    errors). Pixels with zero variance on both sides must agree exactly."""
    factory = STAT_SCENES[scene]
    batches, frames = 16, 4
    g = _gpu_batches(gpu_ctx, factory, kernel, batches, frames, 1000)
    o, H, W = _oracle_batches(factory, batches, frames, 5000)
    gm, om = g.mean(1), o.mean(1)  # image means of each batch
    se_img = np.sqrt(gm.var(ddof=1) / batches + om.var(ddof=1) / batches)
    z, m = _welch(g, o)
    B = len(g)
    p = welch_p(g.mean(0), g.var(0, ddof=1), B, o.mean(0), o.var(0, ddof=1), len(o))[m]

    def tiles(a):
        return a.reshape(a.shape[0], H // 4, 4, W // 4, 4).mean(axis=(2, 4)).reshape(a.shape[0], -1)

    tg, to = tiles(g), tiles(o)
    tp = welch_p(tg.mean(0), tg.var(0, ddof=1), B, to.mean(0), to.var(0, ddof=1), len(o))
    tp = tp[np.isfinite(tp)]
    msg = (f"image mean gpu {gm.mean():.6f} oracle {om.mean():.6f} (SE {se_img:.2e}); pixels with p < 0.0027 / 5.7e-7 "
           f"{(p < 0.0027).mean():.4f}/{(p < 5.7e-7).mean():.5f}; tiles with p < 0.0027 / 2e-9 "
           f"{(tp < 0.0027).mean():.4f}/{(tp < 2e-9).mean():.4f}")
    print(msg)
    assert abs(gm.mean() - om.mean()) <= 4 * se_img, msg
    assert (p < 0.0027).mean() <= 0.008, msg
    assert (p < 5.7e-7).mean() <= 0.0005, msg
    assert (tp < 0.0027).mean() <= 0.01, msg
    assert (tp < 2e-9).sum() == 0, msg
    assert (np.abs(g.mean(0) - o.mean(0))[~m] < 1e-5).all(), msg


def test_kahan_vs_fp64_accumulation(gpu_ctx):
    """FP32 Kahan sums stay within a few ulps of the FP64 accumulation oracle."""
    s, img = gpu_render(gpu_ctx, scenes.PlainSphere(64, 64), 64, fp64=True)
    rng, acc, comp, acc64 = s.readback_state()
    assert (acc64[:, 3] == 64).all() and (acc[:, 3] == 64).all()
    k = acc[:, :3].astype(np.float64) - comp[:, :3].astype(np.float64)
    rel = np.abs(k - acc64[:, :3]) / np.maximum(np.abs(acc64[:, :3]), 1e-30)
    assert rel.max() < 4e-7, rel.max()


@pytest.mark.parametrize("name", ["c1", "atmosphere", "hooks"])
def test_wavefront_equals_path_per_thread(gpu_ctx, name):
    """Both integrators consume the same random numbers in the same order; with strict math they
    differ only in the summation order of the deferred next-event estimate. Bar: >= 97% of pixels
    within 1e-5 relative."""
    a = gpu_render(gpu_ctx, CASES[name](), 3, seed=5, math_mode=N.MATH_STRICT, kernel_mode=N.KERNEL_MEGA)[1]
    b = gpu_render(gpu_ctx, CASES[name](), 3, seed=5, math_mode=N.MATH_STRICT, kernel_mode=N.KERNEL_WAVEFRONT)[1]
    a, b = a.reshape(-1, 4), b.reshape(-1, 4)
    assert (a[:, 3] == b[:, 3]).all()
    ok = _close(b[:, :3], a[:, :3], 1e-5)
    assert ok.mean() >= 0.97, ok.mean()


@pytest.mark.parametrize("name", ["c1", "c2", "atmosphere", "mesh"])
def test_wavefront_parking_does_not_change_results(name):
    """The extend stage parks the longest rays when its work runs out and resumes them in the next
    iteration. A context that parks after 8 drain steps, one that never parks and the default give
    the same image bit for bit: a ray's march is the same sequence of operations however it is
    split."""
    import os
    from snelly_b200 import api
    imgs = []
    for drain in ("8", "0", None):
        old = os.environ.pop("SNELLY_WF_DRAIN", None)
        if drain is not None:
            os.environ["SNELLY_WF_DRAIN"] = drain
        try:
            ctx = api.Context(0)
        finally:
            os.environ.pop("SNELLY_WF_DRAIN", None)
            if old is not None:
                os.environ["SNELLY_WF_DRAIN"] = old
        s, img = gpu_render(ctx, CASES[name](), 3, seed=5, kernel_mode=N.KERNEL_WAVEFRONT)
        imgs.append(img.copy())
        ctx.destroy_job(s.job_id())
        ctx.close()
    np.testing.assert_array_equal(imgs[0], imgs[1])
    np.testing.assert_array_equal(imgs[0], imgs[2])


@pytest.mark.parametrize("name", ["c1", "atmosphere"])
def test_wavefront_split_does_not_change_results(name):
    """The wavefront splits a large image into pixel ranges whose stages run on concurrent
    streams, as contiguous runs of rows or as the rows dealt to the ranges in turn; one, two and
    four contiguous ranges and three and four interleaved ones give the same image bit for bit (a
    path's computation does not depend on its range). 512 rows over three ranges leave them
    unequal (171, 171 and 170 rows)."""
    import os
    from snelly_b200 import api
    imgs = []
    for split, interleave in (("1", "0"), ("2", "0"), ("4", "0"), ("3", "1"), ("4", "1")):
        saved = {k: os.environ.pop(k, None) for k in ("SNELLY_WF_SPLIT", "SNELLY_WF_INTERLEAVE")}
        os.environ["SNELLY_WF_SPLIT"] = split
        os.environ["SNELLY_WF_INTERLEAVE"] = interleave
        try:
            ctx = api.Context(0)
        finally:
            for k, v in saved.items():
                os.environ.pop(k, None)
                if v is not None:
                    os.environ[k] = v
        scene = {"c1": scenes.DispersiveFractal, "atmosphere": scenes.AtmosphereLights}[name](512, 512)
        s, img = gpu_render(ctx, scene, 2, seed=5, kernel_mode=N.KERNEL_WAVEFRONT)
        cfg = ctx.job_wavefront_config(s.job_id())
        assert (cfg["parts"], cfg["interleave"]) == (int(split), int(interleave)), cfg
        imgs.append(img.copy())
        ctx.destroy_job(s.job_id())
        ctx.close()
    for other in imgs[1:]:
        np.testing.assert_array_equal(imgs[0], other)


def test_wavefront_paths_without_shadow_rays_finish_once(gpu_ctx):
    """A path whose last vertex samples no light (no sky; the sun below the vertex's horizon) has
    no ray to wait for and goes straight to the next shade stage's queue while the current stage
    still reads its own. Every pixel must finish every frame exactly once, and the image must
    equal the path-per-thread kernel's under strict math (same bar as above: >= 97% of pixels
    within 1e-5, the rest differ in the summation order of the deferred estimate)."""
    frames = 3
    a = gpu_render(gpu_ctx, scenes.LowSunNoSky(256, 256), frames, seed=7, math_mode=N.MATH_STRICT,
                   kernel_mode=N.KERNEL_MEGA)[1].reshape(-1, 4)
    s, b = gpu_render(gpu_ctx, scenes.LowSunNoSky(256, 256), frames, seed=7, math_mode=N.MATH_STRICT,
                      kernel_mode=N.KERNEL_WAVEFRONT)
    b = b.reshape(-1, 4)
    rng, acc, comp, _ = s.readback_state()
    assert (acc[:, 3] == frames).all(), np.unique(acc[:, 3], return_counts=True)
    assert (b[:, 3] == frames).all()
    ok = _close(b[:, :3], a[:, :3], 1e-5)
    assert ok.mean() >= 0.97, ok.mean()


@pytest.mark.parametrize("name", ["c2", "c2_cloud"])
def test_persistent_walker_does_not_change_results(name):
    """Subsurface walks run by the persistent walker (each lane taking the next walk when its own
    ends) or one thread per walk give the same image bit for bit: every path draws its random
    numbers in the same order either way."""
    import os
    from snelly_b200 import api
    imgs = []
    for walker in ("0", "1"):
        old = os.environ.pop("SNELLY_WF_WALKER", None)
        os.environ["SNELLY_WF_WALKER"] = walker
        try:
            ctx = api.Context(0)
        finally:
            os.environ.pop("SNELLY_WF_WALKER", None)
            if old is not None:
                os.environ["SNELLY_WF_WALKER"] = old
        scene = {"c2": scenes.VolumetricSubsurface, "c2_cloud": scenes.PyroclasticSubsurface}[name](64, 64)
        s, img = gpu_render(ctx, scene, 3, seed=5, kernel_mode=N.KERNEL_WAVEFRONT)
        assert ctx.job_wavefront_config(s.job_id())["walker"] == int(walker)
        imgs.append(img.copy())
        ctx.destroy_job(s.job_id())
        ctx.close()
    np.testing.assert_array_equal(imgs[0], imgs[1])


@pytest.mark.parametrize("math_mode", [None, N.MATH_STRICT])
def test_volume_stage_does_not_change_results(math_mode):
    """Vertices that collide in the heterogeneous medium (C2's cloud) scatter in a stage of their
    own, one thread per medium vertex with its shadow marches, or inside the shade stage: the same
    functions run in the same order on the path's random numbers, so the image is the same bit for
    bit, in the production and the IEEE-strict builds. The stage's launches show that it ran."""
    import os
    from snelly_b200 import api
    imgs, launches = [], []
    for stage in ("0", "1"):
        old = os.environ.pop("SNELLY_WF_VOLUME", None)
        os.environ["SNELLY_WF_VOLUME"] = stage
        try:
            ctx = api.Context(0)
        finally:
            os.environ.pop("SNELLY_WF_VOLUME", None)
            if old is not None:
                os.environ["SNELLY_WF_VOLUME"] = old
        before = ctx.launch_count()
        s, img = gpu_render(ctx, scenes.PyroclasticSubsurface(64, 64), 3, seed=5, math_mode=math_mode,
                            kernel_mode=N.KERNEL_WAVEFRONT)
        launches.append(ctx.launch_count() - before)
        assert ctx.job_wavefront_config(s.job_id())["volume_stage"] == int(stage)
        imgs.append(img.copy())
        ctx.destroy_job(s.job_id())
        ctx.close()
    assert launches[1] > launches[0], launches
    np.testing.assert_array_equal(imgs[0], imgs[1])


@pytest.mark.parametrize("name", ["c1", "c2", "c2_cloud", "lowsun", "hooks", "atmosphere"])
def test_overlapping_frames_do_not_change_results(name):
    """The frames of one advance run overlapped (a path that finishes its pixel's sample starts the
    pixel's next one in place) or one after another give the same image bit for bit: each pixel
    draws its random numbers and adds its samples in the same order either way."""
    import os
    from snelly_b200 import api
    imgs = []
    for overlap in ("0", "1"):
        old = os.environ.pop("SNELLY_WF_OVERLAP", None)
        os.environ["SNELLY_WF_OVERLAP"] = overlap
        try:
            ctx = api.Context(0)
        finally:
            os.environ.pop("SNELLY_WF_OVERLAP", None)
            if old is not None:
                os.environ["SNELLY_WF_OVERLAP"] = old
        scene = scenes.SCENES[name](96, 64)
        s, img = gpu_render(ctx, scene, 5, seed=7, kernel_mode=N.KERNEL_WAVEFRONT)
        assert ctx.job_wavefront_config(s.job_id())["overlap"] == int(overlap)
        imgs.append(img.copy())
        ctx.destroy_job(s.job_id())
        ctx.close()
    np.testing.assert_array_equal(imgs[0], imgs[1])
