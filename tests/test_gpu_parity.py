"""The CUDA path tracer against the reference (golden fixtures) and the oracle: per pixel with
matched seeds, and statistically with independent seeds. Tolerances are written in each test."""
import numpy as np
import pytest

from helpers import CASES, golden, gpu_render, host, oracle_render
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


@pytest.mark.parametrize("kernel", sorted(KERNELS))
@pytest.mark.parametrize("name", sorted(CASES))
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


@pytest.mark.parametrize("kernel", sorted(KERNELS))
@pytest.mark.parametrize("scene_factory,frames_per_batch", [
    (lambda: scenes.DispersiveFractal(160, 92), 4),
    (lambda: scenes.PlainSphere(96, 96), 4),
])
def test_statistical_agreement_independent_seeds(gpu_ctx, scene_factory, frames_per_batch, kernel):
    """GPU and oracle with independent seeds agree within Monte Carlo error: image mean luminance
    within 0.5%; per-pixel luminance differences beyond 3 standard errors in at most 5% of pixels
    (16 GPU batches give the per-pixel variance; caustic and firefly pixels of the dispersive glass
    under a small sun have heavy-tailed estimators whose 16-batch variance underestimates the spread,
    so more than the Gaussian 0.3-0.9% exceed 3 SE); and over 4x4-pixel tiles, whose means are
    closer to Gaussian, in at most 2% of tiles."""
    batches = 16
    ys = []
    for b in range(batches):
        s, img = gpu_render(gpu_ctx, scene_factory(), frames_per_batch, seed=1000 + b, kernel_mode=KERNELS[kernel])
        ys.append(img[..., 1].reshape(-1))
        gpu_ctx.destroy_job(s.job_id())
    ys = np.array(ys, np.float64)
    g_mean = ys.mean(0)
    var_b = ys.var(0, ddof=1)  # variance of a frames_per_batch-frame mean
    h = host("c0")
    from snelly_b200.testing import HostSnelly
    h = HostSnelly(scene_factory(), seed=777)
    pix = np.arange(h.width * h.height)
    of = 4 * frames_per_batch
    xyz, mean, _ = oracle_render(h, pix, of)
    o_mean = xyz[:, 1] / of
    se = np.sqrt(var_b / batches + var_b * frames_per_batch / of)
    mask = se > 0
    z = np.abs(g_mean - o_mean)[mask] / se[mask]
    frac = (z > 3).mean()
    lum_g, lum_o = g_mean.mean(), o_mean.mean()
    # 4x4 tiles: batch means of the tile average, the same test
    H, W = h.height, h.width
    def tiles(a):
        a = a.reshape(*a.shape[:-1], H // 4, 4, W // 4, 4)
        return a.mean(axis=(-1, -3)).reshape(*a.shape[:-4], -1)
    yt = tiles(ys)
    ot = tiles(o_mean)
    tvar = yt.var(0, ddof=1)
    tse = np.sqrt(tvar / batches + tvar * frames_per_batch / of)
    tz = np.abs(yt.mean(0) - ot)[tse > 0] / tse[tse > 0]
    tfrac = (tz > 3).mean()
    msg = f"pixels beyond 3 SE {frac:.4f}, tiles {tfrac:.4f}, mean lum gpu {lum_g:.6f} oracle {lum_o:.6f}"
    assert abs(lum_g - lum_o) / lum_o <= 5e-3, msg
    assert frac <= 0.05, msg
    assert tfrac <= 0.02, msg
    assert (np.abs(g_mean - o_mean)[~mask] < 1e-5).all()


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
