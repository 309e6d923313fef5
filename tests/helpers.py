"""Shared test helpers: golden fixtures, oracle builds, GPU renders."""
import os

import numpy as np

from snelly_b200 import scenes
from snelly_b200.testing import HostSnelly

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

CASES = {
    "c0": lambda: scenes.PlainSphere(64, 64),
    "c1": lambda: scenes.DispersiveFractal(64, 36),
    "c1_rgb": lambda: scenes.DispersiveFractal(48, 27, dispersive=False),
    "c2": lambda: scenes.VolumetricSubsurface(32, 32),
    "atmosphere": lambda: scenes.AtmosphereLights(64, 48),
    "atmosphere_disp": lambda: scenes.AtmosphereLights(32, 24, dispersive=True),
    "hooks": lambda: scenes.HooksAndMaps(48, 48),
    "mesh": lambda: scenes.MeshLike(48, 48, res=64),
    "envmap": lambda: scenes.EnvMapLit(48, 48),
    "abbe": lambda: scenes.DispersiveSphere(40, 40, "Abbe dielectric", abbe=32.0, ior=1.62),
    "polyanskiy": lambda: scenes.DispersiveSphere(40, 40, "Rutile"),
}


FH_CASES = ("c0", "c1", "c2", "atmosphere", "hooks", "mesh", "envmap")


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, f"pt_{name}.npz")))


def golden_ps(name):
    return dict(np.load(os.path.join(GOLDEN, f"ps_{name}.npz")))


def golden_fh(name):
    return dict(np.load(os.path.join(GOLDEN, f"fh_{name}.npz")))


def oracle_firsthit(host, mode, pixels, frames, rng0=None, threads=0):
    """The oracle's first-hit programs (mode 1 normals, 2 AO, 3 pick) for the listed pixels."""
    import oracle
    lib = oracle_for(host)
    if rng0 is None and mode != 3:
        rng0 = lib.seed(host.seed, pixels)
    p, keep = oracle.host_params(host)
    sh = host.scene_shader()
    ub = oracle.pack_uniforms(lib.cpp, sh.calls, sh.textures, params=p)
    return lib.firsthit(mode, p, ub, host.width, host.height, pixels, frames, rng0, threads)


def oracle_for(host):
    import oracle
    return oracle.OracleLib(host.sceneObj.shader(), host.scene_opts())


def oracle_render(host, pixels, frames, rng0=None, threads=0):
    import oracle
    lib = oracle_for(host)
    if rng0 is None:
        rng0 = lib.seed(host.seed, pixels)
    p, keep = oracle.host_params(host)
    sh = host.scene_shader()
    ub = oracle.pack_uniforms(lib.cpp, sh.calls, sh.textures, params=p)
    return lib.render(p, ub, host.width, host.height, pixels, frames, rng0, threads)


def gpu_render(ctx, scene, frames, seed=1, math_mode=None, kernel_mode=None, fp64=False):
    """Render `frames` frames of `scene` through the scene API on the GPU; returns the Snelly
    object and its (H, W, 4) mean image."""
    from snelly_b200 import api
    from snelly_b200 import _native as N
    s = api.Snelly(scene, context=ctx)
    s.seed = seed
    if math_mode is not None:
        s.pathtracer.mathMode = math_mode
    if kernel_mode is not None:
        s.pathtracer.kernelMode = kernel_mode
    s.fp64 = fp64
    s.render(frames)
    return s, s.readback()


def host(name):
    return HostSnelly(CASES[name]())


def welch_p(a_mean, a_var, na, b_mean, b_var, nb):
    """Two-sided p-values of Welch's two-sample t statistic per element (Welch-Satterthwaite
    degrees of freedom), for means and unbiased variances of na and nb samples; NaN where both
    variances are zero."""
    from scipy import stats
    va, vb = a_var / na, b_var / nb
    se2 = va + vb
    with np.errstate(divide="ignore", invalid="ignore"):
        t = np.abs(a_mean - b_mean) / np.sqrt(se2)
        dof = se2 ** 2 / (va ** 2 / (na - 1) + vb ** 2 / (nb - 1))
    p = 2.0 * stats.t.sf(t, dof)
    p[se2 <= 0] = np.nan
    return p
