"""Generate the golden fixtures of tests/golden/ from the reference itself.

Run with $SNELLY_REFERENCE naming a checkout of the reference:
    SNELLY_REFERENCE=<checkout> python tests/golden/make_golden.py

* pt_<case>.npz: the reference's own path tracer shader (shaders/pathtracer-fragment-shader.glsl,
  built for the CPU by oracle/build_ref.py) rendering a small image of one of the package's
  scenes: inputs (scene case, size, frames, seed, the initial per-pixel RNG lanes) and outputs
  (per-pixel running mean X, Y, Z, N after `frames` frames, final RNG lanes).
* fh_<case>.npz: the reference's first-hit programs (shaders/normals-fragment-shader.glsl,
  ao-fragment-shader.glsl, pick-fragment-shader.glsl, built the same way) on the same scenes:
  normals and AO running means and RNG lanes after a few frames, pick distance and material at
  every pixel centre. `python tests/golden/make_golden.py fh` regenerates only these.
* ps_<case>.npz: the reference's simplified path tracer (renderMode 'ptsimple',
  simplepathtracer-fragment-shader.glsl) on the same scenes: running means and RNG lanes.
* tm_golden.npz: the reference's tonemapper program on path-traced and synthetic XYZ texels for
  three display settings.
* bench_c1.npz: the benchmark's own workload (1920x1080 dispersive Menger sponge, gold sphere,
  ground; seed 2) through the reference's path tracer: 20,000 fixed random pixels x 2 frames with
  the seeds the GPU uses for the same pixels (running means and final RNG lanes).
* stat_<case>.npz: the reference's path tracer at matched spp with independent seeds, for
  statistical comparison: a 256x256 crop of the 1080p benchmark frame at 64 spp (16 batches of 4
  frames), and the C0 image at its own 256x256 and 16 spp (16 batches of 1 frame); per-pixel mean
  and variance of the batch-mean luminance, and every batch's image-mean luminance.
* cie_csv.npy: the CIE XYZ table recomputed from scripts/color/lin2012xyz2e_fine_7sf.csv as
  scripts/color/cie.py does (linear interpolation to 1024 samples over 390..750 nm, both ends
  included), to pin the table in snelly_b200/data/materials.json.
"""
import csv
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from snelly_b200 import scenes  # noqa: E402
from snelly_b200.testing import HostSnelly  # noqa: E402
import build_ref  # noqa: E402
import oracle  # noqa: E402

CASES = {
    "c0": (lambda: scenes.PlainSphere(64, 64), 8),
    "c1": (lambda: scenes.DispersiveFractal(64, 36), 4),
    "c1_rgb": (lambda: scenes.DispersiveFractal(48, 27, dispersive=False), 3),
    "c2": (lambda: scenes.VolumetricSubsurface(32, 32), 2),
    "atmosphere": (lambda: scenes.AtmosphereLights(64, 48), 3),
    "atmosphere_disp": (lambda: scenes.AtmosphereLights(32, 24, dispersive=True), 2),
    "hooks": (lambda: scenes.HooksAndMaps(48, 48), 3),
    "mesh": (lambda: scenes.MeshLike(48, 48, res=64), 3),
    "envmap": (lambda: scenes.EnvMapLit(48, 48), 3),
    "abbe": (lambda: scenes.DispersiveSphere(40, 40, "Abbe dielectric", abbe=32.0, ior=1.62), 3),
    "polyanskiy": (lambda: scenes.DispersiveSphere(40, 40, "Rutile"), 3),
}
SEED = 1


def make_pt(name):
    factory, frames = CASES[name]
    h = HostSnelly(factory())
    ref, p, tables, keep = build_ref.ref_for(h)
    lib = oracle.OracleLib(h.sceneObj.shader(), h.scene_opts())
    pix = np.arange(h.width * h.height)
    rng0 = lib.seed(SEED, pix)
    sh = h.scene_shader()
    mean, rng = ref.render(p, sh.calls, tables, h.width, h.height, pix, frames, rng0, scene_textures=sh.textures)
    np.savez_compressed(os.path.join(HERE, f"pt_{name}.npz"), case=name, width=h.width, height=h.height,
                        frames=frames, seed=SEED, rng0=rng0, mean=mean, rng=rng)
    print(f"pt_{name}: {h.width}x{h.height}, {frames} frames, mean XYZ {mean[:, :3].mean(0)}")


FH_CASES = ("c0", "c1", "c2", "atmosphere", "hooks", "mesh", "envmap")
FH_FRAMES = 3


def make_firsthit(name):
    """fh_<case>.npz: the reference's normals and ambient-occlusion programs (FH_FRAMES frames,
    running mean and final RNG lanes) and its pick program at every pixel centre."""
    factory, _ = CASES[name]
    h = HostSnelly(factory())
    lib = oracle.OracleLib(h.sceneObj.shader(), h.scene_opts())
    pix = np.arange(h.width * h.height)
    rng0 = lib.seed(SEED, pix)
    out = dict(case=name, width=h.width, height=h.height, frames=FH_FRAMES, seed=SEED, rng0=rng0)
    sh = h.scene_shader()
    for prog in ("normals", "ao"):
        ref, p, tables, keep = build_ref.ref_for(h, program=prog)
        mean, rng = ref.render(p, sh.calls, tables, h.width, h.height, pix, FH_FRAMES, rng0, scene_textures=sh.textures)
        out[prog + "_mean"] = mean
        out[prog + "_rng"] = rng
    ref, p, tables, keep = build_ref.ref_for(h, program="pick")
    out["pick"] = ref.pick(p, sh.calls, tables, h.width, pix, scene_textures=sh.textures)
    np.savez_compressed(os.path.join(HERE, f"fh_{name}.npz"), **out)
    print(f"fh_{name}: {h.width}x{h.height}, normals/ao {FH_FRAMES} frames, pick hits {(out['pick'][:, 1] >= 0).mean():.3f}")


PS_FRAMES = 3


def make_ptsimple(name):
    """ps_<case>.npz: the reference's simplified path tracer (simplepathtracer-fragment-shader.glsl,
    renderMode 'ptsimple'), PS_FRAMES frames: running mean and final RNG lanes."""
    factory, _ = CASES[name]
    h = HostSnelly(factory())
    lib = oracle.OracleLib(h.sceneObj.shader(), h.scene_opts())
    pix = np.arange(h.width * h.height)
    rng0 = lib.seed(SEED, pix)
    ref, p, tables, keep = build_ref.ref_for(h, program="simplepathtracer")
    sh = h.scene_shader()
    mean, rng = ref.render(p, sh.calls, tables, h.width, h.height, pix, PS_FRAMES, rng0, scene_textures=sh.textures)
    np.savez_compressed(os.path.join(HERE, f"ps_{name}.npz"), case=name, width=h.width, height=h.height,
                        frames=PS_FRAMES, seed=SEED, rng0=rng0, mean=mean, rng=rng)
    print(f"ps_{name}: {h.width}x{h.height}, {PS_FRAMES} frames, mean XYZ {mean[:, :3].mean(0)}")


BENCH_C1_PIXELS, BENCH_C1_FRAMES, BENCH_C1_SEED = 20000, 2, 2


def make_bench_c1():
    """bench_c1.npz: matched seeds on the benchmark's own 1080p frame (see the module docstring)."""
    h = HostSnelly(scenes.DispersiveFractal())
    ref, p, tables, keep = build_ref.ref_for(h, name="bench_c1")
    n = h.width * h.height
    pix = np.sort(np.random.RandomState(20).choice(n, BENCH_C1_PIXELS, replace=False)).astype(np.int32)
    rng0 = oracle.seed_pixels(BENCH_C1_SEED, pix)
    sh = h.scene_shader()
    mean, rng = ref.render(p, sh.calls, tables, h.width, h.height, pix, BENCH_C1_FRAMES, rng0, scene_textures=sh.textures)
    np.savez_compressed(os.path.join(HERE, "bench_c1.npz"), width=h.width, height=h.height, frames=BENCH_C1_FRAMES,
                        seed=BENCH_C1_SEED, pixels=pix, mean=mean, rng=rng)
    print(f"bench_c1: {len(pix)} pixels of {h.width}x{h.height}, {BENCH_C1_FRAMES} frames, mean XYZ {mean[:, :3].mean(0)}")


# (scene factory, crop (x0, y0, w, h) or None for the whole image, batches, frames per batch)
STAT_CASES = {
    "c1_crop": (lambda: scenes.DispersiveFractal(), (832, 412, 256, 256), 16, 4),
    "c0": (lambda: scenes.PlainSphere(), None, 16, 1),
}
STAT_SEED0 = 1000


def stat_pixels(h, crop):
    if crop is None:
        return np.arange(h.width * h.height, dtype=np.int32)
    x0, y0, w, hh = crop
    ys, xs = np.mgrid[y0:y0 + hh, x0:x0 + w]
    return (ys * h.width + xs).reshape(-1).astype(np.int32)


def stat_batches(name, seed0):
    """Per-batch mean luminance (batches, pixels) of the reference's path tracer for STAT_CASES[name]."""
    factory, crop, batches, frames = STAT_CASES[name]
    h = HostSnelly(factory())
    ref, p, tables, keep = build_ref.ref_for(h, name="bench_c1" if name == "c1_crop" else None)
    pix = stat_pixels(h, crop)
    sh = h.scene_shader()
    ys = np.empty((batches, len(pix)), np.float64)
    for b in range(batches):
        rng0 = oracle.seed_pixels(seed0 + b, pix)
        mean, _ = ref.render(p, sh.calls, tables, h.width, h.height, pix, frames, rng0, scene_textures=sh.textures)
        ys[b] = mean[:, 1]
    return ys


def make_stat(name):
    factory, crop, batches, frames = STAT_CASES[name]
    ys = stat_batches(name, STAT_SEED0)
    np.savez_compressed(os.path.join(HERE, f"stat_{name}.npz"), crop=np.asarray(crop or (0, 0, 0, 0), np.int32),
                        batches=batches, frames=frames, seed0=STAT_SEED0, y_mean=ys.mean(0).astype(np.float32),
                        y_var=ys.var(0, ddof=1).astype(np.float32), img_means=ys.mean(1))
    print(f"stat_{name}: {ys.shape[1]} pixels, {batches} x {frames} frames, image mean Y {ys.mean():.6f}")


FULL_BATCHES, FULL_FRAMES, FULL_SEED0, FULL_TILE = 10, 16, 7000, 30


def make_full_c1():
    """full_c1.npz: the reference's path tracer over the whole 1080p benchmark frame at
    FULL_BATCHES x FULL_FRAMES spp (independent seeds per batch): each batch's image-mean XYZ and
    its mean XYZ over FULL_TILE x FULL_TILE pixel tiles. The image mean luminance is known to about
    0.1% from this, which the 0.5% bar needs (a 256x256 crop at 64 spp leaves a 1% standard
    error: the sun's caustics through the sponge make the estimator heavy-tailed)."""
    h = HostSnelly(scenes.DispersiveFractal())
    ref, p, tables, keep = build_ref.ref_for(h, name="bench_c1")
    W, H = h.width, h.height
    pix = np.arange(W * H, dtype=np.int32)
    sh = h.scene_shader()
    img, tiles = [], []
    for b in range(FULL_BATCHES):
        rng0 = oracle.seed_pixels(FULL_SEED0 + b, pix)
        mean, _ = ref.render(p, sh.calls, tables, W, H, pix, FULL_FRAMES, rng0, scene_textures=sh.textures)
        m = mean[:, :3].astype(np.float64).reshape(H, W, 3)
        img.append(m.mean((0, 1)))
        tiles.append(m.reshape(H // FULL_TILE, FULL_TILE, W // FULL_TILE, FULL_TILE, 3).mean((1, 3)))
        print(f"full_c1 batch {b}: image mean XYZ {img[-1]}", flush=True)
    np.savez_compressed(os.path.join(HERE, "full_c1.npz"), batches=FULL_BATCHES, frames=FULL_FRAMES, seed0=FULL_SEED0,
                        tile=FULL_TILE, img_xyz=np.asarray(img), tile_xyz=np.asarray(tiles, np.float32))


TM_PARAMS = [  # exposure, invGamma (= 1/gamma as the host uploads it), contrast, saturation, hueShift
    (0.0, 1.0 / 2.2, 1.0, 1.0, 0.0),   # the Renderer defaults (js/renderer.js:118-122)
    (1.5, 1.0 / 1.8, 1.3, 0.8, 0.25),
    (-2.0, 1.0, 0.7, 1.6, 0.9),
]


def make_tonemap():
    """tm_golden.npz: the reference's tonemapper program (shaders/tonemapper-fragment-shader.glsl)
    on path-traced mean images and on wide-range synthetic XYZ values (out-of-gamut and HDR), for
    three sets of display settings."""
    rs = np.random.RandomState(11)
    c1 = np.load(os.path.join(HERE, "pt_c1.npz"))["mean"]
    atm = np.load(os.path.join(HERE, "pt_atmosphere.npz"))["mean"][:1024]
    x = np.concatenate([c1, atm, np.abs(rs.standard_cauchy((1024, 4))), rs.uniform(-0.2, 3.0, (1024, 4))]).astype(np.float32)
    x[:, 3] = 1.0
    ref = build_ref.tonemapper_lib()
    names = ["exposure", "invGamma", "contrast", "saturation", "hueShift"]
    outs = np.stack([ref.tonemap(x, dict(zip(names, p))) for p in TM_PARAMS])
    np.savez_compressed(os.path.join(HERE, "tm_golden.npz"), xyzn=x, params=np.asarray(TM_PARAMS, np.float32), rgba=outs)
    print(f"tm_golden: {len(x)} texels x {len(TM_PARAMS)} settings")


def make_cie():
    assert build_ref.have_reference(), "set $SNELLY_REFERENCE to a checkout of the reference"
    path = os.path.join(build_ref.REF_ROOT, "scripts", "color", "lin2012xyz2e_fine_7sf.csv")
    rows = [r for r in csv.reader(open(path))]
    lam = np.array([float(r[0]) for r in rows])
    xyz = np.array([[float(r[1]), float(r[2]), float(r[3])] for r in rows])
    l_res = 390.0 + (750.0 - 390.0) / 1023.0 * np.arange(1024)
    out = np.stack([np.interp(l_res, lam, xyz[:, c]) for c in range(3)], 1)
    np.save(os.path.join(HERE, "cie_csv.npy"), out)
    print("cie_csv: 1024 x 3")


if __name__ == "__main__":
    if not build_ref.have_reference():
        sys.exit("set $SNELLY_REFERENCE to a checkout of the reference")
    only = sys.argv[1:]
    if not only or "cie" in only:
        make_cie()
    for n in CASES:
        if not only or "pt" in only:
            make_pt(n)
    for n in FH_CASES:
        if not only or "fh" in only:
            make_firsthit(n)
    for n in FH_CASES:
        if not only or "ps" in only:
            make_ptsimple(n)
    if not only or "bench" in only:
        make_bench_c1()
    for n in STAT_CASES:
        if not only or "stat" in only:
            make_stat(n)
    if "full" in only:  # about 460 M path samples: tens of minutes on a few host cores
        make_full_c1()
    if not only or "tm" in only:
        make_tonemap()
