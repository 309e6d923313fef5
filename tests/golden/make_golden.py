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
    if not only or "tm" in only:
        make_tonemap()
