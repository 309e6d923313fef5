"""The host-side mirror of the reference's scene API: uniform conversions, camera, materials."""
import math

import numpy as np

from snelly_b200 import api, scenes
from snelly_b200.testing import HostSnelly


def test_material_catalogue():
    m = api.Materials()
    assert len(m.metals) == 22 and len(m.dielectrics) == 23
    assert m.getLoadedDielectric().getName() == "Glass (BK7)" and m.getLoadedMetal().getName() == "Aluminium"
    assert m.dielectrics["Glass (BK7)"].model == "sellmeier" and m.dielectrics["Glycerol"].model == "cauchy"


def test_camera_basis_lookat():
    pos, d, x, y = api.camera_basis([0.0, 1.0, 5.0], [0.0, 0.0, 0.0], [0.0, 1.0, 0.0])
    n = math.sqrt(26.0)
    assert np.allclose(d, [0.0, -1.0 / n, -5.0 / n])
    assert np.allclose(x, [-1.0, 0.0, 0.0])  # camX = camUp x camDir points to screen-left
    assert np.allclose(y, [0.0, 5.0 / n, -1.0 / n])
    assert abs(np.dot(d, y)) < 1e-12


def test_uniform_conversions():
    h = HostSnelly(scenes.DispersiveFractal(64, 36))
    p = h.uniform_params()
    r = h.getRenderer()
    assert math.isclose(p.skyPower, 0.5, rel_tol=1e-6) and math.isclose(p.sunPower, 20.0, rel_tol=1e-6)
    assert math.isclose(p.radianceClamp, 1000.0)
    assert p.camAperture == 0.0
    lat = (90.0 - r.sunLatitude) * math.pi / 180.0
    assert np.allclose(list(p.sunDir), [math.sin(lat) * math.cos(math.radians(30)), math.cos(lat),
                                        math.sin(lat) * math.sin(math.radians(30))], atol=1e-6)
    assert p.dieleModel == 4 and p.dieleNumCoeffs == 3 and list(p.dieleCoeffs[:3]) == [1.5, np.float32(0.0042), -2.0]
    assert np.allclose(list(p.metalN), api.DATA["metal_tables"]["gold"]["n"], atol=1e-6)
    h2 = HostSnelly(scenes.AtmosphereLights())
    p2 = h2.uniform_params()
    assert math.isclose(p2.sphereLightPower, 40.0 / (4 * math.pi * 0.3 ** 2), rel_tol=1e-6)
    assert math.isclose(p2.sphereLightRadius, 0.3, rel_tol=1e-6)
    assert math.isclose(p2.camAperture, 1.4142135 ** -4.0, rel_tol=1e-6)
    # Dielectric.syncShader absorption: lengthScale / absorptionScale * (1 - colour)
    assert np.allclose(list(p2.dieleAbsorptionRGB), [0.5 * 0.4, 0.5 * 0.1, 0.5 * 0.2], atol=1e-6)
    assert math.isclose(p2.atmosphereMFP, 10 ** 0.6, rel_tol=1e-6)
    assert list(p2.atmosphereExtinctionCoeffRGB) == list(np.float32([0.4, 0.45, 0.58]))


def test_scene_options_follow_renderer():
    h = HostSnelly(scenes.AtmosphereLights())
    o = h.scene_opts()
    assert (o.has_atmosphere, o.has_fog, o.has_sphere_light, o.max_bounces, o.max_atmosphere_scatters) == (1, 1, 1, 5, 3)
    h = HostSnelly(scenes.PlainSphere())
    o = h.scene_opts()
    assert (o.has_atmosphere, o.has_sphere_light, o.dispersive, o.interactive) == (0, 0, 1, 0)


def test_scene_uniform_recording():
    h = HostSnelly(scenes.HooksAndMaps())
    calls = h.scene_uniforms()
    assert calls["ripple"][1] == [1.5] and calls["tint"][1] == [0.1, 0.6, 0.2]


def test_png_decode_all_scanline_filters():
    """decode_png undoes the five PNG filter types (hand-filtered rows) and reads back what
    png_bytes wrote."""
    import struct
    import zlib

    from snelly_b200 import image
    rs = np.random.RandomState(2)
    h, w, c = 6, 5, 4
    img = rs.randint(0, 256, (h, w, c)).astype(np.uint8)

    def paeth(a, b, cc):
        p = a + b - cc
        pa, pb, pc = abs(p - a), abs(p - b), abs(p - cc)
        return a if pa <= pb and pa <= pc else (b if pb <= pc else cc)

    flat = img.reshape(h, w * c).astype(int)
    rows = []
    for y in range(h):
        f = y % 5
        prev = flat[y - 1] if y else np.zeros(w * c, int)
        line = []
        for i in range(w * c):
            a_ = flat[y, i - c] if i >= c else 0
            b_ = prev[i]
            c_ = prev[i - c] if i >= c else 0
            pred = [0, a_, b_, (a_ + b_) >> 1, paeth(a_, b_, c_)][f]
            line.append((flat[y, i] - pred) & 255)
        rows.append(bytes([f]) + bytes(line))

    def chunk(tag, data):
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)

    png = (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0)) +
           chunk(b"IDAT", zlib.compress(b"".join(rows))) + chunk(b"IEND", b""))
    np.testing.assert_array_equal(image.decode_png(png), img)
    rgb = rs.randint(0, 256, (7, 9, 3)).astype(np.uint8)
    np.testing.assert_array_equal(image.decode_png(image.png_bytes(rgb)), rgb)


def test_sdf_png_round_trip(tmp_path):
    """The packer's SDF-PNG layout (magic, version, sizes, JSON metadata, float32 samples in the
    RGB bytes of a square image) round-trips, and load_texture gives the sampler3D shape."""
    from snelly_b200 import scenes, sdfpng
    g = scenes.sphere_blend_grid(16)[..., 0].astype(np.float32)
    md = {"GRES": [16, 16, 16], "ORIG": [-1.5, -1.5, -1.5], "EDGE": [3.0, 3.0, 3.0]}
    png = sdfpng.pack(g, md)
    raw = __import__("snelly_b200.image", fromlist=["x"]).decode_png(png)[..., :3].reshape(-1)
    assert raw[0] == 0xBE and raw[1] == 0xEF and raw[2] == 1 and raw[3] == 0
    path = tmp_path / "grid.png"
    path.write_bytes(png)
    meta, tex = sdfpng.load_texture(str(path))
    assert meta == md and tex.shape == (16, 16, 16, 1)
    np.testing.assert_array_equal(tex[..., 0], g)


def test_env_map_from_png_file_equals_array(tmp_path):
    """Scene.envMap may return a PNG path (the reference returns a URL) or an array: both bind
    the same sRGB8 texels, row 0 the top row of the image."""
    from snelly_b200 import image, scenes
    from snelly_b200.testing import HostSnelly
    arr = scenes.sky_env_map()
    path = tmp_path / "env.png"
    image.write_png(str(path), arr)

    class FromFile(scenes.EnvMapLit):
        def envMap(self):
            return str(path)

    a = HostSnelly(scenes.EnvMapLit(16, 16)).env_map()
    b = HostSnelly(FromFile(16, 16)).env_map()
    np.testing.assert_array_equal(a, b)
    assert a.shape == (32, 64, 3)


def test_sdf_asset_scene_binds_the_packed_grid(tmp_path):
    from snelly_b200 import scenes, sdfpng
    from snelly_b200.testing import HostSnelly
    g = scenes.sphere_blend_grid(16)[..., 0].astype(np.float32)
    path = tmp_path / "asset.png"
    path.write_bytes(sdfpng.pack(g, {"GRES": [16, 16, 16], "ORIG": [-1.0, -1.0, -1.0], "EDGE": [2.0, 2.0, 2.0]}))
    sh = HostSnelly(scenes.SdfAsset(str(path), 16, 16)).scene_shader()
    tex, linear = sh.textures["sdfTex"]
    assert tex.shape == (16, 16, 16, 1) and tex.dtype == np.float32 and linear
    assert sh.calls["gridMin"][1] == [-1.0, -1.0, -1.0] and sh.calls["gridSize"][1] == [2.0, 2.0, 2.0]


def test_module_cache_prune_drops_modules_older_than_their_sources(tmp_path):
    """A cached module compiled before the latest edit of a file its key includes can never be
    asked for again and is deleted; one compiled after it is kept, and so are files that are not
    modules."""
    import os
    from snelly_b200 import build as B
    src = tmp_path / "kernel.cuh"
    src.write_text("// source")
    cache = tmp_path / "kcache"
    cache.mkdir()
    old, new, other = cache / "old.cubin", cache / "new.cubin", cache / "notes.txt"
    for f in (old, new, other):
        f.write_bytes(b"x")
    t = os.path.getmtime(src)
    os.utime(old, (t - 100, t - 100))
    os.utime(other, (t - 100, t - 100))
    os.utime(new, (t + 100, t + 100))
    assert B.prune_module_cache(str(cache), [str(src)]) == 1
    assert sorted(os.listdir(cache)) == ["new.cubin", "notes.txt"]
    assert all(os.path.exists(f) for f in B.module_key_sources())
