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
