"""The headless scene-API facade without a GPU: dumpScene / initGenerator, the per-frame render
loop (pre/post-frame callbacks, maxSpp, isReady, parameter changes between frames, reset with and
without a recompile), driven through a recording stand-in for the C ABI context."""
import math

import pytest

from snelly_b200 import api, scenes
from snelly_b200.testing import HostSnelly


class RecordingContext:
    """Records what the facade asks of libsnelly; renders nothing."""

    def __init__(self):
        self.events = []
        self.scenes = {}
        self.next_job = 0
        self.live = set()

    def scene_for(self, glsl, opts):
        key = (glsl, bytes(opts))
        if key not in self.scenes:
            self.scenes[key] = len(self.scenes) + 1
            self.events.append(("compile", opts.max_bounces))
        return self.scenes[key]

    def set_uniforms(self, sid, calls):
        self.events.append(("uniforms", sid, dict(calls)))

    def set_texture(self, sid, name, tex, linear=True):
        self.events.append(("texture", sid, name))

    def render(self, sid, desc):
        self.next_job += 1
        self.live.add(self.next_job)
        self.events.append(("render", self.next_job, desc.frames, desc.params.maxBounces,
                            desc.params.surfaceRoughness))
        return self.next_job

    def advance(self, jid, frames):
        assert jid in self.live
        self.events.append(("advance", jid, frames))

    def update_job(self, jid, desc):
        assert jid in self.live
        self.events.append(("update", jid, desc.params.maxBounces, desc.params.surfaceRoughness))

    def destroy_job(self, jid):
        self.live.discard(jid)
        self.events.append(("destroy", jid))

    def pick(self, sid, desc, x, y):
        self.events.append(("pick", x, y))
        return 2.5, 2

    def kinds(self):
        return [e[0] for e in self.events]


def snelly_for(scene):
    ctx = RecordingContext()
    return api.Snelly(scene, context=ctx), ctx


# ---------------------------------------------------------------------------------------------
# dumpScene
# ---------------------------------------------------------------------------------------------
@pytest.mark.parametrize("v,text", [
    (1.0, "1"), (0.1, "0.1"), (-7.0, "-7"), (1e-7, "1e-7"), (1e-6, "0.000001"), (1.234e-6, "0.000001234"),
    (2.5e-7, "2.5e-7"), (1e21, "1e+21"), (1.2345678901234568e20, "123456789012345680000"), (100.0, "100"),
    (0.631430584918957, "0.631430584918957"), (1.7976931348623157e308, "1.7976931348623157e+308"),
    (5e-324, "5e-324"), (0.0, "0"), (-0.0, "0"), (math.inf, "Infinity"), (-math.inf, "-Infinity"),
    (math.nan, "NaN"), (-0.5, "-0.5"), (1234.5678, "1234.5678")])
def test_js_number_to_string(v, text):
    # ECMA-262 Number::toString: shortest round-trip digits, exponent form below 1e-6 and from 1e21
    assert api.js_number(v) == text


def test_dump_scene_js_text():
    """The JavaScript dump has the reference's statements (js/snelly.js:296-407) with the values
    of the current state."""
    h = HostSnelly(scenes.SCENES["c1"]())
    h.getRenderer().exposure = 1.25
    h.getMaterials().getSurface().roughness = 0.125
    t = h.dumpScene()
    assert t.startswith("{\n    /******* copy-pasted console output on 'O', begin *******/\n")
    assert t.endswith("/******* copy-pasted console output on 'O', end *******/\n}")
    lines = [x.strip() for x in t.split("\n")]
    for want in ["let renderer  = snelly.getRenderer();", "snelly.showGUI(true);", "camera.fov = 45;",
                 "camera.aperture = -Infinity;", "camera.auto_focus = false;", "camera.up.set(0, 1, 0);",
                 "controls.target.set(0.6, 0, 0);", "renderer.renderMode = 'pt';", "renderer.dispersive = true;",
                 "renderer.maxBounces = 8;", "renderer.maxMarchSteps = 512;", "renderer.exposure = 1.25;",
                 "renderer.sunAngularSize = 3;", "renderer.skyTintUp = [1, 1, 1];",
                 "let surface = materials.loadSurface();", "surface.roughness = 0.125;",
                 "let metal = materials.loadMetal('Gold');", "metal.roughness = 0.15;",
                 "let dielectric = materials.loadDielectric('C1 Cauchy');", "dielectric.iorVal = undefined;",
                 "let volume = materials.loadVolume();", "volume.fogEnable = false;"]:
        assert want in lines, want
    # statement order follows the reference: camera, renderer, lights, materials, volume last
    order = [lines.index(x) for x in ("camera.fov = 45;", "renderer.renderMode = 'pt';", "renderer.skyPower = "
                                      "-0.3010299956639812;", "let surface = materials.loadSurface();",
                                      "let metal = materials.loadMetal('Gold');", "let volume = materials.loadVolume();")]
    assert order == sorted(order)


def test_dump_scene_lists_only_the_scene_materials():
    t = HostSnelly(scenes.SCENES["c0"]()).dumpScene()
    assert "loadSurface" in t and "loadMetal" not in t and "loadDielectric" not in t and "loadVolume" in t


def test_dump_scene_abbe_dielectric_values():
    h = HostSnelly(scenes.SCENES["c1"]())
    d = h.getMaterials().getDielectrics()
    abbe = next(n for n, x in d.items() if x.model == "abbe")
    h.getMaterials().loadDielectric(abbe)
    t = h.dumpScene()
    assert f"dielectric.iorVal = {api.js_number(d[abbe].iorVal)};" in t
    assert f"dielectric.abbe = {api.js_number(d[abbe].abbe)};" in t


def _state(h):
    return (bytes(h.uniform_params()), bytes(h.scene_opts()), h.tonemap_params(), repr(sorted(h.scene_uniforms().items())),
            h.getMaterials().getLoadedMetal().getName(), h.getMaterials().getLoadedDielectric().getName(),
            h.guiVisible)


@pytest.mark.parametrize("name", sorted(scenes.SCENES))
def test_dump_scene_python_round_trip(name):
    """dumpScene(lang='python') executed on a freshly initialised facade restores every uploaded
    value: uniform block, compile options, tonemapper settings and scene uniforms."""
    h = HostSnelly(scenes.SCENES[name]())
    r, cam, m = h.getRenderer(), h.getCamera(), h.getMaterials()
    cam.position.set(1.5, 0.25, -3.0)
    cam.fov = 33.0
    cam.aperture = 2.0
    cam.focalDistance = 0.3
    h.getControls().target.set(0.1, -0.2, 0.3)
    r.exposure, r.gamma, r.hueShift = 0.7, 2.4, 12.0
    r.maxBounces, r.maxMarchSteps, r.radianceClamp = 6, 300, 1.5
    r.skyTintUp, r.sunLatitude, r.sunLongitude = [0.9, 0.8, 0.7], 33.0, 77.0
    r.sphereLightPower, r.sphereLightPosition = 1.0, [0.5, 2.0, 0.5]
    m.loadSurface().roughness = 0.37
    m.loadSurface().diffuseAlbedo = [0.3, 0.6, 0.9]
    m.loadMetal("Copper").roughness = 0.11
    m.loadDielectric("Diamond").absorptionColor = [0.9, 0.5, 0.2]
    v = m.loadVolume()
    v.fogEnable, v.fogMFP, v.scatteringColor = True, 0.4, [0.1, 0.2, 0.3]
    h.showGUI(False)
    if isinstance(h.sceneObj, scenes.Turntable):
        h.sceneObj.pose(h, 5)  # animated scene parameters, restored by its initGenerator
    before = _state(h)
    code = h.dumpScene("python")
    fresh = HostSnelly(scenes.SCENES[name]())
    exec(code, {"snelly": fresh, "self": fresh.sceneObj})
    if "SDF_METAL(" not in h.sceneObj.shader():  # only the scene's materials are dumped
        fresh.getMaterials().loadMetal("Copper").roughness = 0.11
    if "SDF_DIELECTRIC(" not in h.sceneObj.shader():
        fresh.getMaterials().loadDielectric("Diamond").absorptionColor = [0.9, 0.5, 0.2]
    if "SDF_SURFACE(" not in h.sceneObj.shader():
        fresh.getMaterials().loadSurface().roughness = 0.37
        fresh.getMaterials().loadSurface().diffuseAlbedo = [0.3, 0.6, 0.9]
    assert _state(fresh) == before


def test_init_generator_text_is_inserted():
    sc = scenes.Turntable()
    h = HostSnelly(sc)
    sc.parameters["radius"] = 0.71
    t = h.dumpScene("python")
    assert "self.parameters['radius'] = 0.71" in t.split("\n")
    assert "self.parameters['radius'] = 0.71" in h.dumpScene("js")


def test_material_repr_matches_reference_form():
    s = api.Surface()
    assert s.repr().split("\n")[1] == "    surface.roughness = 0.1;"
    v = api.Volume()
    assert v.repr().strip().split("\n")[-1].strip() == "volume.fogEnable = false;"
    assert api.Metal("x", {"n": [0] * 64, "k": [0] * 64}).repr("python").strip().split("\n")[0] == "metal.roughness = 0.02"


# ---------------------------------------------------------------------------------------------
# render loop
# ---------------------------------------------------------------------------------------------
class Callbacks(scenes.PlainSphere):
    """C0 with counting callbacks; preframeCallback may change the surface roughness."""

    def __init__(self, change_at=None):
        super().__init__(16, 16)
        self.pre = self.post = 0
        self.change_at = change_at

    def preframeCallback(self, snelly, gl):
        self.pre += 1
        if self.change_at is not None and self.pre == self.change_at:
            snelly.getMaterials().getSurface().roughness = 0.6

    def postframeCallback(self, snelly, gl):
        self.post += 1


def test_frames_without_callbacks_go_out_as_one_call():
    s, ctx = snelly_for(scenes.PlainSphere(16, 16))
    s.render(5)
    s.render(3)
    assert ctx.kinds() == ["compile", "uniforms", "render", "advance"]
    assert ctx.events[2][2] == 5 and ctx.events[3][2] == 3
    assert s.getRenderer().getSPP() == 8 and s.getRenderer().numSamples == 8 * 16 * 16


def test_callbacks_run_once_per_frame():
    sc = Callbacks()
    s, ctx = snelly_for(sc)
    s.render(4)
    assert sc.pre == sc.post == 4
    assert ctx.kinds() == ["compile", "uniforms", "render", "advance", "advance", "advance"]
    assert s.getRenderer().getSPP() == 4


def test_parameter_change_between_frames_updates_the_live_job():
    """A preframeCallback change reaches the next frame without a reset (the reference uploads all
    uniforms every frame); the accumulation continues in the same job."""
    sc = Callbacks(change_at=3)
    s, ctx = snelly_for(sc)
    s.render(4)
    k = ctx.kinds()
    assert k == ["compile", "uniforms", "render", "advance", "uniforms", "update", "advance", "advance"]
    upd = ctx.events[k.index("update")]
    assert upd[1] == 1 and abs(upd[3] - 0.6) < 1e-7
    # a change made between render() calls is picked up the same way
    s.getRenderer().exposure = 2.0  # tonemapper only: nothing to upload
    s.getCamera().position.set(0.0, 2.0, 5.0)
    s.render(1)
    assert ctx.kinds()[-3:] == ["uniforms", "update", "advance"]


def test_max_spp_stops_accumulation():
    sc = Callbacks()
    s, ctx = snelly_for(sc)
    r = s.getRenderer()
    r.maxSpp = 5
    r.maxSamplesPerFrame = 2
    s.reset()
    s.render(10)
    # frames of 2 samples: spp 2, 4 run; the third would reach 6 > 5, so spp reads 5 and stops
    assert r.getSPP() == 5
    assert ctx.kinds().count("render") + ctx.kinds().count("advance") == 2
    # as in the reference, spp == maxSpp does not stop the preframe callback (js/renderer.js:467
    # tests spp > maxSpp), only the frame itself
    assert sc.post == 2 and sc.pre == 10
    s.render(3)
    assert ctx.kinds().count("render") + ctx.kinds().count("advance") == 2 and sc.pre == 13


def test_is_ready_gates_frames():
    class NotReady(scenes.PlainSphere):
        ready = False

        def isReady(self, snelly):
            return self.ready

    sc = NotReady(16, 16)
    s, ctx = snelly_for(sc)
    s.render(3)
    assert ctx.events == [] and s.getRenderer().getSPP() == 0
    sc.ready = True
    s.render(3)
    assert s.getRenderer().getSPP() == 3


def test_reset_without_recompile_keeps_the_compiled_bounds():
    """reset(no_recompile=True) keeps the program, so a changed maxBounces (a compile-time
    constant in the reference) only takes effect after a reset that recompiles."""
    s, ctx = snelly_for(scenes.PlainSphere(16, 16))
    s.render(1)
    s.getRenderer().maxBounces = 7
    s.getRenderer().reset(True)
    s.render(1)
    assert [e for e in ctx.events if e[0] == "compile"] == [("compile", 4)]
    assert ctx.events[-1][0] == "render" and ctx.events[-1][3] == 4
    s.reset()
    s.render(1)
    assert ("compile", 7) in ctx.events and ctx.events[-1][3] == 7
    assert ("destroy", 1) in ctx.events and ("destroy", 2) in ctx.events


def test_turntable_animation_protocol():
    got = []
    sc = scenes.Turntable(16, 16, frames=3, target_spp=2, on_frame=lambda i, s: got.append((i, s.getRenderer().getSPP())))
    s, ctx = snelly_for(sc)
    s.render(10)
    assert got == [(0, 2), (1, 2), (2, 2)]
    # one job per animation frame, each reset without a recompile
    assert ctx.kinds().count("compile") == 1 and ctx.kinds().count("render") == 3
    assert ctx.kinds().count("destroy") == 2
    # the last animation frame keeps accumulating without being handed over again
    assert s.getRenderer().getSPP() == 10 - 4


def test_auto_focus_on_reset():
    s, ctx = snelly_for(scenes.PlainSphere(16, 16))
    s.getCamera().auto_focus = True
    s.reset()
    assert ("pick", 8.0, 8.0) in ctx.events
    assert math.isclose(s.getCamera().focalDistance, math.log10(2.5 / s.lengthScale))


def test_resize_restarts_with_new_aspect():
    s, ctx = snelly_for(scenes.PlainSphere(16, 16))
    s.render(2)
    s.resize(32, 8)
    assert (s.width, s.height, s.getCamera().aspect) == (32, 8, 4.0)
    s.render(1)
    assert ctx.kinds()[-2:] == ["uniforms", "render"] and s.getRenderer().getSPP() == 1


def test_facade_accessors():
    s, _ = snelly_for(scenes.PlainSphere(16, 16))
    assert s.getVersion() == [1, 19, 0]
    assert s.getLoadedSpectrum().getName() == "flat"
    assert s.getDielectrics() is s.getMaterials().getDielectrics() and len(s.getMetals()) == 22
    s.enableGUI(False)
    assert not s.guiVisible
    s.getGUI().sync()
    assert s.getGLContext() is None and s.getUserTextureUnitStart() == 7
