"""Headless mirror of the reference's scene API (js/sceneAPI.js, js/snelly.js, js/renderer.js,
js/materials.js, js/spectra.js) over libsnelly.

A user scene is written exactly as for the reference: an object with `init(snelly)`, `shader()`
returning GLSL that defines SDF_SURFACE / SDF_METAL / SDF_DIELECTRIC and optional hooks, and
optional `syncShader(snelly, shader)`, `getLengthScale()`, `getMinLengthScale()`,
`getMaxLengthScale()`, `envMap()`, `preframeCallback`, `postframeCallback`, `isReady`.
`Snelly(scene)` then exposes the same objects (`getRenderer()`, `getCamera()`, `getControls()`,
`getMaterials()`, ...) with the same property names, defaults and unit conventions (log10 powers,
log-sqrt(2) aperture). `render(n)` renders n progressive frames on the GPU, each as one call of the
reference's Renderer.render (callbacks, maxSpp and per-frame uniform changes included).
"""
import ctypes
import json
import math
import os
import textwrap

import numpy as np

from . import _native as N

DATA = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "materials.json")))


# ---------------------------------------------------------------------------------------------
# small 3-vector helpers (THREE.Vector3 semantics where the reference uses THREE)
# ---------------------------------------------------------------------------------------------
class Vector3:
    def __init__(self, x=0.0, y=0.0, z=0.0):
        self.x, self.y, self.z = float(x), float(y), float(z)

    def set(self, x, y, z):
        self.x, self.y, self.z = float(x), float(y), float(z)
        return self

    def copy(self, v):
        return self.set(v.x, v.y, v.z)

    def clone(self):
        return Vector3(self.x, self.y, self.z)

    def tolist(self):
        return [self.x, self.y, self.z]


def _sub(a, b):
    return [a[0] - b[0], a[1] - b[1], a[2] - b[2]]


def _cross(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def _normalize(a):
    n = math.sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2])
    return [a[0] / n, a[1] / n, a[2] / n] if n > 0 else [0.0, 0.0, 0.0]


class Camera:
    """THREE.PerspectiveCamera fields the renderer reads (js/snelly.js:40-47, :244-245)."""

    def __init__(self, fov=45.0, aspect=1.0):
        self.fov = fov
        self.aspect = aspect
        self.position = Vector3(1.0, 1.0, 1.0)
        self.up = Vector3(0.0, 1.0, 0.0)
        self.aperture = -10.0      # log base sqrt(2), relative to lengthScale
        self.focalDistance = 1.0   # log base 10, relative to lengthScale
        self.auto_focus = False


class Controls:
    """The OrbitControls target the camera looks at."""

    def __init__(self):
        self.target = Vector3(0.0, 0.0, 0.0)

    def update(self):
        pass


def camera_basis(position, target, up):
    """camPos, camDir, camX, camY as uploaded by js/renderer.js:521-531.

    THREE's lookAt makes the camera's -z axis point at the target and its x axis
    normalize(cross(up, z)); the world-space up vector is then cross(z, x). camDir is the world
    direction (-z) and camX = cross(camUp, camDir).
    """
    p, t, u = position, target, up
    z = _normalize(_sub(p, t))
    if z == [0.0, 0.0, 0.0]:
        z = [0.0, 0.0, 1.0]
    x = _cross(u, z)
    if math.sqrt(sum(v * v for v in x)) == 0.0:  # up parallel to the view axis: nudge as THREE does
        z = _normalize([z[0] + 1e-4, z[1], z[2]])
        x = _cross(u, z)
    x = _normalize(x)
    y = _cross(z, x)
    cam_dir = [-z[0], -z[1], -z[2]]
    # camera.up.transformDirection(matrixWorld): the up vector expressed through the camera axes
    cam_up = _normalize([x[i] * u[0] + y[i] * u[1] + z[i] * u[2] for i in range(3)])
    cam_x = _cross(cam_up, cam_dir)
    return list(p), cam_dir, cam_x, cam_up


# ---------------------------------------------------------------------------------------------
# materials (js/materials.js)
# ---------------------------------------------------------------------------------------------
class Surface:
    """Uber surface (js/materials.js:39-83)."""

    def __init__(self):
        self.diffuseAlbedo = [1.0, 1.0, 1.0]
        self.specAlbedo = [1.0, 1.0, 1.0]
        self.roughness = 0.1
        self.ior = 1.5
        self.subsurface = 0.0
        self.subsurfaceAlbedoRGB = [0.5, 0.5, 0.5]
        self.subsurfaceMFP = 0.0
        self.subsurfaceAnisotropy = 0.0
        self.subsurfaceDiffuseWeight = 1.0

    def repr(self, lang="js"):
        return material_repr("surface", self, lang)

    def syncShader(self, p, snelly):
        p.surfaceDiffuseAlbedoRGB[:] = self.diffuseAlbedo
        p.surfaceSpecAlbedoRGB[:] = self.specAlbedo
        p.surfaceRoughness = self.roughness
        p.surfaceIor = self.ior
        p.subsurface = self.subsurface
        p.subsurfaceAlbedoRGB[:] = self.subsurfaceAlbedoRGB
        p.subsurfaceMFP = self.subsurfaceMFP
        p.subsurfaceAnisotropy = self.subsurfaceAnisotropy
        p.subsurfaceDiffuseWeight = self.subsurfaceDiffuseWeight


class Volume:
    """Homogeneous atmosphere + fog (js/materials.js:193-275)."""

    def __init__(self):
        self.atmosphereMinX, self.atmosphereMaxX = -10.0, 10.0
        self.atmosphereMinY, self.atmosphereMaxY = 0.0, 10.0
        self.atmosphereMinZ, self.atmosphereMaxZ = -10.0, 10.0
        self.lof10_mfp = 1.0
        self.scatteringColor = [0.0, 0.0, 0.0]
        self.absorptionColor = [0.0, 0.0, 0.0]
        self.anisotropy = 0.0
        self.emission = 0.0
        self.emissionColor = [1.0, 1.0, 1.0]
        self.fogEnable = False
        self.fogMFP = 0.0
        self.fogMaxOpticalDepth = 5.0
        self.fogEmission = [1.0, 1.0, 1.0]
        self.fogTint = [0.5, 0.5, 0.5]

    def repr(self, lang="js"):
        return material_repr("volume", self, lang)

    def syncShader(self, p, snelly):
        sca = list(self.scatteringColor)
        ext = [self.absorptionColor[c] + self.scatteringColor[c] for c in range(3)]
        p.atmosphereMFP = 10.0 ** self.lof10_mfp
        p.atmosphereExtinctionCoeffRGB[:] = ext
        p.atmosphereScatteringCoeffRGB[:] = sca
        p.atmosphereAnisotropy = self.anisotropy
        p.atmosphereBoundsMin[:] = [self.atmosphereMinX, self.atmosphereMinY, self.atmosphereMinZ]
        p.atmosphereBoundsMax[:] = [self.atmosphereMaxX, self.atmosphereMaxY, self.atmosphereMaxZ]
        p.volumeEmission = self.emission
        p.volumeEmissionColorRGB[:] = self.emissionColor
        p.fogEnable = 1 if self.fogEnable else 0
        p.fogMFP = 10.0 ** self.fogMFP
        p.fogMaxOpticalDepth = self.fogMaxOpticalDepth
        p.fogEmission[:] = self.fogEmission
        p.fogTint[:] = self.fogTint


class Metal:
    """Tabulated conductor (js/materials.js:479-501, 631-669)."""

    def __init__(self, name, table):
        self._name = name
        self.roughness = 0.02
        self.specAlbedo = [1.0, 1.0, 1.0]
        self.n = list(table["n"])
        self.k = list(table["k"])

    def getName(self):
        return self._name

    def repr(self, lang="js"):
        return material_repr("metal", self, lang)

    def syncShader(self, p, snelly):
        p.metalRoughness = self.roughness
        p.metalSpecAlbedoRGB[:] = self.specAlbedo
        p.metalN[:] = self.n
        p.metalK[:] = self.k


class Dielectric:
    """Dielectric with one of the reference's IOR models (js/materials.js:727-1099)."""

    def __init__(self, name, model, coeffs):
        self._name = name
        self.model = model
        self.coeffs = list(coeffs)
        self.roughness = 0.005
        self.absorptionScale = -1.0  # set from the scene's maxLengthScale on first use
        self.absorptionColor = [1.0, 1.0, 1.0]
        self.specAlbedo = [1.0, 1.0, 1.0]
        if model == "abbe":
            self.iorVal, self.abbe = coeffs[0], coeffs[1]

    def getName(self):
        return self._name

    def repr(self, lang="js"):
        return material_repr("dielectric", self, lang)

    def syncShader(self, p, snelly):
        if self.absorptionScale < 0.0:
            self.absorptionScale = snelly.maxLengthScale
        p.dieleRoughness = self.roughness
        p.dieleSpecAlbedoRGB[:] = self.specAlbedo
        s = snelly.lengthScale / max(self.absorptionScale, 1.0e-3)
        p.dieleAbsorptionRGB[:] = [s * max(0.0, 1.0 - self.absorptionColor[c]) for c in range(3)]
        p.dieleModel = N.IOR_MODELS[self.model]
        coeffs = [self.iorVal, self.abbe] if self.model == "abbe" else self.coeffs
        p.dieleNumCoeffs = len(coeffs)
        for i, c in enumerate(coeffs):
            p.dieleCoeffs[i] = c


class Materials:
    """Material registry (js/materials.js:1117-1342); defaults BK7 glass and aluminium."""

    def __init__(self):
        self.dielectrics = {n: Dielectric(n, d["model"], d["coeffs"]) for n, d in DATA["dielectrics"].items()}
        self.metals = {n: Metal(n, DATA["metal_tables"][t]) for n, t in DATA["metals"].items()}
        self.surfaceObj = Surface()
        self.volumeObj = Volume()
        self.dielectricObj = self.dielectrics["Glass (BK7)"]
        self.metalObj = self.metals["Aluminium"]

    def loadDielectric(self, name):
        self.dielectricObj = self.dielectrics[name]
        return self.dielectricObj

    def loadMetal(self, name):
        self.metalObj = self.metals[name]
        return self.metalObj

    def loadSurface(self):
        return self.surfaceObj

    def loadVolume(self):
        return self.volumeObj

    getLoadedDielectric = getDielectric = lambda self: self.dielectricObj
    getLoadedMetal = getMetal = lambda self: self.metalObj
    getSurface = loadSurface
    getVolume = loadVolume
    getDielectrics = lambda self: self.dielectrics
    getMetals = lambda self: self.metals

    def syncShader(self, p, snelly):
        self.metalObj.syncShader(p, snelly)
        self.dielectricObj.syncShader(p, snelly)
        self.surfaceObj.syncShader(p, snelly)
        self.volumeObj.syncShader(p, snelly)


# ---------------------------------------------------------------------------------------------
# spectra (js/spectra.js)
# ---------------------------------------------------------------------------------------------
class BlackbodySpectrum:
    def __init__(self, name, desc, temperature):
        self._name, self._desc, self.skyTemperature = name, desc, temperature

    def getName(self):
        return self._name

    def native(self):
        return N.Spectrum(N.SPECTRUM_BLACKBODY, self.skyTemperature, 390.0, 750.0, 550.0)


class FlatSpectrum:
    def __init__(self, name, desc, bandmin, bandmax):
        self._name, self._desc = name, desc
        self.min, self.max = bandmin, bandmax

    def getName(self):
        return self._name

    def native(self):
        return N.Spectrum(N.SPECTRUM_FLAT, 6000.0, self.min, self.max, 550.0)


class MonochromaticSpectrum:
    def __init__(self, name, desc, wavelength):
        self._name, self._desc, self.wavelength = name, desc, wavelength

    def getName(self):
        return self._name

    def native(self):
        return N.Spectrum(N.SPECTRUM_MONO, 6000.0, 390.0, 750.0, self.wavelength)


# ---------------------------------------------------------------------------------------------
# shader uniform recorder: what a scene's syncShader(snelly, shader) calls
# ---------------------------------------------------------------------------------------------
class Shader:
    """Records the uniform* calls a scene makes (js/gl.js:262-408) for snelly_set_uniforms."""

    def __init__(self):
        self.calls = {}
        self.textures = {}

    def _put(self, name, typ, vals):
        self.calls[name] = (typ, vals)

    def uniformF(self, name, v):
        self._put(name, N.U_FLOAT, [float(v)])

    def uniformI(self, name, v):
        self._put(name, N.U_INT, [int(v)])

    def uniform2F(self, name, a, b):
        self._put(name, N.U_VEC2, [float(a), float(b)])

    def uniform3F(self, name, a, b, c):
        self._put(name, N.U_VEC3, [float(a), float(b), float(c)])

    def uniform4F(self, name, a, b, c, d):
        self._put(name, N.U_VEC4, [float(a), float(b), float(c), float(d)])

    def uniform2Fv(self, name, v):
        self._put(name, N.U_VEC2, [float(x) for x in v])

    def uniform3Fv(self, name, v):
        self._put(name, N.U_VEC3, [float(x) for x in v])

    def uniform4Fv(self, name, v):
        self._put(name, N.U_VEC4, [float(x) for x in v])

    def uniform1Fv(self, name, v):
        self._put(name, N.U_FLOAT, [float(x) for x in v])

    def uniformMatrix3Fv(self, name, v):
        self._put(name, N.U_MAT3, [float(x) for x in v])

    def uniformTexture(self, name, texture, linear=True):
        """Bind a texture array to a sampler2D / sampler3D uniform: (h, w, c) or (d, h, w, c) of
        float32, float16 or uint8 (js/gl.js:262 binds a GLU.Texture the same way)."""
        self.textures[name] = (texture, linear)


# ---------------------------------------------------------------------------------------------
# renderer (js/renderer.js) and the application facade (js/snelly.js)
# ---------------------------------------------------------------------------------------------
class Renderer:
    """Renderer settings with the reference's defaults (js/renderer.js:78-126)."""

    def __init__(self, snelly):
        self._snelly = snelly
        self.width = None
        self.height = None
        self.renderMode = "pt"
        self.dispersive = False
        self.maxSamplesPerFrame = 1
        self.maxSpp = 1024
        self.maxBounces = 3
        self.maxAtmosphereScatters = 1
        self.maxMarchSteps = 256
        self.maxSSSSteps = 128
        self.radianceClamp = 3.0
        self.wavelengthSamples = 256
        self.filterRadius = 2.0
        self.goalFPS = 20.0
        self.minsSPPToRedraw = 0.0
        self.shadowStrength = 1.0
        self.maxStepsIsMiss = True
        self.interactive = True
        self.skyPower = 0.0
        self.skyTemperature = 6000.0
        self.skyTintUp = [1.0, 1.0, 1.0]
        self.skyTintDown = [1.0, 1.0, 1.0]
        self.envMapVisible = True
        self.envMapPhiRotation = 0.0
        self.envMapThetaRotation = 0.0
        self.envMapTransitionAngle = 135.0
        self.sunPower = -7.0
        self.sunAngularSize = 5.0
        self.sunColor = [1.0, 1.0, 1.0]
        self.sunLatitude = 50.0
        self.sunLongitude = 0.0  # the reference misspells the default (sunLongitudef, :113)
        self.sunVisibleDirectly = True
        self.sphereLightRadius = 1.0
        self.sphereLightPower = -7.0
        self.sphereLightColor = [1.0, 1.0, 1.0]
        self.sphereLightPosition = [0.0, 0.0, 0.0]
        self.exposure = 0.0
        self.gamma = 2.2
        self.contrast = 1.0
        self.saturation = 1.0
        self.hueShift = 0.0
        self.skipProbability = 0.0
        self.spp = 0.0
        self.numSamples = 0.0
        # B200 build options (no reference counterpart)
        self.mathMode = N.MATH_FAST
        self.kernelMode = N.KERNEL_AUTO  # autotuned per scene module and image size

    def sun_dir(self):
        """updateSunDir, js/renderer.js:371-383."""
        lat = (90.0 - self.sunLatitude) * math.pi / 180.0
        lon = self.sunLongitude * math.pi / 180.0
        return [math.sin(lat) * math.cos(lon), math.cos(lat), math.sin(lat) * math.sin(lon)]

    def getSPP(self):
        return self.spp

    def reset(self, no_recompile=False):
        """Restart accumulating samples (Renderer.prototype.reset, js/renderer.js:191-201); with
        no_recompile the compiled program, and its compile-time settings, stay."""
        self._snelly.reset(no_recompile)

    def pick(self, xPick, yPick):
        """First-hit distance and material along the camera ray through pixel coordinate
        (xPick, yPick) of the frame (Renderer.prototype.pick, js/renderer.js:398-461)."""
        return self._snelly.pick(xPick, yPick)

    def resize(self, width, height):
        self._snelly.resize(width, height)

    def focusAt(self, x, y):
        """Set the camera's focal distance to the first hit under the frame fraction (x, y)
        (Renderer.prototype.focusAt, js/renderer.js:391-396, whose body reads undefined names and
        never sets the focal distance; this does what its documentation states)."""
        s = self._snelly
        hit = self.pick(x * s.width, y * s.height)
        if hit["material"] >= 0:
            s.camera.focalDistance = math.log10(max(hit["distance"], 1.0e-30) / max(s.lengthScale, 1.0e-30))
        return hit


class HeadlessGUI:
    """Stands in for the dat.GUI wrapper (js/gui.js) a scene may call: there are no widgets."""

    closed = True

    def sync(self):
        pass

    def addParameter(self, *a, **k):
        return self

    def addFolder(self, *a, **k):
        return self

    def onChange(self, *a, **k):
        return self


def js_number(v):
    """A number as JavaScript's String(v) writes it (ECMA-262 Number::toString): the shortest
    digits that round-trip, integers without a fraction, exponent form below 1e-6 and from 1e21."""
    v = float(v)
    if v != v:
        return "NaN"
    if v in (math.inf, -math.inf):
        return "Infinity" if v > 0 else "-Infinity"
    if v == 0.0:
        return "0"
    sign = "-" if v < 0 else ""
    m, _, e = repr(abs(v)).partition("e")
    ip, _, fp = m.partition(".")
    digits = (ip + fp).lstrip("0")
    n = len(ip.lstrip("0")) if ip.strip("0") else -(len(fp) - len(fp.lstrip("0")))
    n += int(e) if e else 0
    digits = digits.rstrip("0") or "0"
    k = len(digits)
    if k <= n <= 21:
        out = digits + "0" * (n - k)
    elif 0 < n <= 21:
        out = digits[:n] + "." + digits[n:]
    elif -6 < n <= 0:
        out = "0." + "0" * (-n) + digits
    else:
        out = digits[0] + ("." + digits[1:] if k > 1 else "") + "e" + ("+" if n - 1 >= 0 else "-") + str(abs(n - 1))
    return sign + out


def _fmt(v, lang):
    if v is None:
        return "undefined" if lang == "js" else "None"
    if isinstance(v, bool):
        return ("true" if v else "false") if lang == "js" else repr(v)
    if isinstance(v, str):
        return "'" + v + "'"
    if isinstance(v, (list, tuple)):
        return "[" + ", ".join(_fmt(x, lang) for x in v) + "]"
    if lang == "js":
        return js_number(v)
    if isinstance(v, float) and not math.isfinite(v):
        return f"float('{v!r}')"
    return repr(float(v)) if isinstance(v, float) else repr(v)


_DUMP_RENDERER = [
    ("General rendering settings", ["renderMode", "dispersive", "maxSamplesPerFrame", "maxSpp", "maxBounces",
                                    "maxAtmosphereScatters", "maxMarchSteps", "maxStepsIsMiss", "interactive",
                                    "goalFPS", "minsSPPToRedraw", "filterRadius", "radianceClamp",
                                    "wavelengthSamples", "shadowStrength"]),
    ("Tone-mapping", ["exposure", "gamma", "contrast", "saturation", "hueShift"]),
]
_DUMP_LIGHTS = [
    ("sky light", ["skyPower", "skyTintUp", "skyTintDown", "envMapVisible", "envMapPhiRotation",
                   "envMapThetaRotation", "envMapTransitionAngle"]),
    ("sun light", ["sunPower", "sunColor", "sunAngularSize", "sunLatitude", "sunLongitude", "sunVisibleDirectly"]),
    ("sphere light", ["sphereLightPosition", "sphereLightRadius", "sphereLightPower", "sphereLightColor"]),
]
_REPR = {
    "surface": ["roughness", "ior", "diffuseAlbedo", "specAlbedo", "subsurface", "subsurfaceAlbedoRGB",
                "subsurfaceMFP", "subsurfaceAnisotropy", "subsurfaceDiffuseWeight"],
    "metal": ["roughness", "specAlbedo"],
    "dielectric": ["absorptionColor", "absorptionScale", "roughness", "iorVal", "abbe"],
    "volume": ["atmosphereMinX", "atmosphereMinY", "atmosphereMinZ", "atmosphereMaxX", "atmosphereMaxY",
               "atmosphereMaxZ", "lof10_mfp", "scatteringColor", "absorptionColor", "emission", "emissionColor",
               "fogEmission", "fogTint", "fogMFP", "fogMaxOpticalDepth", "fogEnable"],
}


def material_repr(var, obj, lang="js"):
    """Material.repr (js/materials.js:56-70 Surface, 222-243 Volume, 488-495 Metal, 740-750
    Dielectric): one assignment per property. A property the material lacks (iorVal and abbe of a
    non-Abbe dielectric) reads `undefined` in JavaScript and is left out in Python."""
    end = ";" if lang == "js" else ""
    lines = []
    for f in _REPR[var]:
        v = getattr(obj, f, None)
        if v is None and lang != "js":
            continue
        note = " // mfp in multiples of scene scale" if (lang == "js" and f == "absorptionScale") else ""
        lines.append(f"    {var}.{f} = {_fmt(v, lang)}{end}{note}")
    return "\n" + "\n".join(lines) + "\n    "


def dump_scene(snelly, lang="js"):
    """Snelly.dumpScene (js/snelly.js:296-407) for lang "js" or "python"."""
    if lang not in ("js", "python"):
        raise ValueError("lang must be 'js' or 'python'")
    js = lang == "js"
    end = ";" if js else ""
    com = "//" if js else "#"
    let = "let " if js else ""
    cam, ctl, r, mats = snelly.camera, snelly.camControls, snelly.pathtracer, snelly.materials
    sc = snelly.sceneObj
    out = []
    out.append("{\n    /******* copy-pasted console output on 'O', begin *******/\n" if js
               else "# ------- copy-pasted output of dumpScene, begin -------\n")
    out.append(f"""
    {let}renderer  = snelly.getRenderer(){end}
    {let}camera    = snelly.getCamera(){end}
    {let}controls  = snelly.getControls(){end}
    {let}materials = snelly.getMaterials(){end}
    """)
    if hasattr(sc, "initGenerator"):
        out.append(_Verbatim(sc.initGenerator()))
    out.append(f"\nsnelly.showGUI({_fmt(bool(snelly.guiVisible), lang)}){end}\n")
    out.append(f"\n    {'/**' if js else '#'} Camera settings {'**/' if js else ''}\n")
    for f in ("fov", "aperture", "focalDistance", "auto_focus"):
        v = getattr(cam, f)
        out.append(f"    camera.{f} = {_fmt(v if isinstance(v, bool) else float(v), lang)}{end}\n")
    for name, vec in (("camera.up", cam.up), ("camera.position", cam.position), ("controls.target", ctl.target)):
        out.append(f"    {name}.set({_fmt(vec.x, lang)}, {_fmt(vec.y, lang)}, {_fmt(vec.z, lang)}){end}\n")
    out.append(f"\n    {'/**' if js else '#'} Renderer settings {'**/' if js else ''}\n")
    for title, fields in _DUMP_RENDERER:
        out.append(f"    {com} {title}\n")
        for f in fields:
            out.append(f"    renderer.{f} = {_fmt(getattr(r, f), lang)}{end}\n")
    out.append(f"    {com} Lights\n")
    for title, fields in _DUMP_LIGHTS:
        out.append(f"        {com} {title}\n")
        for f in fields:
            out.append(f"        renderer.{f} = {_fmt(getattr(r, f), lang)}{end}\n")
    out.append(f"\n    {'/**' if js else '#'} Material settings {'**/' if js else ''}")
    shader = sc.shader()
    if "SDF_SURFACE(" in shader:
        out.append(f"\n    {let}surface = materials.loadSurface(){end}")
        out.append(material_repr("surface", mats.loadSurface(), lang))
    if "SDF_METAL(" in shader:
        name = mats.getLoadedMetal().getName()
        out.append(f"\n    {let}metal = materials.loadMetal('{name}'){end}")
        out.append(material_repr("metal", mats.loadMetal(name), lang))
    if "SDF_DIELECTRIC(" in shader:
        name = mats.getLoadedDielectric().getName()
        out.append(f"\n    {let}dielectric = materials.loadDielectric('{name}'){end}")
        out.append(material_repr("dielectric", mats.loadDielectric(name), lang))
    out.append(f"\n    {let}volume = materials.loadVolume(){end}")
    out.append(material_repr("volume", mats.loadVolume(), lang))
    out.append("\n    /******* copy-pasted console output on 'O', end *******/\n}" if js
               else "\n# ------- copy-pasted output of dumpScene, end -------\n")
    if js:
        return "".join(out)
    # Python statements start at column 0; the scene's own text keeps its relative indentation
    return "".join(textwrap.dedent(c) if isinstance(c, _Verbatim) else "\n".join(x.strip() for x in c.split("\n"))
                   for c in out)


class _Verbatim(str):
    """Text a scene supplies (initGenerator), inserted into a dump as it is."""


class Snelly:
    """The application facade of js/snelly.js, headless: one GPU context and one scene."""

    LAMBDA_MIN, LAMBDA_MAX, SPECTRUM_SAMPLES = 390.0, 750.0, 1024

    def __init__(self, scene, width=256, height=256, device=0, hbm_budget=0, context=None):
        self._setup(scene, width, height, context if context is not None else Context(device, hbm_budget))
        self.initScene()

    def _setup(self, scene, width, height, ctx):
        """The facade's objects with their defaults (js/snelly.js:33-105), before initScene."""
        self.sceneObj = scene
        self.width, self.height = width, height
        self.camera = Camera(45.0, width / height)
        self.camControls = Controls()
        self.materials = Materials()
        self.pathtracer = Renderer(self)
        self.spectra = {}
        self.spectrumObj = None
        self._ctx = ctx
        self._scene_id = None
        self._scene_key = None
        self._need_compile = True
        self._compiled_bounces = None
        self._job = None
        self._job_key = None
        self._ready = False  # initScene has finished (Snelly.initialized, js/snelly.js:497-499)
        self.guiVisible = True
        self.guiEnabled = True
        self.statusText = ""
        self.gui = HeadlessGUI()
        self.seed = 1
        self.fp64 = False  # also accumulate in FP64 (precision study)

    # js/snelly.js:209-291
    def initScene(self):
        sc = self.sceneObj
        self.lengthScale = sc.getLengthScale() if hasattr(sc, "getLengthScale") else 1.0
        self.minLengthScale = sc.getMinLengthScale() if hasattr(sc, "getMinLengthScale") else 1.0e-4
        self.minLengthScale = max(1.0e-12, self.minLengthScale)
        self.maxLengthScale = sc.getMaxLengthScale() if hasattr(sc, "getMaxLengthScale") else 1.0e2
        self.maxLengthScale = min(1.0e9, self.maxLengthScale)
        po = 2.0 * self.lengthScale
        self.camera.position.set(po, po, po)
        self.camControls.target.set(0.0, 0.0, 0.0)
        self.camera.aperture = -10.0
        self.camera.focalDistance = 1.0
        if hasattr(sc, "init"):
            sc.init(self)
        r = self.pathtracer
        if r.width is not None and r.height is not None:
            self.width, self.height = int(r.width), int(r.height)
        self.camera.aspect = self.width / self.height  # Snelly._resize
        self.addSpectrum(BlackbodySpectrum("blackbody", "Blackbody spectrum", r.skyTemperature))
        self.loadSpectrum("blackbody")
        self._env = self._load_env_map()
        # What a user does after the scene is set up (the reference's GUI or console: another
        # spectrum, other settings); the reference has no such hook, initScene ends here.
        if hasattr(sc, "after_init"):
            sc.after_init(self)
        self._ready = True
        self.reset()

    def _load_env_map(self):
        """The scene's environment map (Scene.envMap, js/renderer.js:143-157): a PNG file path (the
        reference loads a URL) or an (h, w, 3|4) uint8 sRGB array, row 0 the top row of the image;
        None without one."""
        sc = self.sceneObj
        if not hasattr(sc, "envMap"):
            return None
        src = sc.envMap()
        if src is None:
            return None
        if isinstance(src, (str, bytes, os.PathLike)):
            from .image import read_png
            src = read_png(src)
        a = np.asarray(src, np.uint8)
        if a.ndim == 2:
            a = a[..., None]
        if a.shape[2] == 1:
            a = np.repeat(a, 3, axis=2)
        return np.ascontiguousarray(a[..., :3])

    def env_map(self):
        return getattr(self, "_env", None)

    # accessors of the reference's facade
    def getRenderer(self):
        return self.pathtracer

    def getCamera(self):
        return self.camera

    def getControls(self):
        return self.camControls

    def getMaterials(self):
        return self.materials

    def getSurface(self):
        return self.materials.loadSurface()

    def getVolume(self):
        return self.materials.loadVolume()

    def getLoadedDielectric(self):
        return self.materials.getLoadedDielectric()

    def getLoadedMetal(self):
        return self.materials.getLoadedMetal()

    def loadDielectric(self, name):
        self.materials.loadDielectric(name)
        self.reset()

    def loadMetal(self, name):
        self.materials.loadMetal(name)
        self.reset()

    def getSpectra(self):
        return self.spectra

    def addSpectrum(self, s):
        self.spectra[s.getName()] = s

    def loadSpectrum(self, name):
        """js/snelly.js:420-427: the emission spectrum the wavelengths are drawn from; resets
        without a recompile."""
        self.spectrumObj = self.spectra[name]
        self.reset(True)

    def getLoadedSpectrum(self):
        return self.spectrumObj

    def getDielectrics(self):
        return self.materials.getDielectrics()

    def getMetals(self):
        return self.materials.getMetals()

    def getScene(self):
        return self.sceneObj

    def getVersion(self):
        """The reference version whose scene API this mirrors (js/snelly.js:107-110)."""
        return [1, 19, 0]

    def getGUI(self):
        return self.gui

    def getGLContext(self):
        return None  # headless: there is no WebGL context

    def getUserTextureUnitStart(self):
        """js/snelly.js:660-663. Scene textures are bound by sampler name here, so the unit is
        informational only."""
        return 7

    def showGUI(self, show):
        self.guiVisible = bool(show)

    def enableGUI(self, enable):
        self.guiEnabled = bool(enable)
        if not enable:
            self.showGUI(False)

    def setStatus(self, statusText):
        self.statusText = statusText

    def resize(self, width, height):
        """Snelly._resize (js/snelly.js:588-608) with an explicit size: a headless renderer has no
        window to follow. The camera aspect follows and the accumulation restarts."""
        self.width, self.height = int(width), int(height)
        self.pathtracer.width, self.pathtracer.height = self.width, self.height
        self.camera.aspect = self.width / self.height
        self.reset(True)

    def auto_focus(self):
        """Snelly.auto_focus (js/snelly.js:707-722): focal distance from the first hit under the
        image centre."""
        hit = self.pick(0.5 * self.width, 0.5 * self.height)
        fd = max(1.0e-6, abs(hit["distance"]))
        self.camera.focalDistance = math.log10(fd / self.lengthScale)
        self.gui.sync()

    def dumpScene(self, lang="js"):
        """The code that re-creates the current scene, camera, renderer and material settings
        (Snelly.dumpScene, js/snelly.js:296-407; the reference prints it on key 'O' for pasting
        into a scene's init). lang="js" gives the reference's JavaScript text, statement for
        statement; lang="python" the same statements for a scene written against this module
        (exec it with `snelly` and the scene as `self` in scope). The scene's own initGenerator()
        text is inserted as it is."""
        return dump_scene(self, lang)

    # -- compile + uniforms ---------------------------------------------------------------------
    def scene_opts(self):
        r = self.pathtracer
        v = self.materials.volumeObj
        has_atm = any(c > 0.0 for c in v.scatteringColor) or any(c > 0.0 for c in v.absorptionColor)
        return N.SceneOpts(int(round(r.maxBounces)), int(round(r.maxMarchSteps)), int(round(r.maxAtmosphereScatters)),
                           int(round(r.maxSamplesPerFrame)), 1 if r.dispersive else 0, 1 if r.interactive else 0,
                           1 if has_atm else 0, 1 if v.fogEnable else 0, 1 if r.sphereLightPower > -7.0 else 0,
                           int(r.mathMode), int(r.kernelMode))

    def compileShaders(self):
        """Renderer.compileShaders (js/renderer.js:217-359): one NVRTC module per source+options."""
        glsl = self.sceneObj.shader()
        opts = self.scene_opts()
        key = (glsl, bytes(opts))
        if key != self._scene_key:
            self._scene_id = self._ctx.scene_for(glsl, opts)
            self._scene_key = key
        self._compiled_bounces = opts.max_bounces
        self._need_compile = False
        return self._scene_id

    def uniform_params(self):
        """The uniform block js/renderer.js:520-584 + material syncShader uploads, as SnellyParams."""
        r, cam = self.pathtracer, self.camera
        p = N.SnellyParams()
        p.resolution[:] = [float(self.width), float(self.height)]
        pos, cdir, cx, cy = camera_basis(cam.position.tolist(), self.camControls.target.tolist(), cam.up.tolist())
        p.camPos[:], p.camDir[:], p.camX[:], p.camY[:] = pos, cdir, cx, cy
        p.camFovy = cam.fov
        p.camAspect = cam.aspect
        p.camAperture = 0.0 if cam.aperture == -math.inf else self.lengthScale * 1.4142135 ** cam.aperture
        p.camFocalDistance = self.lengthScale * 10.0 ** cam.focalDistance
        p.filterRadius = r.filterRadius
        p.radianceClamp = 10.0 ** r.radianceClamp
        p.skipProbability = r.skipProbability
        p.lengthScale = max(self.lengthScale, 1.0e-6)
        p.maxLengthScale = max(self.maxLengthScale, 1.0e-6)
        p.minLengthScale = max(self.minLengthScale, 1.0e-6)
        p.shadowStrength = r.shadowStrength
        p.maxSSSSteps = int(r.maxSSSSteps)
        jb = getattr(r, "jobMaxBounces", None)  # per-job limit below the module's bound
        if not jb:  # MAX_BOUNCES is a compile-time constant of the program that runs
            jb = self._compiled_bounces if self._compiled_bounces is not None else r.maxBounces
        p.maxBounces = int(round(jb))
        p.maxStepsIsMiss = 1 if r.maxStepsIsMiss else 0
        p.wavelengthSamples = int(r.wavelengthSamples)
        p.skyPower = 10.0 ** r.skyPower
        p.skyTintUp[:] = r.skyTintUp
        p.skyTintDown[:] = r.skyTintDown
        p.envMapVisible = 1 if r.envMapVisible else 0
        p.envMapPhiRotation = min(max(r.envMapPhiRotation, 0.0), 360.0)
        p.envMapThetaRotation = min(max(r.envMapThetaRotation, 0.0), 180.0)
        p.envMapTransitionAngle = min(max(r.envMapTransitionAngle, 0.0), 180.0)
        p.sunPower = 10.0 ** r.sunPower
        p.sunAngularSize = r.sunAngularSize
        p.sunLatitude = r.sunLatitude
        p.sunLongitude = r.sunLongitude
        p.sunColor[:] = r.sunColor
        p.sunDir[:] = r.sun_dir()
        p.sunVisibleDirectly = 1 if r.sunVisibleDirectly else 0
        p.sphereLightPosition[:] = [x * self.lengthScale for x in r.sphereLightPosition]
        p.sphereLightRadius = r.sphereLightRadius * self.lengthScale
        p.sphereLightPower = 10.0 ** r.sphereLightPower / (4.0 * math.pi * r.sphereLightRadius ** 2)
        p.sphereLightColor[:] = r.sphereLightColor
        self.materials.syncShader(p, self)
        return p

    def scene_shader(self):
        """The scene's syncShader calls, recorded (uniforms and textures)."""
        sh = Shader()
        if hasattr(self.sceneObj, "syncShader"):
            self.sceneObj.syncShader(self, sh)
        return sh

    def scene_uniforms(self):
        return self.scene_shader().calls

    def sync_scene(self, sid):
        """Upload the scene's uniforms and textures (Scene.syncShader, js/renderer.js:604-608)."""
        sh = self.scene_shader()
        self._ctx.set_uniforms(sid, sh.calls)
        for name, (tex, linear) in sh.textures.items():
            self._ctx.set_texture(sid, name, tex, linear)

    def render_desc(self, frames):
        d = N.RenderDesc()
        d.width, d.height = int(self.width), int(self.height)
        d.frames = int(frames)
        d.mode = {"pt": N.MODE_PT, "normals": N.MODE_NORMALS, "ao": N.MODE_AO, "pick": N.MODE_PICK,
                  "ptsimple": N.MODE_PTSIMPLE}.get(self.pathtracer.renderMode, N.MODE_PT)
        d.seed = int(self.seed)
        d.params = self.uniform_params()
        d.spectrum = self.spectrumObj.native()
        d.accum_fp64 = 1 if getattr(self, "fp64", False) else 0
        env = self.env_map()
        if env is not None:
            d.env_map = env.ctypes.data
            d.env_h, d.env_w = int(env.shape[0]), int(env.shape[1])
        return d

    # -- progressive rendering ---------------------------------------------------------------------
    def reset(self, no_recompile=False):
        """Snelly.reset / Renderer.reset (js/snelly.js:497-504, js/renderer.js:191-201): drop the
        accumulated samples; without no_recompile the next frame compiles the program again from
        the current settings (a cached module when they are unchanged). With camera.auto_focus the
        focal distance is first set from the first hit under the image centre."""
        if self._job is not None:
            self._ctx.destroy_job(self._job)
            self._job = None
        if not no_recompile:
            self._need_compile = True
        if self.camera.auto_focus and self._ready:
            self.auto_focus()
        r = self.pathtracer
        r.numSamples = 0.0
        r.spp = 0.0

    def _scene(self):
        """The compiled scene the next frame runs: compiled again only after a reset without
        no_recompile (Renderer.reset, js/renderer.js:199)."""
        if self._scene_id is None or self._need_compile:
            self.compileShaders()
            self._need_compile = False
        return self._scene_id

    def _frame_state(self):
        """Everything Renderer.render uploads before a frame (js/renderer.js:520-611): the uniform
        block, the spectrum, and the scene's recorded uniforms and textures. Compiles first when
        a reset asked for it, since the program's compile-time bounds enter the uniform block."""
        self._scene()
        desc = self.render_desc(0)
        sh = self.scene_shader()
        key = (bytes(desc.params), bytes(desc.spectrum), repr(sorted(sh.calls.items())),
               tuple((n, id(t), lin) for n, (t, lin) in sorted(sh.textures.items())))
        return desc, sh, key

    def _enqueue(self, frames, state):
        """Run `frames` frames with the given frame state: a new job, or the live job after its
        parameters are brought up to date when they changed since its last frame."""
        desc, sh, key = state
        sid = self._scene()
        if self._job is None:
            self._upload_scene(sid, sh)
            desc.frames = int(frames)
            self._job = self._ctx.render(sid, desc)
            self._job_key = key
            return
        if key != self._job_key:
            self._upload_scene(sid, sh)
            self._ctx.update_job(self._job, desc)
            self._job_key = key
        if frames:
            self._ctx.advance(self._job, frames)

    def _upload_scene(self, sid, sh):
        self._ctx.set_uniforms(sid, sh.calls)
        for name, (tex, linear) in sh.textures.items():
            self._ctx.set_texture(sid, name, tex, linear)

    def render(self, frames=1):
        """Renderer.render (js/renderer.js:462-673), called `frames` times: each frame runs the
        scene's preframeCallback, stops once the sample count would pass maxSpp, picks up every
        change of camera, renderer, material or scene uniforms made since the previous frame (the
        accumulated samples stay, as in the reference, until a reset), and runs postframeCallback.
        Frames without callbacks in between go to the GPU as one call. render(0) only compiles,
        allocates and seeds the job."""
        sc, r = self.sceneObj, self.pathtracer
        if hasattr(sc, "isReady") and not sc.isReady(self):  # Snelly.render, js/snelly.js:514-521
            return
        if frames <= 0:
            self._enqueue(0, self._frame_state())
            return
        pre, post = hasattr(sc, "preframeCallback"), hasattr(sc, "postframeCallback")
        if not (pre or post):
            n = 0
            for _ in range(frames):
                if not self._count_frame():
                    break
                n += 1
            if n:
                self._enqueue(n, self._frame_state())
            return
        for _ in range(frames):
            if r.spp > r.maxSpp or (hasattr(sc, "isReady") and not sc.isReady(self)):
                return
            if pre:
                sc.preframeCallback(self, None)
            if not self._count_frame():
                continue
            self._enqueue(1, self._frame_state())
            if post:
                sc.postframeCallback(self, None)

    def _count_frame(self):
        """The sample bookkeeping of Renderer.render (js/renderer.js:467, 480-493): False when
        this frame would take the mean sample count past maxSpp (which then reads maxSpp)."""
        r = self.pathtracer
        if r.spp > r.maxSpp:
            return False
        npix = self.width * self.height
        spf = round(r.maxSamplesPerFrame)
        r.numSamples += ((1.0 - r.skipProbability) if r.interactive else 1.0) * spf * npix
        r.spp = r.numSamples / npix
        if r.spp > r.maxSpp:
            r.spp = r.maxSpp
            return False
        return True

    def pick(self, xPick, yPick):
        """Renderer.pick: {"distance", "material"} of the first hit along the pinhole ray through
        pixel coordinate (xPick, yPick) (gl_FragCoord units; a miss gives maxLengthScale and -1)."""
        sid = self._scene()
        self.sync_scene(sid)
        d, m = self._ctx.pick(sid, self.render_desc(1), xPick, yPick)
        return {"distance": d, "material": m}

    def readback(self, out=None, wait=True):
        """(H, W, 4) float32 array: mean X, Y, Z and sample count; row 0 is the bottom row.
        wait=False only enqueues the copy into `out` behind the frames rendered so far, so that it
        overlaps the next frames; `out` holds the image once the context's sync() returns."""
        return self._ctx.readback(self._job, self.width, self.height, out=out, wait=wait)

    def tonemap_params(self):
        """The tonemapper's uniforms as Renderer.render uploads them (js/renderer.js:623-630)."""
        r = self.pathtracer
        return (r.exposure, 1.0 / r.gamma, r.contrast, r.saturation, r.hueShift)

    def tonemap(self, fmt=N.TONEMAP_RGBA8):
        """The displayed image: the mean radiance through the reference's tonemapper with the
        renderer's exposure, gamma, contrast, saturation and hue shift. (H, W, 4), row 0 bottom."""
        return self._ctx.tonemap(self._job, self.width, self.height, self.tonemap_params(), fmt)

    def screenshot(self, path):
        """Write the displayed image to a PNG file (top row first)."""
        from .image import write_png
        write_png(path, self.tonemap()[::-1])

    def job_id(self):
        return self._job

    def readback_state(self):
        """(rng (n,4) uint32, Kahan sums (n,4), compensations (n,4), FP64 sums (n,4) or None)."""
        return self._ctx.readback_state(self._job, self.width, self.height, fp64=getattr(self, "fp64", False))


# ---------------------------------------------------------------------------------------------
# thin object wrapper of the C ABI
# ---------------------------------------------------------------------------------------------
class Context:
    """One libsnelly context (device, stream, module cache, jobs)."""

    def __init__(self, device=0, hbm_budget=0):
        self._lib = N.lib()
        h = ctypes.c_void_p()
        N.check(self._lib.snelly_init(ctypes.byref(h), int(device), int(hbm_budget)))
        self._h = h
        self._scene_cache = {}  # (scene GLSL, options) -> scene id, shared by Snelly objects
        self._bound = {}        # (scene id, sampler name) -> the array object uploaded last

    def scene_for(self, glsl, opts):
        """The scene id for a scene source and options, created on first use (one module and one
        set of scene textures however many jobs render it)."""
        key = (glsl, bytes(opts))
        if key not in self._scene_cache:
            self._scene_cache[key] = self.create_scene(glsl, opts)
        return self._scene_cache[key]

    def close(self):
        if self._h:
            self._lib.snelly_shutdown(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def create_scene(self, glsl, opts):
        sid = ctypes.c_uint64()
        log = ctypes.create_string_buffer(1 << 16)
        N.check(self._lib.snelly_create_scene(self._h, glsl.encode(), ctypes.byref(opts), ctypes.byref(sid), log,
                                              len(log)))
        return sid.value

    def destroy_scene(self, sid):
        N.check(self._lib.snelly_destroy_scene(self._h, sid))
        self._scene_cache = {k: v for k, v in self._scene_cache.items() if v != sid}
        self._bound = {k: v for k, v in self._bound.items() if k[0] != sid}

    def set_uniforms(self, sid, calls):
        if not calls:
            return
        arr = (N.Uniform * len(calls))()
        keep = []
        for k, (name, (typ, vals)) in enumerate(calls.items()):
            comps = {N.U_FLOAT: 1, N.U_INT: 1, N.U_BOOL: 1, N.U_VEC2: 2, N.U_VEC3: 3, N.U_VEC4: 4, N.U_MAT3: 9}[typ]
            count = max(1, len(vals) // comps)
            arr[k].name = name.encode()
            arr[k].type = typ
            arr[k].count = count
            if typ in (N.U_INT, N.U_BOOL):
                buf = (ctypes.c_int * len(vals))(*vals)
                arr[k].i = buf
            else:
                buf = (ctypes.c_float * len(vals))(*vals)
                arr[k].f = buf
            keep.append(buf)
        N.check(self._lib.snelly_set_uniforms(self._h, sid, arr, len(calls)))

    def set_texture(self, sid, name, array, linear=True):
        if self._bound.get((sid, name)) is array:
            return  # this very array is bound already
        self._bound[(sid, name)] = array
        a = np.ascontiguousarray(array)
        fmt = {np.dtype(np.float32): 0, np.dtype(np.float16): 1, np.dtype(np.uint8): 2}[a.dtype]
        if a.ndim == 3:  # (h, w, c) 2-D texture
            h, w, c = a.shape
            d = 1
        else:            # (d, h, w, c) 3-D texture
            d, h, w, c = a.shape
        N.check(self._lib.snelly_set_texture(self._h, sid, name.encode(), a.ctypes.data, w, h, d, c, fmt,
                                             1 if linear else 0))

    def render(self, sid, desc):
        jid = ctypes.c_uint64()
        N.check(self._lib.snelly_render(self._h, sid, ctypes.byref(desc), ctypes.byref(jid)))
        return jid.value

    def restore(self, sid, desc, rng, acc, comp):
        jid = ctypes.c_uint64()
        rng, acc, comp = (np.ascontiguousarray(x) for x in (rng, acc, comp))
        N.check(self._lib.snelly_restore(self._h, sid, ctypes.byref(desc), rng.ctypes.data, acc.ctypes.data,
                                         comp.ctypes.data, ctypes.byref(jid)))
        return jid.value

    def advance(self, jid, frames):
        N.check(self._lib.snelly_advance(self._h, jid, int(frames)))

    def update_job(self, jid, desc):
        """New parameters and scene uniforms for the job's next frames; samples are kept."""
        N.check(self._lib.snelly_update_job(self._h, jid, ctypes.byref(desc)))

    def advance_batch(self, jobs_frames):
        """Enqueue frames on many jobs in batched launches: {job id: frames}."""
        ids = (ctypes.c_uint64 * len(jobs_frames))(*jobs_frames.keys())
        fr = (ctypes.c_int * len(jobs_frames))(*jobs_frames.values())
        N.check(self._lib.snelly_advance_batch(self._h, ids, fr, len(jobs_frames)))

    def job_kernel(self, jid):
        """The integrator the job runs: N.KERNEL_MEGA or N.KERNEL_WAVEFRONT."""
        k = ctypes.c_int()
        N.check(self._lib.snelly_job_kernel(self._h, jid, ctypes.byref(k)))
        return k.value

    def job_wavefront_config(self, jid):
        """A wavefront job's launch configuration as a dict (pixel ranges, per-material shade
        launches, drain steps, refill chunk, claim size, refill threshold, block size, parking
        threshold, persistent walker, rays per extend lane, overlapping frames, shade grid share,
        interleaved pixel ranges, the heterogeneous medium's own scatter stage)."""
        out = (ctypes.c_int * len(N.WF_CONFIG_NAMES))()
        N.check(self._lib.snelly_job_wavefront_config(self._h, jid, out))
        return dict(zip(N.WF_CONFIG_NAMES, out))

    def tonemap(self, jid, width, height, params, fmt=N.TONEMAP_RGBA8):
        """The job's mean image through the display transform: (H, W, 4) uint8 (RGBA8) or float32
        (RGBA32F); row 0 is the bottom row. params: (exposure, invGamma, contrast, saturation,
        hueShift) as the tonemapper shader receives them."""
        tp = N.TonemapParams(*[float(v) for v in params])
        out = np.empty((height, width, 4), np.uint8 if fmt == N.TONEMAP_RGBA8 else np.float32)
        N.check(self._lib.snelly_tonemap(self._h, jid, ctypes.byref(tp), out.ctypes.data, out.nbytes, int(fmt)))
        return out

    def selftest(self, which):
        """Mismatch count of a device self-test (0: the RNG's conversions and quotients)."""
        n = ctypes.c_uint64()
        N.check(self._lib.snelly_selftest(self._h, int(which), ctypes.byref(n)))
        return n.value

    def pick(self, sid, desc, x, y):
        d, m = ctypes.c_float(), ctypes.c_float()
        N.check(self._lib.snelly_pick(self._h, sid, ctypes.byref(desc), float(x), float(y), ctypes.byref(d),
                                      ctypes.byref(m)))
        return d.value, m.value

    def readback(self, jid, width, height, out=None, poll=False, wait=True):
        """Mean XYZ and count per pixel. wait=False enqueues the copy behind the job's frames and
        returns at once (SNELLY_READ_ASYNC): `out` (page-locked for an overlapped copy) is filled
        once sync() returns, or a later waiting readback of the job."""
        if out is None:
            if not wait:
                raise ValueError("an asynchronous readback needs its output array")
            out = np.empty((height, width, 4), np.float32)
        flags = N.READ_ASYNC if not wait else (N.READ_POLL if poll else N.READ_WAIT)
        N.check(self._lib.snelly_readback(self._h, jid, out.ctypes.data, out.nbytes, flags))
        return out

    def readback_state(self, jid, width, height, fp64=False):
        n = width * height
        rng = np.empty((n, 4), np.uint32)
        acc = np.empty((n, 4), np.float32)
        comp = np.empty((n, 4), np.float32)
        acc64 = np.empty((n, 4), np.float64) if fp64 else None
        N.check(self._lib.snelly_readback_state(self._h, jid, rng.ctypes.data, acc.ctypes.data, comp.ctypes.data,
                                                acc64.ctypes.data if fp64 else None))
        return rng, acc, comp, acc64

    def image_stats(self, jid):
        """Sums over pixels of mean X, Y, Z, Y^2 and the total sample count (float64[5])."""
        out = np.zeros(5, np.float64)
        N.check(self._lib.snelly_image_stats(self._h, jid, out.ctypes.data))
        return out

    def status(self, jid):
        a, b = ctypes.c_int(), ctypes.c_int()
        N.check(self._lib.snelly_job_status(self._h, jid, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def cancel(self, jid):
        N.check(self._lib.snelly_cancel(self._h, jid))

    def destroy_job(self, jid):
        N.check(self._lib.snelly_destroy_job(self._h, jid))

    def sync(self):
        N.check(self._lib.snelly_sync(self._h))

    def stream(self):
        return self._lib.snelly_stream(self._h)

    def launch_count(self):
        return self._lib.snelly_launch_count(self._h)

    def fp32_peak(self):
        t, ms = ctypes.c_double(), ctypes.c_double()
        N.check(self._lib.snelly_measure_fp32_peak(self._h, ctypes.byref(t), ctypes.byref(ms)))
        return t.value, ms.value

    def flush_l2(self, nbytes=256 << 20):
        N.check(self._lib.snelly_flush_l2(self._h, int(nbytes)))
