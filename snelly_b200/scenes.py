"""Benchmark and test scenes, written against the reference's scene API.

Each scene is the synthetic workload of one benchmark configuration: C0 "plain method, small
size", C1 "dispersive and metallic fractal" (the headline 1080p workload), C2 "volumetric and
subsurface". Their GLSL is written for this package; the fractal distance estimators are the
standard Menger-sponge and Mandelbox formulations.
"""
import math

import numpy as np

from .api import Dielectric, FlatSpectrum


class PlainSphere:
    """C0: sphere of radius 1 unioned with the plane y = -1, diffuse grey 0.8, roughness 0.3,
    uniform white environment of radiance 1, 256x256, pinhole camera at (0,1,5) looking at the
    origin, fov 45, maxBounces 4, 16 spp, maxMarchSteps 256, minLengthScale 1e-4, wavelengths
    drawn from a flat 390-750 nm spectrum."""

    width, height, spp = 256, 256, 16

    def __init__(self, width=None, height=None):
        if width:
            self.width = width
        if height:
            self.height = height

    def init(self, snelly):
        r = snelly.getRenderer()
        r.width, r.height = self.width, self.height
        r.dispersive = True
        r.interactive = False
        r.maxBounces = 4
        r.maxMarchSteps = 256
        r.skyPower = 0.0          # 10^0 = radiance 1
        r.sunPower = -7.0         # off
        r.envMapVisible = True
        cam = snelly.getCamera()
        cam.fov = 45.0
        cam.position.set(0.0, 1.0, 5.0)
        cam.aperture = -math.inf  # pinhole
        snelly.getControls().target.set(0.0, 0.0, 0.0)
        s = snelly.getMaterials().loadSurface()
        s.diffuseAlbedo = [0.8, 0.8, 0.8]
        s.specAlbedo = [0.0, 0.0, 0.0]
        s.roughness = 0.3

    def after_init(self, snelly):
        # Snelly.initScene loads the blackbody spectrum after init() (js/snelly.js:285-286), so the
        # flat spectrum is selected afterwards, as a user does from the GUI or console
        snelly.addSpectrum(FlatSpectrum("flat", "Flat spectrum", 390.0, 750.0))
        snelly.loadSpectrum("flat")

    def shader(self):
        return """
float SDF_SURFACE(vec3 X)
{
    float sphere = length(X) - 1.0;
    float ground = X.y + 1.0;
    return min(sphere, ground);
}
"""

    def getMinLengthScale(self):
        return 1.0e-4


class LowSunNoSky(PlainSphere):
    """C0's sphere and ground under a low sun (latitude 8 degrees) and no sky, maxBounces 2:
    surface vertices that face away from the sun sample no light at all, so a path whose last
    vertex is one of them finishes with no shadow ray to trace."""

    def __init__(self, width=None, height=None, sun_latitude=8.0):
        super().__init__(width, height)
        self.sun_latitude = sun_latitude

    def init(self, snelly):
        super().init(snelly)
        r = snelly.getRenderer()
        r.maxBounces = 2
        r.skyPower = -7.0         # off
        r.sunPower = math.log10(20.0)
        r.sunAngularSize = 3.0
        r.sunLatitude = self.sun_latitude
        r.sunLongitude = 120.0

    def after_init(self, snelly):
        pass


class DispersiveSphere:
    """A rough dielectric sphere of radius 1 on a diffuse ground plane y = -1 under a 2-degree
    sun and a sky, dispersive, maxBounces 6: the scene of the IOR-model parity cases. `dielectric`
    names one of the reference's registered dielectrics (js/materials.js:1125-1147); `abbe`, when
    given, sets the Abbe number (and `ior` the refractive index at the d line) of the Abbe model."""

    width, height = 48, 48

    def __init__(self, width=None, height=None, dielectric="Rutile", abbe=None, ior=None):
        if width:
            self.width = width
        if height:
            self.height = height
        self.dielectric, self.abbe, self.ior = dielectric, abbe, ior

    def init(self, snelly):
        r = snelly.getRenderer()
        r.width, r.height = self.width, self.height
        r.dispersive = True
        r.interactive = False
        r.maxBounces = 6
        r.maxMarchSteps = 256
        r.skyPower = math.log10(0.6)
        r.sunPower = math.log10(12.0)
        r.sunAngularSize = 2.0
        r.sunLatitude = 40.0
        r.sunLongitude = 200.0
        cam = snelly.getCamera()
        cam.fov = 40.0
        cam.position.set(0.4, 1.2, 4.2)
        cam.aperture = -math.inf
        snelly.getControls().target.set(0.0, -0.2, 0.0)
        m = snelly.getMaterials()
        d = m.loadDielectric(self.dielectric)
        if self.abbe is not None:
            d.abbe = self.abbe
        if self.ior is not None:
            d.iorVal = self.ior
        d.roughness = 0.03
        s = m.loadSurface()
        s.diffuseAlbedo = [0.7, 0.7, 0.7]
        s.specAlbedo = [0.0, 0.0, 0.0]
        s.roughness = 0.4

    def shader(self):
        return """
float SDF_DIELECTRIC(vec3 X)
{
    return length(X) - 1.0;
}

float SDF_SURFACE(vec3 X)
{
    return X.y + 1.0;
}
"""

    def getMinLengthScale(self):
        return 1.0e-4


def c1_camera(seed=2):
    """Camera pose of C1 drawn from `seed`: a point at distance U(4.5, 6) from the look-at point
    (0.6, 0, 0), azimuth U(60, 120) degrees about +y from the +x axis (so the sponge and the gold
    sphere are side by side in view), elevation U(12, 35) degrees."""
    rs = np.random.RandomState(seed)
    az = math.radians(rs.uniform(60.0, 120.0))
    el = math.radians(rs.uniform(12.0, 35.0))
    dist = rs.uniform(4.5, 6.0)
    target = (0.6, 0.0, 0.0)
    pos = (target[0] + dist * math.cos(el) * math.cos(az), target[1] + dist * math.sin(el),
           target[2] + dist * math.cos(el) * math.sin(az))
    return pos, target


class DispersiveFractal:
    """C1: a 5-iteration Menger sponge of side 2 as a dispersive dielectric (Cauchy
    n = 1.50 + 0.0042 / lambda_um^2, roughness 0.02), a gold sphere of radius 0.7 at (1.8, 0, 0)
    (the reference's tabulated gold n,k, roughness 0.15) and a ground plane y = -1.2 of diffuse
    albedo 0.5; a 3-degree sun cone of radiance 20 over a sky of radiance 0.5. 1920x1080,
    64 spp, maxBounces 8, maxMarchSteps 512."""

    width, height, spp = 1920, 1080, 64

    def __init__(self, width=None, height=None, iterations=5, seed=2, dispersive=True):
        if width:
            self.width = width
        if height:
            self.height = height
        self.iterations = iterations
        self.seed = seed
        self.dispersive = dispersive

    def init(self, snelly):
        r = snelly.getRenderer()
        r.width, r.height = self.width, self.height
        r.dispersive = self.dispersive
        r.interactive = False
        r.maxBounces = 8
        r.maxMarchSteps = 512
        r.skyPower = math.log10(0.5)
        r.sunPower = math.log10(20.0)
        r.sunAngularSize = 3.0
        r.sunLatitude = 45.0
        r.sunLongitude = 30.0
        r.envMapTransitionAngle = 135.0
        cam = snelly.getCamera()
        cam.fov = 45.0
        pos, target = c1_camera(self.seed)
        cam.position.set(*pos)
        cam.aperture = -math.inf
        snelly.getControls().target.set(*target)
        m = snelly.getMaterials()
        d = Dielectric("C1 Cauchy", "cauchy", [1.50, 0.0042, -2.0])  # CauchyDielectric coefficients
        m.dielectrics[d.getName()] = d
        m.loadDielectric(d.getName())
        d.roughness = 0.02
        g = m.loadMetal("Gold")
        g.roughness = 0.15
        s = m.loadSurface()
        s.diffuseAlbedo = [0.5, 0.5, 0.5]
        s.specAlbedo = [0.0, 0.0, 0.0]
        s.roughness = 0.5

    def shader(self):
        return f"""
float box(vec3 p, vec3 halfSize)
{{
    vec3 q = abs(p) - halfSize;
    return min(max(q.x, max(q.y, q.z)), 0.0) + length(max(q, 0.0));
}}

float SDF_DIELECTRIC(vec3 X)
{{
    // Menger sponge of side 2 centred at the origin
    float d = box(X, vec3(1.0));
    float s = 1.0;
    for (int i = 0; i < {self.iterations}; ++i)
    {{
        vec3 a = mod(X * s, 2.0) - 1.0;
        s *= 3.0;
        vec3 r = abs(1.0 - 3.0 * abs(a));
        float da = max(r.x, r.y);
        float db = max(r.y, r.z);
        float dc = max(r.z, r.x);
        float c = (min(da, min(db, dc)) - 1.0) / s;
        d = max(d, c);
    }}
    return d;
}}

float SDF_METAL(vec3 X)
{{
    return length(X - vec3(1.8, 0.0, 0.0)) - 0.7;
}}

float SDF_SURFACE(vec3 X)
{{
    return X.y + 1.2;
}}
"""

    def getMinLengthScale(self):
        return 1.0e-4


class VolumetricSubsurface:
    """C2 (surface part): a 12-iteration Mandelbox of scale 2 and minimum radius 0.5 with
    subsurface scattering (albedo (0.9, 0.6, 0.4), mean free path 0.05, Henyey-Greenstein
    g = 0.3), sky light and sun; 1024x1024, 128 spp, maxBounces 12."""

    width, height, spp = 1024, 1024, 128

    def __init__(self, width=None, height=None):
        if width:
            self.width = width
        if height:
            self.height = height

    def init(self, snelly):
        r = snelly.getRenderer()
        r.width, r.height = self.width, self.height
        r.dispersive = True
        r.interactive = False
        r.maxBounces = 12
        r.maxMarchSteps = 256
        r.maxSSSSteps = 128
        r.skyPower = math.log10(0.8)
        r.sunPower = math.log10(8.0)
        r.sunAngularSize = 4.0
        r.sunLatitude = 55.0
        r.sunLongitude = 120.0
        cam = snelly.getCamera()
        cam.fov = 45.0
        cam.position.set(-7.5, 5.0, -6.0)
        cam.aperture = -math.inf
        snelly.getControls().target.set(0.0, 0.0, 0.0)
        s = snelly.getMaterials().loadSurface()
        s.diffuseAlbedo = [0.8, 0.7, 0.6]
        s.specAlbedo = [0.1, 0.1, 0.1]
        s.roughness = 0.2
        s.subsurface = 1.0
        s.subsurfaceAlbedoRGB = [0.9, 0.6, 0.4]
        s.subsurfaceMFP = 0.05
        s.subsurfaceAnisotropy = 0.3

    def shader(self):
        return """
uniform float boxScale;
uniform float minRadius2;

float SDF_SURFACE(vec3 X)
{
    // Mandelbox distance estimate: box fold, sphere fold, scale and translate
    vec3 z = X;
    float dr = 1.0;
    float fixedRadius2 = 1.0;
    for (int i = 0; i < 12; ++i)
    {
        z = clamp(z, -1.0, 1.0) * 2.0 - z;
        float r2 = dot(z, z);
        if (r2 < minRadius2) { float t = fixedRadius2 / minRadius2; z *= t; dr *= t; }
        else if (r2 < fixedRadius2) { float t = fixedRadius2 / r2; z *= t; dr *= t; }
        z = boxScale * z + X;
        dr = dr * abs(boxScale) + 1.0;
    }
    return length(z) / abs(dr);
}
"""

    def syncShader(self, snelly, shader):
        shader.uniformF("boxScale", 2.0)
        shader.uniformF("minRadius2", 0.25)

    def getMinLengthScale(self):
        return 1.0e-4


class PyroclasticSubsurface(VolumetricSubsurface):
    """C2 complete: the subsurface Mandelbox together with a pyroclastic cloud between it and the
    camera, a sphere of radius 1 at `centre` displaced by 5-octave fBm value noise of amplitude
    0.3 (lattice hash offset by `seed`), scattering coefficient 2 and absorption 0.1 per unit
    length, Henyey-Greenstein g = 0.5. The cloud is a heterogeneous medium given through the
    VOLUME_EXTINCTION / VOLUME_EXTINCTION_MAX hooks, which the reference declares but never calls:
    this build's extension renders it (delta tracking), the reference's shader would not."""

    def __init__(self, width=None, height=None, seed=3, centre=(-4.8, 3.4, -3.9)):
        super().__init__(width, height)
        self.seed = seed
        self.centre = centre

    def init(self, snelly):
        super().init(snelly)
        v = snelly.getMaterials().loadVolume()
        cx, cy, cz = self.centre
        v.atmosphereMinX, v.atmosphereMaxX = cx - 1.5, cx + 1.5
        v.atmosphereMinY, v.atmosphereMaxY = cy - 1.5, cy + 1.5
        v.atmosphereMinZ, v.atmosphereMaxZ = cz - 1.5, cz + 1.5
        v.lof10_mfp = 0.0
        v.scatteringColor = [2.0, 2.0, 2.0]
        v.absorptionColor = [0.1, 0.1, 0.1]
        v.anisotropy = 0.5

    def shader(self):
        return super().shader() + """
uniform vec3 cloudCentre;
uniform float cloudSeed;

// pseudo-random value in [0, 1) at an integer lattice point
float cloudLattice(vec3 q)
{
    q = fract(q * vec3(0.1183, 0.1517, 0.1297) + vec3(cloudSeed * 0.0713));
    q += dot(q, q.yzx + 23.17);
    return fract((q.x + q.y) * q.z * 95.43);
}

// trilinear value noise with smoothstep weights, in [0, 1]
float cloudNoise(vec3 p)
{
    vec3 i = floor(p);
    vec3 f = p - i;
    f = f * f * (3.0 - 2.0 * f);
    float n000 = cloudLattice(i);
    float n100 = cloudLattice(i + vec3(1.0, 0.0, 0.0));
    float n010 = cloudLattice(i + vec3(0.0, 1.0, 0.0));
    float n110 = cloudLattice(i + vec3(1.0, 1.0, 0.0));
    float n001 = cloudLattice(i + vec3(0.0, 0.0, 1.0));
    float n101 = cloudLattice(i + vec3(1.0, 0.0, 1.0));
    float n011 = cloudLattice(i + vec3(0.0, 1.0, 1.0));
    float n111 = cloudLattice(i + vec3(1.0, 1.0, 1.0));
    float x00 = mix(n000, n100, f.x);
    float x10 = mix(n010, n110, f.x);
    float x01 = mix(n001, n101, f.x);
    float x11 = mix(n011, n111, f.x);
    return mix(mix(x00, x10, f.y), mix(x01, x11, f.y), f.z);
}

// 5-octave fBm in [-1, 1]
float cloudFbm(vec3 p)
{
    float sum = 0.0;
    float amp = 0.5;
    float norm = 0.0;
    for (int o = 0; o < 5; ++o)
    {
        sum += amp * (2.0 * cloudNoise(p) - 1.0);
        norm += amp;
        p *= 2.03;
        amp *= 0.5;
    }
    return sum / norm;
}

float VOLUME_EXTINCTION(float extinction_ui, vec3 X)
{
    vec3 q = X - cloudCentre;
    float r = 1.0 + 0.3 * cloudFbm(2.5 * q);
    return length(q) < r ? extinction_ui : 0.0;
}

float VOLUME_EXTINCTION_MAX(float extinction_ui)
{
    return extinction_ui;
}
"""

    def syncShader(self, snelly, shader):
        super().syncShader(snelly, shader)
        shader.uniform3F("cloudCentre", *self.centre)
        shader.uniformF("cloudSeed", float(self.seed))


class AtmosphereLights:
    """Coverage scene: homogeneous atmosphere with multiple scattering, fake fog, sphere light,
    sun and sky over a metal sphere, a glass box with absorption and a diffuse ground (RGB mode,
    thin-lens camera). Exercises PT:971-1457 and the sphere-light paths."""

    width, height, spp = 64, 48, 4

    def __init__(self, width=None, height=None, dispersive=False):
        if width:
            self.width = width
        if height:
            self.height = height
        self.dispersive = dispersive

    def init(self, snelly):
        r = snelly.getRenderer()
        r.width, r.height = self.width, self.height
        r.dispersive = self.dispersive
        r.interactive = False
        r.maxBounces = 5
        r.maxAtmosphereScatters = 3
        r.maxMarchSteps = 200
        r.skyPower = math.log10(0.7)
        r.sunPower = math.log10(5.0)
        r.sunAngularSize = 6.0
        r.sunLatitude = 35.0
        r.sunLongitude = 60.0
        r.sphereLightPower = math.log10(40.0)
        r.sphereLightRadius = 0.3
        r.sphereLightPosition = [-1.2, 1.6, 0.6]
        r.sphereLightColor = [1.0, 0.8, 0.6]
        r.envMapTransitionAngle = 60.0
        r.skyTintUp = [0.6, 0.7, 1.0]
        r.skyTintDown = [0.9, 0.8, 0.6]
        cam = snelly.getCamera()
        cam.fov = 50.0
        cam.position.set(0.3, 1.4, 4.5)
        cam.aperture = -4.0
        cam.focalDistance = math.log10(4.3)
        snelly.getControls().target.set(0.0, 0.2, 0.0)
        m = snelly.getMaterials()
        m.loadMetal("Copper").roughness = 0.08
        d = m.loadDielectric("Glass (BK7)")
        d.roughness = 0.05
        d.absorptionColor = [0.6, 0.9, 0.8]
        d.absorptionScale = 2.0
        s = m.loadSurface()
        s.diffuseAlbedo = [0.7, 0.65, 0.6]
        s.specAlbedo = [0.3, 0.3, 0.3]
        s.roughness = 0.25
        v = m.loadVolume()
        v.scatteringColor = [0.35, 0.4, 0.5]
        v.absorptionColor = [0.05, 0.05, 0.08]
        v.lof10_mfp = 0.6
        v.anisotropy = 0.3
        v.atmosphereMinY = -1.0
        v.atmosphereMaxY = 3.0
        v.fogEnable = True
        v.fogMFP = 1.0
        v.fogMaxOpticalDepth = 0.5

    def shader(self):
        return """
float SDF_METAL(vec3 X) { return length(X - vec3(0.9, 0.0, 0.0)) - 0.6; }
float SDF_DIELECTRIC(vec3 X)
{
    vec3 q = abs(X - vec3(-0.8, 0.0, 0.2)) - vec3(0.45, 0.6, 0.45);
    return min(max(q.x, max(q.y, q.z)), 0.0) + length(max(q, 0.0)) - 0.05;
}
float SDF_SURFACE(vec3 X) { return X.y + 0.6; }
"""


class HooksAndMaps:
    """Coverage scene: every material hook of the scene API (diffuse / specular / roughness /
    subsurface albedo hooks, metal and dielectric hooks, normal maps on all three materials),
    INIT() state and scene uniforms, a custom primary-ray hook using rand(), a monochromatic
    spectrum (dispersive mode)."""

    width, height, spp = 48, 48, 4

    def __init__(self, width=None, height=None):
        if width:
            self.width = width
        if height:
            self.height = height

    def init(self, snelly):
        r = snelly.getRenderer()
        r.width, r.height = self.width, self.height
        r.dispersive = True
        r.interactive = False
        r.maxBounces = 4
        r.maxMarchSteps = 160
        r.skyPower = 0.0
        r.sunPower = math.log10(3.0)
        r.sunLatitude = 60.0
        cam = snelly.getCamera()
        cam.fov = 40.0
        cam.position.set(0.0, 1.0, 4.0)
        snelly.getControls().target.set(0.0, 0.0, 0.0)
        m = snelly.getMaterials()
        m.loadMetal("Silver").roughness = 0.1
        m.loadDielectric("Water").roughness = 0.02
        s = m.loadSurface()
        s.diffuseAlbedo = [0.8, 0.3, 0.2]
        s.specAlbedo = [0.2, 0.2, 0.2]
        s.roughness = 0.3
        s.subsurface = 0.5
        s.subsurfaceMFP = 0.1
        s.subsurfaceAlbedoRGB = [0.8, 0.8, 0.7]

    def after_init(self, snelly):
        from .api import MonochromaticSpectrum
        snelly.addSpectrum(MonochromaticSpectrum("mono", "550 nm", 550.0))  # selected after initScene
        snelly.loadSpectrum("mono")

    def shader(self):
        return """
uniform float ripple;
uniform vec3 tint;
mat2 spin;
void INIT() { float a = 0.3 * ripple; spin = mat2(cos(a), sin(a), -sin(a), cos(a)); }
float SDF_SURFACE(vec3 X) { return min(X.y + 1.0, length(X - vec3(-1.1, -0.4, 0.0)) - 0.6); }
float SDF_METAL(vec3 X) { vec3 p = X - vec3(1.1, -0.3, 0.0); p.xz = spin * p.xz; return length(max(abs(p) - vec3(0.4), 0.0)) - 0.1; }
float SDF_DIELECTRIC(vec3 X) { return length(X - vec3(0.0, -0.3, 0.3)) - 0.5; }
vec3 SURFACE_DIFFUSE_REFLECTANCE(in vec3 C, in vec3 X, in vec3 N, in vec3 V)
{
    float c = mod(floor(2.0*X.x) + floor(2.0*X.z), 2.0);
    return mix(C, tint, c);
}
vec3 SURFACE_SPECULAR_REFLECTANCE(in vec3 C, in vec3 X, in vec3 N, in vec3 V) { return C * (0.5 + 0.5*abs(N.y)); }
float SURFACE_ROUGHNESS(in float roughness, in vec3 X, in vec3 N) { return roughness * (1.0 + 0.5*sin(3.0*X.x)); }
vec3 SUBSURFACE_ALBEDO(in vec3 C, in vec3 X, in vec3 N) { return C.zyx; }
vec3 METAL_SPECULAR_REFLECTANCE(in vec3 C, in vec3 X, in vec3 N, in vec3 V) { return vec3(1.0, 0.9, 0.8) * C; }
float METAL_ROUGHNESS(in float roughness, in vec3 X, in vec3 N) { return roughness + 0.05*fract(X.y*3.0); }
vec3 DIELECTRIC_SPECULAR_REFLECTANCE(in vec3 C, in vec3 X, in vec3 N, in vec3 V) { return vec3(0.95); }
float DIELECTRIC_ROUGHNESS(in float roughness, in vec3 X, in vec3 N) { return roughness; }
vec3 DIELECTRIC_ABSORPTION(vec3 absorption_ui, vec3 X) { return absorption_ui + vec3(0.2, 0.05, 0.0); }
vec3 SURFACE_NORMAL_MAP(in vec3 X, in vec3 N) { return vec3(0.1*sin(8.0*X.x), 0.1*cos(8.0*X.z), 1.0); }
vec3 METAL_NORMAL_MAP(in vec3 X, in vec3 N) { return vec3(0.05*sin(20.0*X.y), 0.0, 1.0); }
vec3 DIELECTRIC_NORMAL_MAP(in vec3 X, in vec3 N) { return vec3(0.0, 0.08*sin(12.0*X.x), 1.0); }
void CONSTRUCT_PRIMARY_RAY(in vec2 pixel, inout vec4 rnd, inout vec3 primaryStart, inout vec3 primaryDir)
{
    vec2 ndc = -1.0 + 2.0*(pixel/vec2(48.0, 48.0));
    float jitter = 0.002 * (rand(rnd) - 0.5);
    primaryStart = vec3(0.0, 1.0, 4.0);
    primaryDir = normalize(vec3(0.36*ndc.x + jitter, 0.36*ndc.y - 0.25, -1.0));
}
"""

    def syncShader(self, snelly, shader):
        shader.uniformF("ripple", 1.5)
        shader.uniform3Fv("tint", [0.1, 0.6, 0.2])


def sky_env_map(width=64, height=32):
    """A procedural lat-long environment map (sRGB8, row 0 = the top row, as an image loads): a
    blue-to-white sky gradient over a brown ground with a bright sun patch, for the env-map
    coverage scene."""
    v = (np.arange(height) + 0.5) / height  # 0 at the top (theta = 0)
    u = (np.arange(width) + 0.5) / width
    uu, vv = np.meshgrid(u, v)
    sky = np.stack([0.35 + 0.6 * vv, 0.55 + 0.4 * vv, 0.95 + 0.0 * vv], -1)
    ground = np.stack([0.35 + 0.0 * vv, 0.25 + 0.0 * vv, 0.15 + 0.0 * vv], -1)
    img = np.where((vv < 0.5)[..., None], sky, ground)
    sun = np.exp(-(((uu - 0.3) / 0.04) ** 2 + ((vv - 0.25) / 0.06) ** 2))[..., None]
    img = np.clip(img + 3.0 * sun, 0.0, 1.0)
    return np.ascontiguousarray((img * 255.0 + 0.5).astype(np.uint8))


class EnvMapLit:
    """Coverage scene lit by a lat-long environment map (Scene.envMap): a diffuse sphere and a
    polished aluminium sphere on a ground plane, the map rotated by envMapPhiRotation /
    envMapThetaRotation and visible to camera rays; no sun."""

    width, height, spp = 48, 48, 4

    def __init__(self, width=None, height=None):
        if width:
            self.width = width
        if height:
            self.height = height

    def init(self, snelly):
        r = snelly.getRenderer()
        r.width, r.height = self.width, self.height
        r.dispersive = True
        r.interactive = False
        r.maxBounces = 4
        r.maxMarchSteps = 200
        r.skyPower = math.log10(1.5)
        r.sunPower = -7.0
        r.envMapVisible = True
        r.envMapPhiRotation = 40.0
        r.envMapThetaRotation = 15.0
        cam = snelly.getCamera()
        cam.fov = 50.0
        cam.position.set(0.0, 0.8, 4.0)
        cam.aperture = -math.inf
        snelly.getControls().target.set(0.0, 0.0, 0.0)
        s = snelly.getMaterials().loadSurface()
        s.diffuseAlbedo = [0.7, 0.6, 0.5]
        s.specAlbedo = [0.1, 0.1, 0.1]
        s.roughness = 0.3
        snelly.getMaterials().loadMetal("Aluminium").roughness = 0.05

    def shader(self):
        return """
float SDF_SURFACE(vec3 X) { return min(length(X - vec3(-0.9, 0.0, 0.0)) - 0.8, X.y + 0.8); }
float SDF_METAL(vec3 X) { return length(X - vec3(0.9, -0.2, 0.0)) - 0.6; }
"""

    def envMap(self):
        return sky_env_map()


_GRIDS = {}


def sphere_blend_grid(res=256, seed=4, count=32, k=0.1, extent=1.5):
    """The mesh-like distance grid: res^3 float16 samples, at texel centres of the cube
    [-extent, extent]^3, of the polynomial smooth minimum (blend width k) of `count` sphere
    distances, radii U(0.1, 0.4) and centres U[-1, 1]^3 drawn from `seed`. Shape (d, h, w, 1),
    x fastest. Cached per argument set, so every scene instance binds the same array."""
    key = (res, seed, count, k, extent)
    if key not in _GRIDS:
        rs = np.random.RandomState(seed)
        centres = rs.uniform(-1.0, 1.0, (count, 3)).astype(np.float32)
        radii = rs.uniform(0.1, 0.4, count).astype(np.float32)
        c = ((np.arange(res, dtype=np.float32) + 0.5) / res * 2.0 - 1.0) * extent
        y, x = np.meshgrid(c, c, indexing="ij")
        grid = np.empty((res, res, res, 1), np.float16)
        for iz in range(res):
            d = None
            for n in range(count):
                dn = np.sqrt((x - centres[n, 0]) ** 2 + (y - centres[n, 1]) ** 2 + (c[iz] - centres[n, 2]) ** 2) - radii[n]
                if d is None:
                    d = dn
                else:
                    h = np.maximum(k - np.abs(d - dn), 0.0) / k
                    d = np.minimum(d, dn) - h * h * k * 0.25
            grid[iz, :, :, 0] = d
        _GRIDS[key] = grid
    return _GRIDS[key]


class MeshLike:
    """C3's mesh-like SDF: a 256^3 float16 distance grid sampled trilinearly (a sampler3D, as the
    reference's mesh scenes bind theirs), holding the smooth minimum of 32 spheres (radii
    U(0.1, 0.4), centres U[-1, 1]^3, seed 4), over a ground plane y = -1.6; diffuse grey surface,
    sky radiance 1 and a sun."""

    width, height, spp = 512, 512, 16

    def __init__(self, width=None, height=None, res=256, seed=4):
        if width:
            self.width = width
        if height:
            self.height = height
        self.res, self.seed = res, seed

    def init(self, snelly):
        r = snelly.getRenderer()
        r.width, r.height = self.width, self.height
        r.dispersive = True
        r.interactive = False
        r.maxBounces = 6
        r.maxMarchSteps = 256
        r.skyPower = 0.0
        r.sunPower = math.log10(5.0)
        r.sunAngularSize = 4.0
        r.sunLatitude = 55.0
        r.sunLongitude = 20.0
        cam = snelly.getCamera()
        cam.fov = 40.0
        cam.position.set(0.0, 1.5, 5.5)
        cam.aperture = -math.inf
        snelly.getControls().target.set(0.0, -0.2, 0.0)
        s = snelly.getMaterials().loadSurface()
        s.diffuseAlbedo = [0.7, 0.7, 0.7]
        s.specAlbedo = [0.04, 0.04, 0.04]
        s.roughness = 0.4

    def shader(self):
        return """
uniform sampler3D sdfTex;
uniform vec3 gridMin;
uniform vec3 gridSize;

float sdBox(vec3 X, vec3 bmin, vec3 bmax)
{
    vec3 d = abs(X - 0.5*(bmin + bmax)) - 0.5*(bmax - bmin);
    return min(max(d.x, max(d.y, d.z)), 0.0) + length(max(d, 0.0));
}

float SDF_SURFACE(vec3 X)
{
    float ground = X.y + 1.6;
    float box = sdBox(X, gridMin, gridMin + gridSize);
    float mesh;
    if (box > 0.0) mesh = box + 0.02;  // outside the grid: a lower bound of the distance to its contents
    else mesh = texture(sdfTex, (X - gridMin) / gridSize).r;
    return min(mesh, ground);
}
"""

    def syncShader(self, snelly, shader):
        shader.uniformTexture("sdfTex", sphere_blend_grid(self.res, self.seed))
        shader.uniform3Fv("gridMin", [-1.5, -1.5, -1.5])
        shader.uniform3Fv("gridSize", [3.0, 3.0, 3.0])


class SdfAsset(MeshLike):
    """A mesh distance grid loaded from an SDF-PNG asset (scripts/pngPacker.html format, see
    sdfpng.py) over a ground plane, bound like the reference's mesh scenes bind theirs: the grid
    spans ORIG .. ORIG + EDGE of the asset's metadata."""

    def __init__(self, path, width=None, height=None):
        super().__init__(width, height)
        from .sdfpng import load_texture
        self.meta, self.grid = load_texture(path)

    def syncShader(self, snelly, shader):
        shader.uniformTexture("sdfTex", self.grid)
        shader.uniform3Fv("gridMin", [float(v) for v in self.meta["ORIG"]])
        shader.uniform3Fv("gridSize", [float(v) for v in self.meta["EDGE"]])


class Turntable:
    """An animated scene written to the reference's scene template (js/sceneAPI.js:16-397): a
    sphere smoothly blended with a box above a ground plane, the scene parameters `radius` and
    `blend` uploaded as uniforms, init/initGenerator for those parameters, and a turntable orbit
    of the camera about the look-at point driven from preframeCallback. Every animation frame
    accumulates `target_spp` samples; postframeCallback then hands the finished frame to
    `on_frame(index, snelly)` (the reference posts the canvas to a local server there) and the
    next preframeCallback moves to the next animation frame and resets the accumulation
    without a recompile."""

    width, height = 96, 96

    def __init__(self, width=None, height=None, frames=24, target_spp=16, period=24.0, on_frame=None):
        if width:
            self.width = width
        if height:
            self.height = height
        self.frames, self.target_spp, self.period, self.on_frame = frames, target_spp, period, on_frame

    def init(self, snelly):
        self.parameters = {"radius": 0.6, "blend": 0.25}
        self.animFrame = 0
        self.advanceFrame = False
        self.exported = -1
        r = snelly.getRenderer()
        r.width, r.height = self.width, self.height
        r.dispersive = True
        r.interactive = False
        r.maxBounces = 4
        r.maxMarchSteps = 192
        r.skyPower = 0.0
        r.sunPower = math.log10(4.0)
        r.sunLatitude = 55.0
        cam = snelly.getCamera()
        cam.fov = 40.0
        cam.aperture = -math.inf
        cam.position.set(0.0, 1.2, 4.0)
        snelly.getControls().target.set(0.2, -0.2, 0.0)
        srf = snelly.getMaterials().loadSurface()
        srf.diffuseAlbedo = [0.7, 0.45, 0.3]
        srf.specAlbedo = [0.1, 0.1, 0.1]
        srf.roughness = 0.25

    def initGenerator(self):
        """The init statements that restore the current parameters (Scene.initGenerator,
        js/sceneAPI.js:83-91), for Snelly.dumpScene(lang="python")."""
        return (f"\nself.parameters = {{}}\nself.parameters['radius'] = {self.parameters['radius']!r}\n"
                f"self.parameters['blend'] = {self.parameters['blend']!r}\nself.animFrame = {self.animFrame!r}\n"
                f"self.advanceFrame = False\nself.exported = -1\n")

    def shader(self):
        return """
uniform float radius;
uniform float blend;
float sdBox(vec3 p, vec3 b) { vec3 q = abs(p) - b; return length(max(q, 0.0)) + min(max(q.x, max(q.y, q.z)), 0.0); }
float smin(float a, float b, float k) { float h = clamp(0.5 + 0.5*(b - a)/k, 0.0, 1.0); return mix(b, a, h) - k*h*(1.0 - h); }
float SDF_SURFACE(vec3 X)
{
    float s = length(X) - radius;
    float b = sdBox(X - vec3(0.8, -0.45, 0.0), vec3(0.35));
    return min(smin(s, b, blend), X.y + 0.8);
}
"""

    def syncShader(self, snelly, shader):
        shader.uniformF("radius", self.parameters["radius"])
        shader.uniformF("blend", self.parameters["blend"])

    def pose(self, snelly, frame):
        """Camera and scene parameters of animation frame `frame`: the camera turned about the
        vertical axis through the look-at point by 360 degrees per `period` frames, the sphere
        radius and the blend width breathing with the same phase."""
        if not hasattr(self, "_orbit"):
            cam, tgt = snelly.getCamera().position, snelly.getControls().target
            self._orbit = (tgt.tolist(), [cam.x - tgt.x, cam.y - tgt.y, cam.z - tgt.z])
        (tx, ty, tz), (ox, oy, oz) = self._orbit
        phase = 2.0 * math.pi * frame / self.period
        c, s = math.cos(phase), math.sin(phase)
        snelly.getCamera().position.set(tx + c * ox + s * oz, ty + oy, tz - s * ox + c * oz)
        self.parameters["radius"] = 0.6 + 0.15 * math.sin(phase)
        self.parameters["blend"] = 0.25 + 0.15 * math.cos(phase)

    def preframeCallback(self, snelly, gl):
        if self.advanceFrame:  # the previous frame was handed over: start the next one
            self.animFrame += 1
            self.advanceFrame = False
            snelly.getRenderer().reset(True)
        self.pose(snelly, self.animFrame)

    def postframeCallback(self, snelly, gl):
        r = snelly.getRenderer()
        if self.animFrame < self.frames and r.getSPP() >= self.target_spp and self.exported != self.animFrame:
            if self.on_frame is not None:
                self.on_frame(self.animFrame, snelly)
            self.exported = self.animFrame
            self.advanceFrame = self.animFrame + 1 < self.frames


SCENES = {"c0": PlainSphere, "c1": DispersiveFractal, "c2": VolumetricSubsurface, "atmosphere": AtmosphereLights,
          "hooks": HooksAndMaps, "mesh": MeshLike, "envmap": EnvMapLit, "turntable": Turntable,
          "lowsun": LowSunNoSky, "c2_cloud": PyroclasticSubsurface}
