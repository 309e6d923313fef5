"""CPU oracle for the spectral path tracer: build per scene, render pixels, seed, compare.

TEST INFRASTRUCTURE. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this module. It compiles oracle/pt_oracle.h (a sequential C++ restatement of
shaders/pathtracer-fragment-shader.glsl) together with one scene into a shared library with
g++ (-O3, no fast-math, no FMA contraction, OpenMP over pixels).

The host-side steps the reference performs before drawing are restated here as well:
  * the hook defaults and #defines of Renderer.compileShaders (js/renderer.js:217-316);
  * the emission-spectrum inverse CDF of Spectrum.inverseCDF (js/spectra.js:28-61) with float32
    storage and float64 arithmetic, as the reference's Float32Arrays do.
The GLSL-to-C++ translation itself is the package's translator (snelly_glsl_to_cpp).
"""
import ctypes
import hashlib
import json
import os
import re
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(HERE, "_build")

# js/renderer.js:228-263: (substring searched for, default appended when absent)
HOOK_DEFAULTS = [
    ("INIT(", "void INIT() {}"),
    ("SURFACE_DIFFUSE_REFLECTANCE(", "vec3 SURFACE_DIFFUSE_REFLECTANCE(in vec3 C, in vec3 X, in vec3 N, in vec3 V) { return C; }"),
    ("SURFACE_SPECULAR_REFLECTANCE(", "vec3 SURFACE_SPECULAR_REFLECTANCE(in vec3 C, in vec3 X, in vec3 N, in vec3 V) { return C; }"),
    ("SURFACE_ROUGHNESS(", "float SURFACE_ROUGHNESS(in float roughness, in vec3 X, in vec3 N) { return roughness; }"),
    ("SUBSURFACE_ALBEDO(", "vec3 SUBSURFACE_ALBEDO(in vec3 C, in vec3 X, in vec3 N) { return C; }"),
    ("METAL_SPECULAR_REFLECTANCE(", "vec3 METAL_SPECULAR_REFLECTANCE(in vec3 C, in vec3 X, in vec3 N, in vec3 V) { return C; }"),
    ("METAL_ROUGHNESS(", "float METAL_ROUGHNESS(in float roughness, in vec3 X, in vec3 N) { return roughness; }"),
    ("DIELECTRIC_SPECULAR_REFLECTANCE(", "vec3 DIELECTRIC_SPECULAR_REFLECTANCE(in vec3 C, in vec3 X, in vec3 N, in vec3 V) { return C; }"),
    ("DIELECTRIC_ROUGHNESS(", "float DIELECTRIC_ROUGHNESS(in float roughness, in vec3 X, in vec3 N) { return roughness; }"),
    ("DIELECTRIC_ABSORPTION(", "vec3 DIELECTRIC_ABSORPTION(vec3 absorption_ui, vec3 X) { return absorption_ui; }"),
    ("VOLUME_EXTINCTION(", "float VOLUME_EXTINCTION(float extinction_ui, vec3 X) { return extinction_ui; }"),
    ("VOLUME_EXTINCTION_MAX(", "float VOLUME_EXTINCTION_MAX(float extinction_ui) { return extinction_ui; }"),
    ("VOLUME_SCATTERING_COLOR(", "vec3 VOLUME_SCATTERING_COLOR(vec3 scattering_color_ui, vec3 X) { return scattering_color_ui; }"),
    ("VOLUME_ABSORPTION_COLOR(", "vec3 VOLUME_ABSORPTION_COLOR(vec3 absorption_color_ui, vec3 X) { return absorption_color_ui; }"),
    ("VOLUME_ANISOTROPY(", "float VOLUME_ANISOTROPY(float anisotropy, vec3 X) { return anisotropy; }"),
    ("VOLUME_EMISSION(", "vec3 VOLUME_EMISSION(vec3 emission, vec3 X) { return emission; }"),
]


def assemble(glsl, opts):
    """(GLSL with defaults, #define block) as js/renderer.js:217-316 builds them."""
    s = glsl
    for needle, body in HOOK_DEFAULTS:
        if needle not in s:
            s += "\n " + body + "\n"
    d = []
    if "CONSTRUCT_PRIMARY_RAY(" in glsl:
        d.append("HAS_CUSTOM_CAMERA")
    for key, name in (("SDF_SURFACE(", "HAS_SURFACE"), ("SDF_METAL(", "HAS_METAL"), ("SDF_DIELECTRIC(", "HAS_DIELECTRIC")):
        if key in glsl:
            d.append(name)
    if "VOLUME_EXTINCTION(" in glsl:  # the heterogeneous-medium extension replaces the atmosphere
        d.append("HAS_HETERO_VOLUME")
    elif opts.has_atmosphere:
        d.append("HAS_ATMOSPHERE")
    if opts.has_fog:
        d.append("HAS_FOG")
    if "VOLUME_EMISSION(" in glsl:
        d.append("HAS_VOLUME_EMISSION")
    d.append("HAS_GEOMETRY")
    nm = [k for k in ("SURFACE_NORMAL_MAP(", "METAL_NORMAL_MAP(", "DIELECTRIC_NORMAL_MAP(") if k in glsl]
    if nm:
        d.append("HAS_NORMALMAP")
    for k in nm:
        d.append("HAS_" + k[:-len("_NORMAL_MAP(")] + "_NORMALMAP")
    if opts.interactive:
        d.append("INTERACTIVE_MODE")
    if opts.dispersive:
        d.append("DISPERSION_ENABLED")
    if opts.has_sphere_light:
        d.append("HAS_SPHERE_LIGHT")
    defs = "".join(f"#define {x}\n" for x in d)
    defs += (f"#define MAX_MARCH_STEPS {opts.max_march_steps}\n#define MAX_BOUNCES {opts.max_bounces}\n"
             f"#define MAX_ATMOSPHERE_SCATTERS {opts.max_atmosphere_scatters}\n"
             f"#define MAX_SAMPLES_PER_FRAME {opts.max_samples_per_frame}\n")
    return s, defs


def inverse_cdf(kind, temperature=6000.0, band=(390.0, 750.0), wavelength=550.0, lmin=390.0, lmax=750.0, ns=1024):
    """Spectrum.inverseCDF (js/spectra.js:28-61): float64 arithmetic, float32 stores."""
    if kind == "mono":  # js/spectra.js:76-86
        w = max(lmin, min(wavelength, lmax))
        return np.full(4 * ns, np.float32((w - lmin) / (lmax - lmin)), np.float32)

    def spec(l):
        if kind == "flat":  # js/spectra.js:123-128
            return 0.0 if (l < band[0] or l > band[1]) else 1.0
        b = 1.43877737467e7 / (l * temperature)  # js/spectra.js:179-184
        x = l / 360.0
        return 1.0 / (x * x * x * x * x * (np.exp(b) - 1.0))

    cdf = np.zeros(ns + 1, np.float32)
    dl = (lmax - lmin) / ns
    for n in range(ns):
        cdf[n + 1] = np.float32(float(cdf[n]) + spec(lmin + dl * n))
    total = float(cdf[ns])
    for n in range(ns):
        cdf[n + 1] = np.float32(float(cdf[n + 1]) / total)
    cdf[ns] = 1.0
    icdf = np.zeros(4 * ns, np.float32)
    idx = 0
    for n in range(4 * ns):
        xi = min((n + 1) / (4.0 * ns), 1.0)
        while float(cdf[idx]) < xi:
            idx += 1
        idx = max(1, idx)
        lo, hi = float(cdf[idx - 1]), float(cdf[idx])
        icdf[n] = np.float32((idx - 1.0) / ns + (1.0 / ns) * (xi - lo) / (hi - lo))
    return icdf


def _translate(glsl):
    from snelly_b200 import _native
    return _native.glsl_to_cpp(glsl, "Scene")


def uniform_layout(cpp):
    """[(name, type, offset, array_len)] from the translated uniform block."""
    body = re.search(r"struct SceneUniforms \{(.*?)\};", cpp, re.S).group(1)
    out = []
    for m in re.finditer(r"(\w+) (\w+)(?:\[(\d+)\])?;\s*// offset (\d+)", body):
        out.append((m.group(2), m.group(1), int(m.group(4)), int(m.group(3) or 0)))
    size = int(re.search(r"sizeof\(SceneUniforms\) == (\d+)", cpp).group(1))
    return out, size


def renderer_uniforms(cpp):
    """Names of the renderer's own uniforms the translation added to the scene's block (the scene
    reads them without declaring them); their values come from the job's parameters."""
    body = re.search(r"struct SceneUniforms \{(.*?)\};", cpp, re.S).group(1)
    return set(re.findall(r"\w+ (\w+);\s*// offset \d+, renderer uniform", body))


def sampler_record(kind, array, linear=True):
    """The 32-byte sampler2D / sampler3D record of glslcompat.h for a texture array ((h, w, c) or
    (d, h, w, c) of float32 / float16 / uint8): {data pointer, w, h, [d,] channels, format,
    filter, [srgb]}. The array must stay alive while the record is used."""
    import struct
    fmt = {np.dtype(np.float32): 0, np.dtype(np.float16): 1, np.dtype(np.uint8): 2}[array.dtype]
    if kind == "sampler2D":
        h, w, c = array.shape
        return struct.pack("<Q6i", array.ctypes.data, w, h, c, fmt, 1 if linear else 0, 0)
    d, h, w, c = array.shape
    return struct.pack("<Q6i", array.ctypes.data, w, h, d, c, fmt, 1 if linear else 0)


def pack_uniforms(cpp, calls, textures=None, params=None):
    """Uniform block bytes for the recorded shader.uniform* calls ({name: (type, values)}) and
    the bound textures ({name: (array, linear)}; the arrays must be contiguous and stay alive).
    Renderer uniforms the scene reads without declaring take their values from `params` (the
    job's SnellyParams), as snelly_render does."""
    layout, size = uniform_layout(cpp)
    from_params = renderer_uniforms(cpp) if params is not None else set()
    buf = bytearray(size)
    for name, typ, off, alen in layout:
        if typ in ("sampler2D", "sampler3D"):
            if textures and name in textures:
                arr, linear = textures[name]
                buf[off:off + 32] = sampler_record(typ, arr, linear)
            continue
        if name in from_params:
            v = getattr(params, name)
            vals = list(v) if hasattr(v, "__len__") else [v]
        elif name not in calls:
            continue
        else:
            _, vals = calls[name]
        if typ in ("int",):
            buf[off:off + 4 * len(vals)] = np.asarray(vals, np.int32).tobytes()
        else:
            buf[off:off + 4 * len(vals)] = np.asarray(vals, np.float32).tobytes()
    return bytes(buf)


class OracleLib:
    """A compiled oracle for one scene string and one set of compile-time options."""

    def __init__(self, glsl, opts, count_ops=False):
        self.count_ops = count_ops
        full, defs = assemble(glsl, opts)
        cpp = _translate(full)
        self.cpp = cpp
        key = hashlib.sha1((defs + cpp + str(count_ops)).encode() + self._sources_digest()).hexdigest()[:16]
        d = os.path.join(BUILD, key)
        so = os.path.join(d, "liboracle.so")
        if not os.path.exists(so):
            os.makedirs(d, exist_ok=True)
            with open(os.path.join(d, "scene.inc"), "w") as f:
                f.write(defs + cpp)
            cmd = ["g++", "-O3", "-march=native", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-std=c++17",
                   "-shared", "-fPIC", "-w", "-I" + os.path.join(ROOT, "snelly_b200", "csrc"),
                   "-I" + os.path.join(ROOT, "include"), "-I" + HERE, "-I" + d, '-DSCENE_INC="scene.inc"']
            if count_ops:
                cmd.append("-DORACLE_COUNT_OPS")
            cmd += [os.path.join(HERE, "oracle_main.cpp"), "-o", so + ".tmp"]
            subprocess.run(cmd, check=True)
            os.replace(so + ".tmp", so)
        self.path = so
        L = ctypes.CDLL(so)
        vp, i32 = ctypes.c_void_p, ctypes.c_int
        L.oracle_render.argtypes = [vp, vp, i32, i32, vp, i32, i32, vp, vp, vp, i32]
        L.oracle_render.restype = i32
        L.oracle_firsthit.argtypes = [vp, vp, i32, i32, i32, vp, i32, i32, vp, vp, vp, i32]
        L.oracle_firsthit.restype = i32
        L.oracle_tonemap.argtypes = [vp, i32, vp, vp]
        L.oracle_tonemap.restype = i32
        L.oracle_seed.argtypes = [ctypes.c_uint64, ctypes.c_uint64, vp]
        L.oracle_rand.argtypes = [vp]
        L.oracle_rand.restype = ctypes.c_float
        L.oracle_uniform_block_size.restype = ctypes.c_size_t
        L.oracle_counts.argtypes = [vp, vp]
        L.oracle_last_team.restype = i32
        self.lib = L

    def counts(self):
        """(FP32 ops, special-function ops) tallied on this thread since the last call."""
        a, b = ctypes.c_uint64(), ctypes.c_uint64()
        self.lib.oracle_counts(ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    @staticmethod
    def _sources_digest():
        h = hashlib.sha1()
        try:  # builds use -march=native: key them by the host CPU as well
            flags = [l for l in open("/proc/cpuinfo") if l.startswith(("flags", "model name"))][:2]
            h.update("".join(flags).encode())
        except OSError:
            pass
        for f in ("pt_oracle.h", "pt_oracle_bsdf.inc", "pt_oracle_integrator.inc", "fh_oracle.inc", "ps_oracle.inc",
                  "tm_oracle.h", "oracle_main.cpp", "counted.h"):
            p = os.path.join(HERE, f)
            if os.path.exists(p):
                h.update(open(p, "rb").read())
        for p in (os.path.join(ROOT, "snelly_b200", "csrc", "glslcompat.h"), os.path.join(ROOT, "include", "snelly_params.h")):
            h.update(open(p, "rb").read())
        return h.digest()

    def seed(self, seed, pixels):
        out = np.empty((len(pixels), 4), np.uint32)
        for k, p in enumerate(pixels):
            self.lib.oracle_seed(seed, int(p), out[k].ctypes.data)
        return out

    def last_team(self):
        """Threads the last render / firsthit call ran on."""
        return int(self.lib.oracle_last_team())

    def render(self, params, uniforms, width, height, pixels, frames, rng, threads=0):
        """Render `frames` frames of the listed pixels. Returns (xyz_sum float64 (n,3),
        running mean float32 (n,4), final rng (n,4))."""
        pixels = np.ascontiguousarray(pixels, np.int32)
        n = len(pixels)
        rng = np.ascontiguousarray(rng, np.uint32).copy()
        xyz = np.zeros((n, 3), np.float64)
        mean = np.zeros((n, 4), np.float32)
        ub = ctypes.create_string_buffer(bytes(uniforms), max(1, len(uniforms)))
        rc = self.lib.oracle_render(ctypes.byref(params), ub, int(width), int(height), pixels.ctypes.data, n,
                                    int(frames), rng.ctypes.data, xyz.ctypes.data, mean.ctypes.data, int(threads))
        assert rc == 0
        return xyz, mean, rng

    def firsthit(self, mode, params, uniforms, width, height, pixels, frames, rng=None, threads=0):
        """The other programs: mode 1 normals, 2 ambient occlusion, 4 the simplified path tracer
        (returns xyz_sum, running mean, final rng as render() does), 3 pick (returns (n, 2)
        distance and material at the pixel centres)."""
        pixels = np.ascontiguousarray(pixels, np.int32)
        n = len(pixels)
        rng = np.ascontiguousarray(rng if rng is not None else np.ones((n, 4)), np.uint32).copy()
        xyz = np.zeros((n, 3), np.float64)
        mean = np.zeros((n, 4), np.float32)
        ub = ctypes.create_string_buffer(bytes(uniforms), max(1, len(uniforms)))
        rc = self.lib.oracle_firsthit(ctypes.byref(params), ub, int(mode), int(width), int(height), pixels.ctypes.data,
                                      n, int(frames), rng.ctypes.data, xyz.ctypes.data, mean.ctypes.data, int(threads))
        assert rc == 0
        if mode == 3:
            return mean[:, :2].copy()
        return xyz, mean, rng

    def tonemap(self, xyzn, params):
        """Display transform of (n, 4) mean XYZ pixels; params = (exposure, invGamma, contrast,
        saturation, hueShift) as the shader receives them. Returns (n, 4) RGBA floats."""
        a = np.ascontiguousarray(xyzn, np.float32).reshape(-1, 4)
        out = np.zeros_like(a)
        p = np.asarray(params, np.float32)
        assert self.lib.oracle_tonemap(a.ctypes.data, len(a), p.ctypes.data, out.ctypes.data) == 0
        return out


_RNG_MODULI = np.array([4194287, 4194277, 4194191, 4194167], np.uint64)


def seed_pixels(seed, pixels):
    """The per-pixel RNG seeding of the CUDA path tracer (oracle_seed, restated in numpy so that
    a process can seed without loading any compiled library): lane k of pixel i is
    1 + (z_k mod (m_k - 1)) for successive SplitMix64 outputs z_k of the stream keyed by
    splitmix64(seed) ^ i. Returns (n, 4) uint32."""
    M = (1 << 64) - 1

    def nxt(s):
        s = (s + 0x9E3779B97F4A7C15) & M
        z = s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        return s, z ^ (z >> 31)

    _, k0 = nxt(int(seed) & M)
    with np.errstate(over="ignore"):
        key = np.uint64(k0) ^ np.asarray(pixels, np.uint64)
        out = np.empty((len(key), 4), np.uint32)
        for lane in range(4):
            key = key + np.uint64(0x9E3779B97F4A7C15)
            z = key.copy()
            z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
            z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
            z = z ^ (z >> np.uint64(31))
            out[:, lane] = (np.uint64(1) + z % (_RNG_MODULI[lane] - np.uint64(1))).astype(np.uint32)
    return out


def host_params(snelly):
    """SnellyParams of a host-mirror Snelly object with host table pointers filled in for the
    oracle: the XYZ table and the inverse CDF of the loaded spectrum (restated here)."""
    from snelly_b200 import api
    p = snelly.uniform_params()
    xyz = np.asarray(api.DATA["xyz_table"], np.float32)
    sp = snelly.spectrumObj
    if isinstance(sp, api.FlatSpectrum):
        icdf = inverse_cdf("flat", band=(sp.min, sp.max))
    elif isinstance(sp, api.MonochromaticSpectrum):
        icdf = inverse_cdf("mono", wavelength=sp.wavelength)
    else:
        icdf = inverse_cdf("blackbody", temperature=sp.skyTemperature)
    env = snelly.env_map()
    keep = (xyz, icdf, env)
    p.xyzTable = xyz.ctypes.data
    p.icdfTable = icdf.ctypes.data
    if env is not None:  # as snelly_render binds desc.env_map
        p.envMap = env.ctypes.data
        p.envMapH, p.envMapW = int(env.shape[0]), int(env.shape[1])
        p.haveEnvMap = 1
    return p, keep


def flops_per_path(snelly, pixels=2000, frames=2, seed=5):
    """Algorithmic FP32 operations per path sample of a workload, counted by the oracle's
    counting build on a fixed random subset of its pixels (single thread). Returns
    (flops per path sample, special ops per path sample, samples counted)."""
    lib = OracleLib(snelly.sceneObj.shader(), snelly.scene_opts(), count_ops=True)
    n = snelly.width * snelly.height
    pix = np.sort(np.random.RandomState(seed).choice(n, min(pixels, n), replace=False))
    p, keep = host_params(snelly)
    sh = snelly.scene_shader()
    ub = pack_uniforms(lib.cpp, sh.calls, sh.textures, params=p)
    lib.counts()
    lib.render(p, ub, snelly.width, snelly.height, pix, frames, lib.seed(snelly.seed, pix), threads=1)
    f, sp = lib.counts()
    samples = len(pix) * frames * snelly.scene_opts().max_samples_per_frame
    return f / samples, sp / samples, samples
