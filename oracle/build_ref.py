"""Build the reference's own fragment shaders as CPU libraries: oracle/_ref/<key>/libref.so.

TEST INFRASTRUCTURE (the recipe for the reference build). Reads
shaders/pathtracer-fragment-shader.glsl (or the normals, ao or pick program) from a checkout of
the reference, applies the same
source substitutions the reference host applies before compiling it (Renderer.compileShaders,
js/renderer.js:217-316, via GLU.applyShaderReplacements, js/gl.js:157-168), including the
__IOR_FUNC__ code that the material objects generate (the JS string builders of
js/materials.js:640-657, 842-861, 905-930, 956-981, 1014-1034, 1064-1089, restated below),
translates the GLSL to C++ with the package's translator and compiles it with g++ against
glslcompat.h and oracle/ref_harness.cpp. Nothing of the reference is copied into the repository:
outputs go to oracle/_ref/ only (git-ignored), and they travel to GPU machines as built files.

The harness runs the shader's main() once per pixel and frame, binding the Radiance and RngData
textures to that pixel's state (NEAREST) and the tables to LINEAR textures:
WavelengthToXYZ (1024 texels), ICDF (4096), iorTex and kTex (64 each; the reference host binds
the k table to a uniform named "k_tex", js/materials.js:665, so kTex is in fact unbound there;
the harness binds it to the k table, the intended behaviour).
"""
import ctypes
import hashlib
import os
import re
import struct
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF_ROOT = os.environ.get("SNELLY_REFERENCE", "")  # the reference checkout; unset: prebuilt libraries only


def have_reference():
    """True when $SNELLY_REFERENCE names a checkout of the reference (its shaders/ folder)."""
    return bool(REF_ROOT) and os.path.isdir(os.path.join(REF_ROOT, "shaders"))
OUT = os.path.join(HERE, "_ref")
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)
import oracle as O  # noqa: E402


def ior_glsl(model, ncoeffs):
    """The IOR_DIELE GLSL a Dielectric object's ior() returns, and the metal's IOR_METAL/K_METAL."""
    if model == "abbe":
        return """
uniform float _iorVal;
uniform float _abbe;
float IOR_DIELE(float wavelength_nm)
{
    if (_abbe <= 0.0)
        return _iorVal;
    float nD2 = 0.5893; nD2 *= nD2;
    float nF2 = 0.4861; nF2 *= nF2;
    float nC2 = 0.6563; nC2 *= nC2;
    float cauchyC = (_iorVal - 1.0)/_abbe * (nC2*nF2)/(nC2 - nF2);
    float cauchyB = _iorVal - cauchyC/nD2;
    float wavelength_um = 1.0e-3*wavelength_nm;
    float l = wavelength_um;
    return cauchyB + cauchyC/(l*l);
}
"""
    uniforms = "".join(f"uniform float _C{n};\n" for n in range(1, ncoeffs + 1))
    terms = (ncoeffs - 1) // 2
    if model in ("sellmeier", "sellmeier2"):
        f = "1.0 + _C1 "
        for t in range(1, terms + 1):
            pole = f"_C{2 * t + 1}*_C{2 * t + 1}" if model == "sellmeier" else f"_C{2 * t + 1}"
            f += f"+ _C{2 * t}*l2/(l2 - {pole})"
        return uniforms + f"""
float IOR_DIELE(float wavelength_nm)
{{
    float wavelength_um = 1.0e-3*wavelength_nm;
    float l2 = wavelength_um*wavelength_um;
    float n2 = {f};
    return max(sqrt(abs(n2)), 1.0e-3);
}}"""
    if model == "polyanskiy":
        return """
uniform float _C1;
uniform float _C2;
uniform float _C3;
uniform float _C4;
uniform float _C5;
float IOR_DIELE(float wavelength_nm)
{
    float wavelength_um = 1.0e-3*wavelength_nm;
    float l = wavelength_um;
    float n2 = _C1 + _C2*pow(l, _C3)/(l*l - pow(_C4, _C5));
    return max(sqrt(abs(n2)), 1.0e-3);
}"""
    f = "_C1"
    for t in range(1, terms + 1):
        f += f" + _C{2 * t}*pow(l, _C{2 * t + 1})"
    return uniforms + f"""
float IOR_DIELE(float wavelength_nm)
{{
    float wavelength_um = 1.0e-3*wavelength_nm;
    float l = wavelength_um;
    float n = {f};
    return max(n, 1.0e-3);
}}"""


METAL_GLSL = """
float IOR_METAL(float wavelength_nm)
{
    float u = (wavelength_nm - 390.0) * 0.002777777777777778;
    return texture(iorTex, vec2(u, 0.5)).r;
}
float K_METAL(float wavelength_nm)
{
    float u = (wavelength_nm - 390.0) * 0.002777777777777778;
    return texture(kTex, vec2(u, 0.5)).r;
}
"""

MODEL_NAMES = {0: "abbe", 1: "sellmeier", 2: "sellmeier2", 3: "polyanskiy", 4: "cauchy"}


PROGRAMS = ("pathtracer", "normals", "ao", "pick", "tonemapper", "simplepathtracer")


def shader_source(scene_glsl, opts, diele_model, ncoeffs, program="pathtracer"):
    """The fragment shader of `program` with the host's substitutions applied (the same set for
    every program, js/renderer.js:287-316; the tonemapper gets none, js/renderer.js:358)."""
    assert program in PROGRAMS
    src = open(os.path.join(REF_ROOT, "shaders", f"{program}-fragment-shader.glsl")).read()
    if program == "tonemapper":
        return src
    full, defs = O.assemble(scene_glsl, opts)
    # the reference host's #define block, without the loop bounds (those are substituted)
    defines = "\n".join(l for l in defs.splitlines() if not l.startswith("#define MAX_"))
    reps = {
        "__SHADER__": full,
        "__IOR_FUNC__": ior_glsl(MODEL_NAMES[diele_model], ncoeffs) + "\n" + METAL_GLSL,
        "__MAX_MARCH_STEPS__": str(opts.max_march_steps),
        "__MAX_BOUNCES__": str(opts.max_bounces),
        "__MAX_ATMOSPHERE_SCATTERS__": str(opts.max_atmosphere_scatters),
        "__MAX_SAMPLES_PER_FRAME__": str(opts.max_samples_per_frame),
        "__DEFINES__": "\n" + defines + "\n",
    }
    for k, v in reps.items():
        src = re.sub(k, lambda m: v, src)
    return src


def workload_key(scene_glsl, opts, diele_model, ncoeffs, program="pathtracer"):
    """Identity of a reference build: scene source + compile-time options + dielectric model
    (+ the program, for the first-hit programs)."""
    tag = "" if program == "pathtracer" else "/" + program
    return hashlib.sha1((scene_glsl + repr(bytes(opts)) + f"{diele_model}/{ncoeffs}{tag}").encode()).hexdigest()[:16]


class RefLib:
    """The reference shader for one scene + options, compiled for the CPU."""

    def __init__(self, scene_glsl, opts, diele_model, ncoeffs, name=None, program="pathtracer"):
        """Build (needs the reference checkout) into oracle/_ref/<hash>, or, with `name`, into
        oracle/_ref/<name> together with a key file so that load() finds it without the reference.
        `program`: the fragment shader to build (pathtracer, normals, ao or pick)."""
        from snelly_b200 import _native
        self.program = program
        src = shader_source(scene_glsl, opts, diele_model, ncoeffs, program)
        cpp = _native.glsl_to_cpp(src, "RefShader", "  vec4 gl_FragCoord;\n")
        self.cpp = cpp
        h = hashlib.sha1(cpp.encode() + program.encode())
        for f in (os.path.join(HERE, "ref_harness.cpp"), os.path.join(ROOT, "snelly_b200", "csrc", "glslcompat.h")):
            h.update(open(f, "rb").read())
        d = os.path.join(OUT, name if name else h.hexdigest()[:16])
        so = os.path.join(d, "libref.so")
        stamp = os.path.join(d, "build.sha1")
        if name and (not os.path.exists(stamp) or open(stamp).read() != h.hexdigest()):
            if os.path.exists(so):
                os.remove(so)
        if not os.path.exists(so):
            os.makedirs(d, exist_ok=True)
            with open(os.path.join(d, "ref_shader.inc"), "w") as f:
                f.write(cpp)
            # portable AVX2 target: the library may run on another machine's host CPU
            cmd = ["g++", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-std=c++17",
                   "-shared", "-fPIC", "-w", "-I" + os.path.join(ROOT, "snelly_b200", "csrc"), "-I" + d,
                   os.path.join(HERE, "ref_harness.cpp"), "-o", so + ".tmp"]
            if program == "pick":
                cmd.insert(1, "-DREF_PICK")
            elif program == "tonemapper":
                cmd.insert(1, "-DREF_TONEMAP")
            subprocess.run(cmd, check=True)
            os.replace(so + ".tmp", so)
            with open(stamp, "w") as f:
                f.write(h.hexdigest())
            with open(os.path.join(d, "workload.key"), "w") as f:
                f.write(workload_key(scene_glsl, opts, diele_model, ncoeffs, program))
        self._load(so, cpp)

    @classmethod
    def load(cls, name, scene_glsl, opts, diele_model, ncoeffs, program="pathtracer"):
        """A named prebuilt reference library (no reference checkout needed), or None if absent or
        built for another workload."""
        d = os.path.join(OUT, name)
        so, inc, keyf = (os.path.join(d, f) for f in ("libref.so", "ref_shader.inc", "workload.key"))
        if not (os.path.exists(so) and os.path.exists(inc) and os.path.exists(keyf)):
            return None
        if open(keyf).read() != workload_key(scene_glsl, opts, diele_model, ncoeffs, program):
            return None
        self = cls.__new__(cls)
        self.program = program
        self.cpp = open(inc).read()
        self._load(so, self.cpp)
        return self

    def _load(self, so, cpp):
        self.path = so
        L = ctypes.CDLL(so)
        vp, i32, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t
        if self.program == "pick":
            L.ref_pick.argtypes = [vp, sz, sz, i32, vp, i32, vp, i32]
            L.ref_pick.restype = i32
        elif self.program == "tonemapper":
            L.ref_tonemap.argtypes = [vp, sz, sz, vp, i32, vp]
            L.ref_tonemap.restype = i32
        else:
            L.ref_render.argtypes = [vp, sz, sz, sz, i32, i32, vp, i32, i32, vp, vp, i32]
            L.ref_render.restype = i32
        L.ref_block_size.restype = sz
        L.ref_last_team.restype = i32
        self.lib = L
        self.layout, self.size = self._layout(cpp)

    @staticmethod
    def _layout(cpp):
        body = re.search(r"struct RefShaderUniforms \{(.*?)\};", cpp, re.S).group(1)
        lay = {}
        for m in re.finditer(r"(\w+) (\w+)(?:\[(\d+)\])?;\s*// offset (\d+)", body):
            lay[m.group(2)] = (m.group(1), int(m.group(4)), int(m.group(3) or 0))
        size = int(re.search(r"sizeof\(RefShaderUniforms\) == (\d+)", cpp).group(1))
        return lay, size

    def block(self, params, scene_calls, tables, scene_textures=None):
        """Uniform block bytes: shader uniforms from SnellyParams fields of the same names, IOR
        coefficients, samplers bound to the host tables, scene uniforms from syncShader calls."""
        buf = bytearray(self.size)
        for name, (typ, off, alen) in self.layout.items():
            if typ in ("sampler2D", "sampler3D"):
                continue
            vals = None
            if name in scene_calls:
                vals = scene_calls[name][1]
            elif hasattr(params, name):
                v = getattr(params, name)
                vals = list(v) if hasattr(v, "__len__") else [v]
            elif re.fullmatch(r"_C\d+", name):
                vals = [params.dieleCoeffs[int(name[2:]) - 1]]
            elif name == "_iorVal":
                vals = [params.dieleCoeffs[0]]
            elif name == "_abbe":
                vals = [params.dieleCoeffs[1]]
            if vals is None:
                continue
            dt = np.int32 if typ == "int" else np.float32
            b = np.asarray(vals, dt).tobytes()
            buf[off:off + len(b)] = b
        for name, rec in tables.items():
            ptr, w, h, ch, linear = rec[:5]
            fmt, srgb = rec[5:7] if len(rec) > 5 else (0, 0)
            if name in self.layout:
                off = self.layout[name][1]
                buf[off:off + 32] = struct.pack("<Q6i", ptr, w, h, ch, fmt, linear, srgb)
        for name, (arr, linear) in (scene_textures or {}).items():
            if name in self.layout:
                off = self.layout[name][1]
                buf[off:off + 32] = O.sampler_record(self.layout[name][0], arr, linear)
        return bytes(buf)

    def last_team(self):
        """Threads the last render / pick call ran on."""
        return int(self.lib.ref_last_team())

    def pick(self, params, scene_calls, tables, width, pixels, threads=0, scene_textures=None):
        """The pick program at the centre of each listed pixel: (n, 2) distance and material."""
        pixels = np.ascontiguousarray(pixels, np.int32)
        out = np.zeros((len(pixels), 4), np.float32)
        blk = self.block(params, scene_calls, tables, scene_textures)
        ub = ctypes.create_string_buffer(blk, len(blk))
        rc = self.lib.ref_pick(ub, len(blk), self.layout["mousePick"][1], int(width), pixels.ctypes.data, len(pixels),
                               out.ctypes.data, int(threads))
        assert rc == 0
        return out[:, :2].copy()

    def tonemap(self, xyzn, uniforms):
        """The tonemapper program on (n, 4) radiance texels with the given shader uniforms
        {exposure, invGamma, contrast, saturation, hueShift}: (n, 4) output colours."""
        a = np.ascontiguousarray(xyzn, np.float32).reshape(-1, 4)
        out = np.zeros_like(a)
        buf = bytearray(self.size)
        for name, val in uniforms.items():
            off = self.layout[name][1]
            buf[off:off + 4] = np.float32(val).tobytes()
        blk = bytes(buf)
        ub = ctypes.create_string_buffer(blk, len(blk))
        rc = self.lib.ref_tonemap(ub, len(blk), self.layout["Radiance"][1], a.ctypes.data, len(a), out.ctypes.data)
        assert rc == 0
        return out

    def render(self, params, scene_calls, tables, width, height, pixels, frames, rng, threads=0, scene_textures=None):
        pixels = np.ascontiguousarray(pixels, np.int32)
        n = len(pixels)
        rng = np.ascontiguousarray(rng, np.uint32).copy()
        mean = np.zeros((n, 4), np.float32)
        blk = self.block(params, scene_calls, tables, scene_textures)
        ub = ctypes.create_string_buffer(blk, len(blk))
        rc = self.lib.ref_render(ub, len(blk), self.layout["Radiance"][1], self.layout["RngData"][1], int(width),
                                 int(height), pixels.ctypes.data, n, int(frames), rng.ctypes.data, mean.ctypes.data,
                                 int(threads))
        assert rc == 0
        return mean, rng


def tonemapper_lib():
    """The reference's tonemapper program built for the CPU (scene-independent)."""
    from snelly_b200 import _native
    opts = _native.SceneOpts()
    return RefLib("", opts, 0, 0, name="tonemapper", program="tonemapper")


def ref_for(snelly, name=None, prebuilt_only=False, program="pathtracer"):
    """RefLib + table bindings for a host-mirror Snelly object. With `name`, use (or create) the
    named build in oracle/_ref/<name>; prebuilt_only: never build (returns None if absent);
    program: which fragment shader (pathtracer, normals, ao, pick)."""
    p, keep = O.host_params(snelly)
    xyz, icdf, env = keep
    metal_n = np.asarray(list(p.metalN), np.float32)
    metal_k = np.asarray(list(p.metalK), np.float32)
    tables = {
        "WavelengthToXYZ": (xyz.ctypes.data, 1024, 1, 4, 1),
        "ICDF": (icdf.ctypes.data, 4096, 1, 1, 1),
        "iorTex": (metal_n.ctypes.data, 64, 1, 1, 1),
        "kTex": (metal_k.ctypes.data, 64, 1, 1, 1),
    }
    if env is not None:  # SRGB8 RGB, LINEAR (GLU.loadImageAndCreateTextureInfo, js/gl.js:532-559)
        tables["envMap"] = (env.ctypes.data, env.shape[1], env.shape[0], 3, 1, 2, 1)
    args = (snelly.sceneObj.shader(), snelly.scene_opts(), p.dieleModel, p.dieleNumCoeffs)
    lib = RefLib.load(name, *args, program=program) if name else None
    if lib is None:
        if prebuilt_only or not have_reference():
            return None
        lib = RefLib(*args, name=name, program=program)
    return lib, p, tables, (xyz, icdf, metal_n, metal_k, env)


if __name__ == "__main__":
    print("usage: import build_ref; build_ref.ref_for(snelly)")
