"""ctypes binding of libsnelly.so (include/snelly.h).

The structs mirror the C declarations; SnellyParams is generated from include/snelly_params.h so
the two cannot drift, and every struct size is checked against the library at load time. Any
failure to load the library raises: there is no fallback implementation.
"""
import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "libsnelly.so")

SNELLY_OK = 0
ERRORS = {
    -1: "EINVAL", -2: "ECOMPILE", -3: "ENOMEM_BUDGET", -4: "EBUSY", -5: "ETIMEOUT", -6: "EDEVICE",
    -7: "ENOTFOUND", -8: "ECANCELLED",
}
KERNEL_AUTO, KERNEL_MEGA, KERNEL_WAVEFRONT = 0, 1, 2
MATH_FAST, MATH_STRICT = 0, 1
MODE_PT, MODE_NORMALS, MODE_AO, MODE_PICK, MODE_PTSIMPLE = 0, 1, 2, 3, 4
SPECTRUM_BLACKBODY, SPECTRUM_FLAT, SPECTRUM_MONO = 0, 1, 2
READ_WAIT, READ_POLL, READ_ASYNC = 1, 2, 4
U_FLOAT, U_INT, U_BOOL, U_VEC2, U_VEC3, U_VEC4 = 0, 1, 2, 3, 4, 5
U_IVEC2, U_IVEC3, U_IVEC4, U_MAT2, U_MAT3, U_MAT4, U_SAMPLER2D, U_SAMPLER3D = 6, 7, 8, 9, 10, 11, 12, 13
IOR_MODELS = {"abbe": 0, "sellmeier": 1, "sellmeier2": 2, "polyanskiy": 3, "cauchy": 4}
# snelly_job_wavefront_config's fields, in order (SNELLY_WF_CONFIG_FIELDS of them)
WF_CONFIG_NAMES = ("parts", "shade_split", "drain", "chunk", "grab", "refill", "block", "park_left", "walker",
                   "lane_rays", "overlap", "shade_share", "interleave", "volume_stage")


def header_define(name):
    """The integer value of a #define in include/snelly.h."""
    text = open(os.path.join(ROOT, "include", "snelly.h")).read()
    return int(re.search(r"#define %s (\d+)" % name, text).group(1))


if header_define("SNELLY_WF_CONFIG_FIELDS") != len(WF_CONFIG_NAMES):
    raise ImportError("WF_CONFIG_NAMES does not match SNELLY_WF_CONFIG_FIELDS of include/snelly.h")


class SnellyError(RuntimeError):
    """A libsnelly call returned an error code; .code holds it, the message is the library's."""

    def __init__(self, code, message):
        super().__init__(f"{ERRORS.get(code, code)}: {message}")
        self.code = code


def _params_fields():
    text = open(os.path.join(ROOT, "include", "snelly_params.h")).read()
    defines = {k: int(v) for k, v in re.findall(r"#define (\w+) (\d+)", text)}
    body = re.search(r"typedef struct SnellyParams \{(.*?)\} SnellyParams;", text, re.S).group(1)
    body = re.sub(r"//[^\n]*", "", body)
    types = {"float": ctypes.c_float, "int": ctypes.c_int}
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        if "*" in decl:  # a device pointer (one declarator per line in the header)
            fields.append((re.findall(r"\w+", decl)[-1], ctypes.c_void_p))
            continue
        m = re.match(r"(\w+)\s+(.*)", decl, re.S)
        base, rest = m.group(1), m.group(2)
        for name in rest.split(","):
            name = name.strip()
            is_ptr = False
            am = re.match(r"(\w+)\[(\w+)\]", name)
            if is_ptr:
                t = ctypes.c_void_p
            else:
                t = types[base]
            if am:
                n = am.group(2)
                n = defines[n] if n in defines else int(n)
                fields.append((am.group(1), t * n))
            else:
                fields.append((name, t))
    return fields


class SnellyParams(ctypes.Structure):
    _fields_ = _params_fields()


class SceneOpts(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in (
        "max_bounces", "max_march_steps", "max_atmosphere_scatters", "max_samples_per_frame", "dispersive",
        "interactive", "has_atmosphere", "has_fog", "has_sphere_light", "math_mode", "kernel_mode")]


class Spectrum(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("temperature", ctypes.c_float), ("band_min", ctypes.c_float),
                ("band_max", ctypes.c_float), ("wavelength", ctypes.c_float)]


class TonemapParams(ctypes.Structure):
    """snelly_tonemap_params: the tonemapper shader's uniforms."""
    _fields_ = [(n, ctypes.c_float) for n in ("exposure", "invGamma", "contrast", "saturation", "hueShift")]


TONEMAP_RGBA8, TONEMAP_RGBA32F = 0, 1


class RenderDesc(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int), ("height", ctypes.c_int), ("frames", ctypes.c_int), ("mode", ctypes.c_int),
                ("seed", ctypes.c_uint64), ("params", SnellyParams), ("spectrum", Spectrum),
                ("env_map", ctypes.c_void_p), ("env_w", ctypes.c_int), ("env_h", ctypes.c_int),
                ("accum_fp64", ctypes.c_int), ("reserved", ctypes.c_int)]


class Uniform(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char_p), ("type", ctypes.c_int), ("count", ctypes.c_int),
                ("f", ctypes.POINTER(ctypes.c_float)), ("i", ctypes.POINTER(ctypes.c_int))]


_lib = None


def lib():
    """Load libsnelly.so (in-tree) and declare its signatures. Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m snelly_b200.build` "
                          "(or __graft_entry__.build())")
    L = ctypes.CDLL(LIB_PATH)
    P, vp, i32, u64, sz = ctypes.POINTER, ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64, ctypes.c_size_t
    sig = {
        "snelly_init": (i32, [P(vp), i32, sz]),
        "snelly_shutdown": (i32, [vp]),
        "snelly_last_error": (ctypes.c_char_p, []),
        "snelly_version": (ctypes.c_char_p, []),
        "snelly_create_scene": (i32, [vp, ctypes.c_char_p, P(SceneOpts), P(u64), ctypes.c_char_p, sz]),
        "snelly_destroy_scene": (i32, [vp, u64]),
        "snelly_set_uniforms": (i32, [vp, u64, P(Uniform), sz]),
        "snelly_set_texture": (i32, [vp, u64, ctypes.c_char_p, vp, i32, i32, i32, i32, i32, i32]),
        "snelly_render": (i32, [vp, u64, P(RenderDesc), P(u64)]),
        "snelly_advance": (i32, [vp, u64, i32]),
        "snelly_update_job": (i32, [vp, u64, P(RenderDesc)]),
        "snelly_advance_batch": (i32, [vp, P(u64), P(i32), sz]),
        "snelly_readback": (i32, [vp, u64, vp, sz, i32]),
        "snelly_readback_state": (i32, [vp, u64, vp, vp, vp, vp]),
        "snelly_selftest": (i32, [vp, i32, P(u64)]),
        "snelly_png_unfilter": (i32, [vp, sz, i32, i32, i32, vp]),
        "snelly_job_kernel": (i32, [vp, u64, P(i32)]),
        "snelly_job_wavefront_config": (i32, [vp, u64, P(i32)]),
        "snelly_image_stats_static": (i32, [vp, u64, P(ctypes.c_double)]),
        "snelly_tonemap": (i32, [vp, u64, P(TonemapParams), vp, sz, i32]),
        "snelly_pick": (i32, [vp, u64, P(RenderDesc), ctypes.c_float, ctypes.c_float, P(ctypes.c_float),
                              P(ctypes.c_float)]),
        "snelly_restore": (i32, [vp, u64, P(RenderDesc), vp, vp, vp, P(u64)]),
        "snelly_job_status": (i32, [vp, u64, P(i32), P(i32)]),
        "snelly_cancel": (i32, [vp, u64]),
        "snelly_destroy_job": (i32, [vp, u64]),
        "snelly_sync": (i32, [vp]),
        "snelly_stream": (vp, [vp]),
        "snelly_launch_count": (u64, [vp]),
        "snelly_measure_fp32_peak": (i32, [vp, P(ctypes.c_double), P(ctypes.c_double)]),
        "snelly_flush_l2": (i32, [vp, sz]),
        "snelly_image_stats": (i32, [vp, u64, vp]),
        "snelly_abi_sizeof": (sz, [i32]),
        "snelly_inverse_cdf": (i32, [P(Spectrum), vp]),
        "snelly_compile_check": (i32, [ctypes.c_char_p, P(SceneOpts), ctypes.c_char_p, sz, P(sz)]),
        "snelly_glsl_to_cpp": (i32, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, sz]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    for which, st in enumerate((SnellyParams, RenderDesc, SceneOpts, Uniform, Spectrum)):
        got = L.snelly_abi_sizeof(which)
        if got != ctypes.sizeof(st):
            raise ImportError(f"ABI mismatch for {st.__name__}: library {got} bytes, binding {ctypes.sizeof(st)}")
    _lib = L
    return L


def check(rc):
    if rc != SNELLY_OK:
        raise SnellyError(rc, lib().snelly_last_error().decode(errors="replace"))
    return rc


def glsl_to_cpp(glsl, struct_name="Scene", extra_members=None):
    """C++ text of a GLSL scene string (the translation snelly_create_scene compiles)."""
    cap = 16 * len(glsl) + (1 << 16)
    buf = ctypes.create_string_buffer(cap)
    extra = extra_members.encode() if extra_members is not None else None
    check(lib().snelly_glsl_to_cpp(glsl.encode(), struct_name.encode(), extra, buf, cap))
    return buf.value.decode()


def compile_check(glsl, opts):
    """NVRTC-compile a scene for sm_100a without a GPU; returns (cubin bytes, log)."""
    log = ctypes.create_string_buffer(1 << 16)
    n = ctypes.c_size_t()
    rc = lib().snelly_compile_check(glsl.encode(), ctypes.byref(opts), log, len(log), ctypes.byref(n))
    if rc != SNELLY_OK:
        raise SnellyError(rc, log.value.decode(errors="replace"))
    return n.value, log.value.decode(errors="replace")
