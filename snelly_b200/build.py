"""Build libsnelly.so (host runtime + ahead-of-time sm_100a kernels) in place.

The scene-dependent kernels (csrc/kernels/*.cu[h]) are compiled at run time by NVRTC for
sm_100a, one module per scene; this step compiles the C ABI runtime, the GLSL translator and the
scene-independent kernels with nvcc for sm_100a into snelly_b200/libsnelly.so.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
SOURCES = ["runtime.cpp", "glsl_transform.cpp", "wavefront.cpp", "aot_kernels.cu", "tonemap.cu", "png_unfilter.cpp"]
OUT = os.path.join(HERE, "libsnelly.so")


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    csrc = os.path.join(HERE, "csrc")
    for dp, _, fs in os.walk(csrc):
        for f in fs:
            if os.path.getmtime(os.path.join(dp, f)) > t:
                return True
    for f in os.listdir(os.path.join(ROOT, "include")):
        if os.path.getmtime(os.path.join(ROOT, "include", f)) > t:
            return True
    return False


def build(force=False, verbose=False):
    if not force and not needs_build():
        return OUT
    csrc = os.path.join(HERE, "csrc")
    # --fmad=false: the ahead-of-time kernels restate reference formulas operation by operation
    # (the tonemapper) or check arithmetic against IEEE results (the self-tests)
    cmd = [os.path.join(CUDA, "bin", "nvcc"), "-shared", "-Xcompiler", "-fPIC", "-O2", "-std=c++17",
           "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "--fmad=false",
           "-I" + csrc, "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(CUDA, "include"),
           "-o", OUT + ".tmp"]
    cmd += [os.path.join(csrc, s) for s in SOURCES]
    cmd += ["-L" + os.path.join(CUDA, "lib64"),
            "-lnvrtc", "-lcudart", "-Xlinker", "-rpath=" + os.path.join(CUDA, "lib64")]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)


def _compile_one(item):
    glsl, opts_bytes = item
    from snelly_b200 import _native as N
    opts = N.SceneOpts.from_buffer_copy(opts_bytes)
    N.compile_check(glsl, opts)
    return True


def prebuild_modules(hosts, math_modes=(0, 1), workers=None):
    """NVRTC-compile the scene modules of `hosts` (host-mirror Snelly objects) for sm_100a in each
    math mode (0 fast, 1 IEEE-strict), in parallel, into the in-tree module cache
    (snelly_b200/_build/kcache), where a context on a GPU machine finds them instead of compiling.
    Returns the number of distinct modules."""
    import concurrent.futures as cf
    import multiprocessing as mp
    items = {}
    for h in hosts:
        glsl = h.sceneObj.shader()
        for mm in math_modes:
            o = h.scene_opts()
            o.math_mode = mm
            o.kernel_mode = 0
            items[(glsl, bytes(o))] = True
    work = list(items)
    prune_module_cache()
    with cf.ProcessPoolExecutor(max_workers=workers or min(8, os.cpu_count() or 1),
                                mp_context=mp.get_context("spawn")) as ex:
        list(ex.map(_compile_one, work))
    return len(work)


CACHE_DIR = os.path.join(HERE, "_build", "kcache")


def module_key_sources():
    """The files whose contents every module's cache key includes (the runtime's module_key): the
    kernel directory, the GLSL compatibility header and its swizzle table, the parameter block."""
    kdir = os.path.join(HERE, "csrc", "kernels")
    files = [os.path.join(kdir, f) for f in os.listdir(kdir) if not f.startswith(".")]
    files += [os.path.join(HERE, "csrc", "glslcompat.h"), os.path.join(HERE, "csrc", "glsl_swizzles.inc"),
              os.path.join(ROOT, "include", "snelly_params.h")]
    return files


def prune_module_cache(cache_dir=CACHE_DIR, sources=None):
    """Delete cached modules compiled before the latest edit of a file their keys include: such a
    module's key covers the file's old contents, so no build asks for it again (unless the edit is
    undone, when it is compiled once more). Without this the cache keeps a full set of modules per
    kernel edit. Returns the number of files deleted."""
    if not os.path.isdir(cache_dir):
        return 0
    newest = max(os.path.getmtime(f) for f in (sources if sources is not None else module_key_sources()))
    deleted = 0
    for f in os.listdir(cache_dir):
        p = os.path.join(cache_dir, f)
        if f.endswith(".cubin") and os.path.getmtime(p) < newest:
            os.remove(p)
            deleted += 1
    return deleted
