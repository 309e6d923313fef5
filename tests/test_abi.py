"""libsnelly's C ABI without a GPU: symbols, struct layouts, device-free compiles, errors."""
import ctypes
import os
import re
import subprocess

import pytest

from snelly_b200 import _native as N
from snelly_b200 import scenes
from snelly_b200.testing import HostSnelly

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            text = open(os.path.join(ROOT, "include", f)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(snelly_\w+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    L = N.lib()
    out = subprocess.run(["nm", "-D", "--defined-only", N.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (snelly_\w+)", out))
    missing = declared_functions() - exported
    assert not missing, missing
    for name in declared_functions():
        assert hasattr(L, name)


def test_struct_layouts_match():
    L = N.lib()
    for which, st in enumerate((N.SnellyParams, N.RenderDesc, N.SceneOpts, N.Uniform, N.Spectrum)):
        assert L.snelly_abi_sizeof(which) == ctypes.sizeof(st)


def test_init_without_gpu_fails_cleanly():
    if os.path.exists("/dev/nvidiactl"):
        pytest.skip("a GPU is present")
    L = N.lib()
    h = ctypes.c_void_p()
    rc = L.snelly_init(ctypes.byref(h), 0, 0)
    assert rc == -6 and not h.value
    assert b"device" in L.snelly_last_error()


def test_null_arguments_rejected():
    L = N.lib()
    assert L.snelly_render(None, 1, None, None) == -1
    assert L.snelly_readback(None, 1, None, 0, 1) == -1
    assert L.snelly_shutdown(None) == -1


@pytest.mark.parametrize("name,math_mode", [(n, N.MATH_FAST) for n in sorted(scenes.SCENES)] + [("c1", N.MATH_STRICT)])
def test_every_scene_compiles_for_sm100a(name, math_mode):
    h = HostSnelly(scenes.SCENES[name]())
    opts = h.scene_opts()
    opts.math_mode = math_mode
    nbytes, log = N.compile_check(h.sceneObj.shader(), opts)
    assert nbytes > 10000


def test_compile_errors_carry_the_log():
    opts = N.SceneOpts(3, 64, 1, 1, 0, 0, 0, 0, 0, 0, 1)
    with pytest.raises(N.SnellyError) as e:
        N.compile_check("float SDF_SURFACE(vec3 X) { return undefined_thing(X); }", opts)
    assert e.value.code == -2 and "undefined_thing" in str(e.value)
    with pytest.raises(N.SnellyError) as e:
        N.compile_check("float nothing(vec3 X) { return 1.0; }", opts)
    assert "SDF_SURFACE" in str(e.value)
