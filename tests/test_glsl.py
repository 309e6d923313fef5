"""The GLSL-to-C++ translator and the GLSL compat header (host build)."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from snelly_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_cpp(scene_glsl, body):
    """Translate `scene_glsl`, compile it with a main() running `body`, return stdout."""
    cpp = N.glsl_to_cpp(scene_glsl)
    src = ('#include "glslcompat.h"\n#include <cstdio>\nnamespace glsl {\n' + cpp +
           '\n}\nusing namespace glsl;\nint main() {\n' + body + '\n return 0; }\n')
    with tempfile.TemporaryDirectory() as d:
        f = os.path.join(d, "t.cpp")
        open(f, "w").write(src)
        subprocess.run(["g++", "-std=c++17", "-O1", "-w", "-I" + os.path.join(ROOT, "snelly_b200", "csrc"), f, "-o",
                        os.path.join(d, "t")], check=True)
        return subprocess.run([os.path.join(d, "t")], capture_output=True, text=True, check=True).stdout


def test_translation_rules():
    cpp = N.glsl_to_cpp("""
precision highp float;
uniform float R; uniform vec3 C[2]; uniform bool flag; uniform sampler3D tex;
float helper(vec3 p);
float g[3] = float[3](1.0, 2.0, 3.0);
float SDF_SURFACE(in vec3 X) { float a; return helper(X) + 1e-3 + .5; }
float helper(vec3 p) { return length(p) - R; }
void setv(out vec3 v, inout float w) { v = vec3(1.0); w += 2.0; }
""")
    assert "1e-3f" in cpp and ".5f" in cpp and "1.0f" in cpp
    assert "gfloat a{}" in cpp
    assert "vec3& v, gfloat& w" in cpp
    assert "gfloat helper(vec3 p);" not in cpp  # prototype dropped
    assert "{1.0f, 2.0f, 3.0f}" in cpp
    assert "const gfloat& R;" in cpp and "const vec3 (&C)[2];" in cpp and "const int& flag;" in cpp
    assert "precision" not in cpp


def test_uniform_block_layout():
    import oracle
    cpp = N.glsl_to_cpp("uniform float a; uniform vec3 b; uniform int c; uniform sampler2D t; uniform mat3 m;"
                        "float SDF_SURFACE(vec3 X) { return 0.0; }")
    lay, size = oracle.uniform_layout(cpp)
    assert [(n, off) for n, t, off, _ in lay] == [("a", 0), ("b", 4), ("c", 16), ("t", 24), ("m", 56)]
    assert size == 96


def test_glsl_builtins_and_swizzles():
    out = run_cpp("float SDF_SURFACE(vec3 X) { return 0.0; }", r'''
  vec3 X(1.5f, 2.0f, -0.25f);
  X.xz = mod(X.xz, 1.0f) - vec2(0.5f);
  vec4 p(X, 1.0f);
  mat3 rot(1,0,0, 0,0,1, 0,1,0);
  p.xyz *= rot;
  vec3 r = rot * vec3(1.0f, 2.0f, 3.0f);
  printf("%g %g %g|%g %g %g %g|%g %g %g|", X.x, X.y, X.z, p.x, p.y, p.z, p.w, r.x, r.y, r.z);
  printf("%g %g %g %g|", sign(-2.0f), fract(-1.25f), smoothstep(0.0f, 2.0f, 1.0f), mod(-1.0f, 3.0f));
  printf("%g %g|", clamp(5.0f, 0.0f, 1.0f), mix(1.0f, 3.0f, 0.25f));
  vec3 e(0.1f, 0.0f, 0.0f); vec3 q = e.xyy + e.yxy + e.yyx; printf("%g %g %g|", q.x, q.y, q.z);
  vec3 zero; float z{}; printf("%g %g", zero.x + zero.y + zero.z, z);
''')
    vals = [list(map(float, part.split())) for part in out.split("|")]
    assert vals[0] == [0.0, 2.0, 0.25]
    assert vals[1] == [0.0, 0.25, 2.0, 1.0]
    assert vals[2] == [1.0, 3.0, 2.0]  # m * v: column combination
    assert vals[3] == [-1.0, 0.75, 0.5, 2.0]
    assert vals[4] == [1.0, 1.5]
    assert np.allclose(vals[5], [0.1, 0.1, 0.1])
    assert vals[6] == [0.0, 0.0]


def test_texture_filtering_semantics():
    out = run_cpp("float SDF_SURFACE(vec3 X) { return 0.0; }", r'''
  float data[4] = {0.0f, 1.0f, 2.0f, 3.0f};
  sampler2D lin{data, 4, 1, 1, 0, 1, 0}, nea{data, 4, 1, 1, 0, 0, 0};
  printf("%g %g %g %g %g", texture(lin, vec2(0.125f, 0.5f)).x, texture(lin, vec2(0.25f, 0.5f)).x,
         texture(lin, vec2(0.0f, 0.5f)).x, texture(lin, vec2(1.0f, 0.5f)).x, texture(nea, vec2(0.3f, 0.5f)).x);
''')
    assert list(map(float, out.split())) == [0.0, 0.5, 0.0, 3.0, 1.0]
