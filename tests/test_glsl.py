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


def test_out_and_inout_arguments_take_swizzles():
    """GLSL passes out / inout arguments by copy-in, copy-out, so a swizzle or a component may be
    passed: f(p.xz) writes the result back into p's x and z. A variable of the parameter's own
    type still goes to the function itself (by reference)."""
    out = run_cpp("""
void pR(inout vec2 p, float a) { p = vec2(p.x * a, p.y + a); }
float bump(inout float x, out float y) { x += 1.0; y = 2.0 * x; return x + y; }
vec3 both(inout vec3 q) { q = q.zyx; return q; }
float SDF_SURFACE(vec3 X) { return 0.0; }""", r'''
  Scene sc{SceneUniforms{}};
  vec3 p(1.0f, 2.0f, 3.0f);
  sc.pR(p.xz, 10.0f);                   // swizzle: x *= 10, z += 10
  vec2 v(1.0f, 1.0f);
  sc.pR(v, 2.0f);                       // a variable of the parameter's type
  float y0 = 0.0f;
  float r = sc.bump(p.y, y0);           // a component and an out parameter
  vec4 w(1.0f, 2.0f, 3.0f, 4.0f);
  vec3 s = sc.both(w.wzy);              // swizzled inout with a result
  printf("%g %g %g|%g %g|%g %g|%g %g %g %g|%g %g %g", p.x, p.y, p.z, v.x, v.y, r, y0, w.x, w.y, w.z, w.w, s.x, s.y, s.z);
''')
    vals = [list(map(float, part.split())) for part in out.split("|")]
    assert vals[0] == [10.0, 3.0, 13.0]
    assert vals[1] == [2.0, 3.0]
    assert vals[2] == [9.0, 6.0]
    assert vals[3] == [1.0, 4.0, 3.0, 2.0]  # w.wzy = (4, 3, 2) reversed to (2, 3, 4) -> w = (1, 4, 3, 2)
    assert vals[4] == [2.0, 3.0, 4.0]


def test_constructors_conversions_and_matrix_operators():
    """Constructors that take only the leading components of their last argument, float(v) as
    the first component, float vectors from integer and boolean ones, the component-wise
    comparisons with any / all / not, and the matrix unary minus, subtraction, scalar division
    and compound assignments (m *= n is the matrix product)."""
    out = run_cpp("float SDF_SURFACE(vec3 X) { return 0.0; }", r'''
  vec2 n(5.0f, 6.0f);
  vec3 a(1.0f, 2.0f, n);
  vec4 b(vec3(1.0f, 2.0f, 3.0f), n);
  vec4 c(n, vec3(7.0f, 8.0f, 9.0f));
  printf("%g %g %g|%g %g %g %g|%g %g %g %g|", a.x, a.y, a.z, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w);
  printf("%g %g|", gfloat(vec3(4.0f, 5.0f, 6.0f)), gfloat(n));
  vec3 fi = vec3(ivec3(1, -2, 3));
  vec4 fb = vec4(equal(vec4(1.0f, 2.0f, 3.0f, 4.0f), vec4(1.0f, 0.0f, 3.0f, 0.0f)));
  printf("%g %g %g|%g %g %g %g|", fi.x, fi.y, fi.z, fb.x, fb.y, fb.z, fb.w);
  bvec3 lt = lessThan(vec3(1.0f, 5.0f, 2.0f), vec3(2.0f, 4.0f, 2.0f));
  printf("%d %d %d %d %d %d|", lt.x, lt.y, lt.z, any(lt), all(lt), not_g(lt).y);
  mat2 m(1.0f, 2.0f, 3.0f, 4.0f), k(0.0f, 1.0f, 1.0f, 0.0f);
  mat2 neg = -m, diff = m - k, half = m / 2.0f;
  mat2 prod = m; prod *= k;
  mat2 sc = m; sc *= 3.0f;
  printf("%g %g %g %g|%g %g|%g|%g %g %g %g|%g", neg.c[0].x, neg.c[1].y, diff.c[0].y, diff.c[1].x,
         half.c[0].y, half.c[1].y, sc.c[1].x, prod.c[0].x, prod.c[0].y, prod.c[1].x, prod.c[1].y, (m * k).c[0].x);
''')
    vals = [list(map(float, part.split())) for part in out.split("|")]
    assert vals[0] == [1.0, 2.0, 5.0]
    assert vals[1] == [1.0, 2.0, 3.0, 5.0]
    assert vals[2] == [5.0, 6.0, 7.0, 8.0]
    assert vals[3] == [4.0, 5.0]
    assert vals[4] == [1.0, -2.0, 3.0]
    assert vals[5] == [1.0, 0.0, 1.0, 0.0]
    assert vals[6] == [1.0, 0.0, 0.0, 1.0, 0.0, 1.0]
    assert vals[7] == [-1.0, -4.0, 1.0, 2.0]
    assert vals[8] == [1.0, 2.0]
    assert vals[9] == [9.0]
    assert vals[10] == [3.0, 4.0, 1.0, 2.0]  # columns of m * k: m * (0,1) and m * (1,0)
    assert vals[11] == [3.0]


@pytest.mark.reference
def test_reference_example_scenes_translate_and_compile():
    """Every example scene of the reference whose shader() is one template literal translates and
    compiles (host build) against the compatibility header, with each ${...} substitution replaced
    by 1. The one known exception, fractals/IFS/meshmenger, calls functions it never defines (sd,
    sdf) and reads undeclared names (size, rot)."""
    import glob
    import re

    from conftest import REFERENCE
    known = {"fractals/IFS/meshmenger.html"}
    base = os.path.join(REFERENCE, "exampleScenes")
    tried, failed = 0, []
    for f in sorted(glob.glob(os.path.join(base, "**", "*.html"), recursive=True)):
        text = open(f, encoding="utf-8", errors="replace").read()
        m = re.search(r"prototype\.shader\s*=\s*function\s*\(\)\s*\{", text)
        if not m:
            continue
        i = text.find("`", m.end())
        j = text.find("`", i + 1)
        if i < 0 or j < 0 or i - m.end() > 400:  # built from strings in JavaScript: not extractable here
            continue
        glsl = re.sub(r"\$\{[^}]*\}", "1", text[i + 1:j])
        rel = os.path.relpath(f, base)
        tried += 1
        cpp = N.glsl_to_cpp(glsl)
        src = '#include "glslcompat.h"\nnamespace glsl {\n' + cpp + '\n}\nint main() { return 0; }\n'
        with tempfile.TemporaryDirectory() as d:
            p = os.path.join(d, "t.cpp")
            open(p, "w").write(src)
            r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-w", "-I" + os.path.join(ROOT, "snelly_b200", "csrc"),
                                p], capture_output=True, text=True)
        if r.returncode and rel not in known:
            failed.append(rel)
    assert tried >= 50, tried
    assert not failed, failed


@pytest.mark.reference
@pytest.mark.parametrize("rel", ["fractals/IFS/mandalay_mod.html", "fractals/doyleSpirals.html"])
def test_reference_example_scene_compiles_for_the_gpu(rel):
    """Two example scenes that need the copy-in/copy-out overloads (swizzles passed to inout
    parameters) and the vector relational functions, conversions and matrix operators, compiled
    by NVRTC for sm_100a with the path tracer's kernels (no GPU needed)."""
    import re

    from conftest import REFERENCE
    from snelly_b200 import scenes
    from snelly_b200.testing import HostSnelly
    text = open(os.path.join(REFERENCE, "exampleScenes", rel), encoding="utf-8", errors="replace").read()
    m = re.search(r"prototype\.shader\s*=\s*function\s*\(\)\s*\{", text)
    i = text.find("`", m.end())
    glsl = re.sub(r"\$\{[^}]*\}", "1", text[i + 1:text.find("`", i + 1)])
    nbytes, _ = N.compile_check(glsl, HostSnelly(scenes.PlainSphere(32, 32)).scene_opts())
    assert nbytes > 0


def test_scene_reads_renderer_uniforms():
    """Scene code sits inside the reference's fragment shader, so it may read the path tracer's
    own uniforms (minLengthScale, sunDir, ...) without declaring them. The translation adds each
    one it reads to the scene's uniform block, after the scene's own uniforms and marked as a
    renderer uniform, and the job's parameters fill it (snelly_render here; the oracle's uniform
    packing likewise). A uniform the scene declares itself stays the scene's own."""
    import oracle
    from snelly_b200 import _native as N
    cpp = N.glsl_to_cpp("""uniform float R; uniform float skyPower;
float SDF_SURFACE(vec3 X) { return length(X) - R - minLengthScale + 0.0 * (sunDir.x + skyPower); }""")
    layout, size = oracle.uniform_layout(cpp)
    assert [(n, t, off) for n, t, off, _ in layout] == [("R", "gfloat", 0), ("skyPower", "gfloat", 4),
                                                         ("minLengthScale", "gfloat", 8), ("sunDir", "vec3", 12)]
    assert oracle.renderer_uniforms(cpp) == {"minLengthScale", "sunDir"}
    p = N.SnellyParams()
    p.minLengthScale = 0.125
    p.sunDir[:] = [1.0, 2.0, 3.0]
    p.skyPower = 9.0  # the scene's own skyPower uniform is set by its syncShader, not from here
    ub = np.frombuffer(oracle.pack_uniforms(cpp, {"R": ("float", [1.5]), "skyPower": ("float", [0.5])}, params=p),
                       np.float32)
    assert ub.tolist() == [1.5, 0.5, 0.125, 1.0, 2.0, 3.0]
    plain = N.glsl_to_cpp("float SDF_SURFACE(vec3 X) { return length(X) - 1.0; }")
    assert "renderer uniform" not in plain
