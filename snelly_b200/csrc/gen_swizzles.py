"""Generate glsl_swizzles.inc: the swizzle union members of glsl::vec2/vec3/vec4.

GLSL lets any vector expose 2-, 3- or 4-component "swizzles" (`v.xzy`, `c.rgb`, `t.st`)
that can be read and, when no component repeats, written (`X.xz = ...`). The compat header
models each swizzle as a union member of type swN<Storage, I...> that aliases the vector's
float storage; this script writes one member declaration per name, for the three GLSL
component-name sets (xyzw, rgba, stpq).

Run: python gen_swizzles.py  (rewrites glsl_swizzles.inc beside this file)
"""
import itertools
import os

SETS = ["xyzw", "rgba", "stpq"]


def members(n):
    out = []
    for names in SETS:
        comp = names[:n]
        for k in (2, 3, 4):
            for idx in itertools.product(range(n), repeat=k):
                name = "".join(comp[i] for i in idx)
                args = ",".join(str(i) for i in idx)
                out.append(f"sw{k}<{n},{args}> {name};")
    return out


def main():
    here = os.path.dirname(os.path.abspath(__file__))
    path = os.path.join(here, "glsl_swizzles.inc")
    lines = ["// Generated by gen_swizzles.py; do not edit.", ""]
    for n in (2, 3, 4):
        lines.append(f"#if GLSL_SWIZZLE_STORAGE == {n}")
        ms = members(n)
        for i in range(0, len(ms), 6):
            lines.append(" ".join(ms[i:i + 6]))
        lines.append("#endif")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    print(f"wrote {path}")


if __name__ == "__main__":
    main()
