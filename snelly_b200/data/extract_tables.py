"""Extract the reference's spectral data tables into this package.

The path tracer needs the same numerical tables as the reference to give the same results:

* the CIE XYZ colour-matching table, 1024 x vec4 over 390..750 nm (js/color.js:24-284);
* the 23 tabulated metal n,k spectra, 64 samples each over 390..750 nm (js/materials.js:536-627;
  22 are registered by Materials, js/materials.js:1150-1171);
* the dielectric catalogue: model and coefficients (js/materials.js:1125-1147).

This script reads them from a checkout of the reference and writes
  snelly_b200/data/materials.json        (metals, dielectrics, xyz table)
  snelly_b200/csrc/cie_xyz_table.inc     (the XYZ table as a C initialiser for libsnelly)
Both outputs are committed; nothing reads the reference at run time.

Usage: python extract_tables.py /path/to/reference
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

# Constructor name in js/materials.js -> model name used by this package.
MODELS = {
    "AbbeDielectric": "abbe",
    "SellmeierDielectric": "sellmeier",
    "Sellmeier2Dielectric": "sellmeier2",
    "PolyanskiyDielectric": "polyanskiy",
    "CauchyDielectric": "cauchy",
}


def parse_floats(text):
    return [float(x) for x in re.findall(r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?", text)]


def extract(ref):
    color = open(os.path.join(ref, "js", "color.js")).read()
    m = re.search(r"function wavelengthToXYZTable\(\)\s*\{\s*return new Float32Array\(\[(.*?)\]\);", color, re.S)
    xyz = parse_floats(m.group(1))
    assert len(xyz) == 4096, len(xyz)

    mats = open(os.path.join(ref, "js", "materials.js")).read()
    metals = {}
    for fm in re.finditer(r"function tabulated_(\w+)\(\)\s*\{.*?n:\s*new Float32Array\(\[(.*?)\]\).*?"
                          r"k:\s*new Float32Array\(\[(.*?)\]\)", mats, re.S):
        n = parse_floats(fm.group(2))
        k = parse_floats(fm.group(3))
        assert len(n) == 64 and len(k) == 64, fm.group(1)
        metals[fm.group(1)] = {"n": n, "k": k}
    registered = {}
    for rm in re.finditer(r'addMetal\(\s*new TabulatedMetal\("([^"]+)",\s*tabulated_(\w+)\(\)', mats):
        registered[rm.group(1)] = rm.group(2)

    dielectrics = {}
    for dm in re.finditer(r'addDielectric\(\s*new (\w+)\("([^"]+)",\s*(.*?)\)\s*\);', mats):
        ctor, name, args = dm.group(1), dm.group(2), dm.group(3)
        coeffs = parse_floats(args)
        dielectrics[name] = {"model": MODELS[ctor], "coeffs": coeffs}
    return xyz, metals, registered, dielectrics


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SNELLY_REFERENCE", "")
    if not ref:
        sys.exit("usage: extract_tables.py <reference checkout> (or set $SNELLY_REFERENCE)")
    xyz, metals, registered, dielectrics = extract(ref)
    out = {
        "source": "portsmouth/snelly js/color.js, js/materials.js",
        "xyz_table": xyz,
        "metal_tables": metals,
        "metals": registered,
        "dielectrics": dielectrics,
    }
    with open(os.path.join(HERE, "materials.json"), "w") as f:
        json.dump(out, f, indent=0)
    inc = os.path.join(HERE, "..", "csrc", "cie_xyz_table.inc")
    with open(inc, "w") as f:
        f.write("// CIE XYZ colour-matching table, 1024 x (X, Y, Z, 0) over 390..750 nm, as in the\n")
        f.write("// reference's js/color.js:24-284. Generated by snelly_b200/data/extract_tables.py.\n")
        for i in range(0, len(xyz), 8):
            f.write(", ".join(repr(float(v)) + "f" for v in xyz[i:i + 8]) + ",\n")
    print(f"{len(metals)} metal tables, {len(registered)} registered, {len(dielectrics)} dielectrics")


if __name__ == "__main__":
    main()
