"""The CPU oracle against the reference's own outputs (golden fixtures from the reference shader),
and its building blocks: RNG, seeding, inverse CDF, tables."""
import numpy as np
import pytest

from helpers import (CASES, FH_CASES, GOLDEN, golden, golden_fh, golden_ps, host, oracle_firsthit, oracle_for,
                     oracle_render)


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_golden(name):
    """The restatement reproduces the reference shader bit for bit (running means and RNG)."""
    g = golden(name)
    h = host(name)
    assert (h.width, h.height) == (int(g["width"]), int(g["height"]))
    pix = np.arange(h.width * h.height)
    xyz, mean, rng = oracle_render(h, pix, int(g["frames"]), rng0=g["rng0"])
    np.testing.assert_array_equal(rng, g["rng"])
    np.testing.assert_array_equal(mean, g["mean"])


@pytest.mark.parametrize("name", FH_CASES)
def test_firsthit_oracle_matches_reference_golden(name):
    """The restatements of the normals, ambient-occlusion and pick programs reproduce the
    reference's own shaders bit for bit (running means, RNG lanes, pick distance and material)."""
    g = golden_fh(name)
    h = host(name)
    assert (h.width, h.height) == (int(g["width"]), int(g["height"]))
    pix = np.arange(h.width * h.height)
    for mode, prog in ((1, "normals"), (2, "ao")):
        xyz, mean, rng = oracle_firsthit(h, mode, pix, int(g["frames"]), rng0=g["rng0"])
        np.testing.assert_array_equal(rng, g[prog + "_rng"], err_msg=prog)
        np.testing.assert_array_equal(mean, g[prog + "_mean"], err_msg=prog)
    np.testing.assert_array_equal(oracle_firsthit(h, 3, pix, 1), g["pick"])


def test_tonemap_oracle_matches_reference_golden():
    """The display-transform restatement reproduces the reference's tonemapper program bit for bit
    on path-traced and out-of-gamut / HDR inputs, for three display settings."""
    g = np.load(f"{GOLDEN}/tm_golden.npz")
    lib = oracle_for(host("c0"))
    for k, p in enumerate(g["params"]):
        out = lib.tonemap(g["xyzn"], p)
        np.testing.assert_array_equal(out, g["rgba"][k])


@pytest.mark.parametrize("name", FH_CASES)
def test_ptsimple_oracle_matches_reference_golden(name):
    """The restatement of the simplified path tracer reproduces the reference's own program bit for
    bit (running means and RNG lanes)."""
    g = golden_ps(name)
    h = host(name)
    pix = np.arange(h.width * h.height)
    xyz, mean, rng = oracle_firsthit(h, 4, pix, int(g["frames"]), rng0=g["rng0"])
    np.testing.assert_array_equal(rng, g["rng"])
    np.testing.assert_array_equal(mean, g["mean"])


def test_seeding_is_deterministic_and_in_range():
    h = host("c0")
    lib = oracle_for(h)
    pix = np.arange(4096)
    a = lib.seed(1, pix)
    b = lib.seed(1, pix)
    c = lib.seed(2, pix)
    np.testing.assert_array_equal(a, b)
    assert (a != c).any(axis=1).all()
    m = np.array([4194287, 4194277, 4194191, 4194167])
    assert (a >= 1).all() and (a < m).all()
    np.testing.assert_array_equal(a, golden("c0")["rng0"][:4096])


def test_float_rng_equals_integer_schrage():
    """PT:119-130 in float arithmetic equals exact (a*x) mod m on integer states."""
    h = host("c0")
    lib = oracle_for(h)
    a = np.array([3423, 2646, 1707, 1999], np.int64)
    m = np.array([4194287, 4194277, 4194191, 4194167], np.int64)
    st = lib.seed(7, np.arange(2000)).astype(np.int64)
    for px in range(0, 2000, 97):
        s = st[px].astype(np.uint32).copy()
        x = st[px].copy()
        for _ in range(50):
            u = lib.lib.oracle_rand(s.ctypes.data)
            x = (a * x) % m
            assert (s.astype(np.int64) == x).all()
            v = np.float32(x[0]) / np.float32(m[0]) - np.float32(x[1]) / np.float32(m[1])
            v = np.float32(v + np.float32(x[2]) / np.float32(m[2])) - np.float32(x[3]) / np.float32(m[3])
            v = np.float32(v)
            assert u == np.float32(v - np.floor(v))


def test_cie_table_matches_csv():
    """snelly_b200/data/materials.json's XYZ table is the reference's color.js table, which is the
    CSV resampled by scripts/color/cie.py and printed to 6 decimals."""
    from snelly_b200 import api
    t = np.asarray(api.DATA["xyz_table"]).reshape(1024, 4)
    csv = np.load(f"{GOLDEN}/cie_csv.npy")
    assert np.abs(t[:, :3] - csv).max() <= 5.01e-7
    assert (t[:, 3] == 0).all()


@pytest.mark.parametrize("spec", [("blackbody", 6000.0), ("blackbody", 3000.0), ("flat", (390.0, 750.0)),
                                  ("flat", (450.0, 600.0)), ("mono", 550.0)])
def test_inverse_cdf_runtime_matches_oracle(spec):
    """The runtime's ICDF (C++) equals the oracle's restatement of Spectrum.inverseCDF."""
    import ctypes
    import oracle
    from snelly_b200 import _native as N
    kind, arg = spec
    if kind == "blackbody":
        ref = oracle.inverse_cdf("blackbody", temperature=arg)
        s = N.Spectrum(N.SPECTRUM_BLACKBODY, arg, 390.0, 750.0, 550.0)
    elif kind == "flat":
        ref = oracle.inverse_cdf("flat", band=arg)
        s = N.Spectrum(N.SPECTRUM_FLAT, 6000.0, arg[0], arg[1], 550.0)
    else:
        ref = oracle.inverse_cdf("mono", wavelength=arg)
        s = N.Spectrum(N.SPECTRUM_MONO, 6000.0, 390.0, 750.0, arg)
    out = np.empty(4096, np.float32)
    N.check(N.lib().snelly_inverse_cdf(ctypes.byref(s), out.ctypes.data))
    np.testing.assert_array_equal(out, ref)
    assert (np.diff(ref) >= 0).all() and 0.0 <= ref[0] and ref[-1] <= 1.0


def test_flat_spectrum_icdf_is_linear():
    import oracle
    icdf = oracle.inverse_cdf("flat", band=(390.0, 750.0))
    x = (np.arange(4096) + 1) / 4096.0
    assert np.abs(icdf - x).max() < 1e-3
