// pt_oracle.h - CPU oracle: a sequential restatement of the reference's spectral path tracer,
// shaders/pathtracer-fragment-shader.glsl (cited PT:line), and of its first-hit programs
// (fh_oracle.inc), for checking the CUDA kernels.
//
// TEST INFRASTRUCTURE. This file is compiled only into the oracle library that tests and the
// benchmark's CPU-baseline leg load; the product never includes or links it.
//
// It follows the shader line by line with GLSL semantics (glslcompat.h types, zero-initialised
// locals as WebGL implementations do, float arithmetic), one pixel at a time, in the order the
// reference consumes random numbers. The scene is included by the build recipe as
// `glsl::SceneUniforms` / `glsl::Scene` (the same GLSL-to-C++ translation the product uses), and
// the per-job uniforms come in as the SnellyParams block of include/snelly_params.h.
#pragma once
#include "snelly_params.h"

namespace oracle {
using namespace glsl;

#ifdef DISPERSION_ENABLED
typedef gfloat RadianceType;
#else
typedef vec3 RadianceType;
#endif

// PT:105-114
static const gfloat DENOM_TOLERANCE = 1.0e-7f, PDF_EPSILON = 1.0e-6f, THROUGHPUT_EPSILON = 1.0e-5f,
                    RADIANCE_EPSILON = 1.0e-6f;
static const gfloat M_PI_F = 3.141592653589793f;
enum { MAT_INVAL = -1, MAT_DIELE = 0, MAT_METAL = 1, MAT_SURFA = 2 };

inline vec3 U3(const float* a) { return vec3(a[0], a[1], a[2]); }

// One pixel's shader invocation: the uniforms, the scene instance and the invocation globals.
struct Invocation {
  const SnellyParams& u;
  Scene& sc;
  struct Basis {
    vec3 nW, tW, bW;
  };
  Basis sunBasis;

  Invocation(const SnellyParams& p, Scene& s) : u(p), sc(s) {}

  // PT:119-130, the four-lane LCG in float arithmetic
  gfloat rand(vec4& rnd) {
    const vec4 q = vec4(1225.0f, 1585.0f, 2457.0f, 2098.0f);
    const vec4 r = vec4(1112.0f, 367.0f, 92.0f, 265.0f);
    const vec4 a = vec4(3423.0f, 2646.0f, 1707.0f, 1999.0f);
    const vec4 m = vec4(4194287.0f, 4194277.0f, 4194191.0f, 4194167.0f);
    vec4 beta = floor(rnd / q);
    vec4 p = a * (rnd - beta * q) - beta * r;
    beta = (1.0f - sign(p)) * 0.5f * m;
    rnd = p + beta;
    return fract(dot(rnd / m, vec4(1.0f, -1.0f, 1.0f, -1.0f)));
  }

  // PT:152-206
  vec3 safe_normalize(vec3 N) { gfloat l = length(N); return N / max(l, DENOM_TOLERANCE); }
  gfloat cosTheta2(vec3 n) { return n.z * n.z; }
  gfloat cosTheta(vec3 n) { return n.z; }
  gfloat tanTheta2(vec3 n) { gfloat ct2 = cosTheta2(n); return max(gfloat(0.0f), 1.0f - ct2) / max(ct2, gfloat(1.0e-7f)); }
  gfloat tanTheta(vec3 n) { return sqrt(max(gfloat(0.0f), tanTheta2(n))); }
  Basis makeBasis(vec3 nW) {
    Basis b;
    b.nW = nW;
    if (abs(nW.z) < abs(nW.x)) { b.tW.x = nW.z; b.tW.y = 0.0f; b.tW.z = -nW.x; }
    else { b.tW.x = 0.0f; b.tW.y = nW.z; b.tW.z = -nW.y; }
    b.tW = safe_normalize(b.tW);
    b.bW = cross(nW, b.tW);
    return b;
  }
  vec3 worldToLocal(vec3 v, const Basis& b) { return vec3(dot(v, b.tW), dot(v, b.bW), dot(v, b.nW)); }
  vec3 localToWorld(vec3 v, const Basis& b) { return b.tW * v.x + b.bW * v.y + b.nW * v.z; }

  // PT:208-271
  vec3 xyzToRgb(vec3 XYZ) {
    vec3 RGB;
    RGB.r = 3.2404542f * XYZ.x - 1.5371385f * XYZ.y - 0.4985314f * XYZ.z;
    RGB.g = -0.9692660f * XYZ.x + 1.8760108f * XYZ.y + 0.0415560f * XYZ.z;
    RGB.b = 0.0556434f * XYZ.x - 0.2040259f * XYZ.y + 1.0572252f * XYZ.z;
    gfloat delta = -min(gfloat(0.0f), min(min(RGB.r, RGB.g), RGB.b));
    RGB.r += delta; RGB.g += delta; RGB.b += delta;
    gfloat sum = RGB.r + RGB.g + RGB.b;
    RGB /= sum;
    return RGB;
  }
  vec3 rgbToXyz(vec3 RGB) {
    vec3 XYZ;
    XYZ.x = 0.4124564f * RGB.r + 0.3575761f * RGB.g + 0.1804375f * RGB.b;
    XYZ.y = 0.2126729f * RGB.r + 0.7151522f * RGB.g + 0.0721750f * RGB.b;
    XYZ.z = 0.0193339f * RGB.r + 0.1191920f * RGB.g + 0.9503041f * RGB.b;
    return XYZ;
  }
#ifdef DISPERSION_ENABLED
  RadianceType rgbToAlbedo(vec3 RGB, vec3 rgb) { return dot(RGB, rgb); }
#else
  RadianceType rgbToAlbedo(vec3 RGB, vec3) { return RGB; }
#endif
  gfloat maxComponent(vec3 v) { return max(max(v.r, v.g), v.b); }
  gfloat maxComponent(gfloat f) { return f; }
  gfloat averageComponent(vec3 v) { return (v.r + v.g + v.b) / 3.0f; }
  gfloat averageComponent(gfloat f) { return f; }

  // PT:301-372
  vec3 sampleSphereUniformly(vec4& rnd) {
    gfloat z = 1.0f - 2.0f * rand(rnd);
    gfloat r = sqrt(max(gfloat(0.0f), 1.0f - z * z));
    (void)r;
    gfloat phi = 2.0f * M_PI_F * rand(rnd);
    return vec3(cos(phi), sin(phi), z);
  }
  vec3 sampleHemisphereUniformly(vec4& rnd) {
    gfloat xi = rand(rnd);
    gfloat r = sqrt(1.0f - xi * xi);
    gfloat phi = 2.0f * M_PI_F * rand(rnd);
    return vec3(r * cos(phi), r * sin(phi), xi);
  }
  vec3 sampleHemisphereCosineWeighted(vec4& rnd, gfloat& pdf) {
    gfloat r = sqrt(rand(rnd));
    gfloat theta = 2.0f * M_PI_F * rand(rnd);
    gfloat x = r * cos(theta), y = r * sin(theta);
    gfloat z = sqrt(max(gfloat(0.0f), 1.0f - x * x - y * y));
    pdf = abs(z) / M_PI_F;
    return vec3(x, y, z);
  }
  gfloat pdfHemisphereCosineWeighted(vec3 wiL) {
    if (wiL.z < 0.0f) return 0.0f;
    return wiL.z / M_PI_F;
  }
  gfloat powerHeuristic(gfloat a, gfloat b) { return a / (a + b); }
  gfloat phaseFunction(gfloat mu, gfloat g) {
    gfloat gSqr = g * g;
    return (1.0f / (4.0f * M_PI_F)) * (1.0f - gSqr) / pow(1.0f - 2.0f * g * mu + gSqr, gfloat(1.5f));
  }
  vec3 samplePhaseFunction(vec3 rayDir, gfloat g, vec4& rnd) {
    gfloat costheta;
    if (abs(g) < 1.0e-3f) costheta = 1.0f - 2.0f * rand(rnd);
    else costheta = 1.0f / (2.0f * g) * (1.0f + g * g - ((1.0f - g * g) * (1.0f - g + 2.0f * g * rand(rnd))));
    gfloat sintheta = sqrt(max(gfloat(0.0f), 1.0f - costheta * costheta));
    gfloat phi = 2.0f * M_PI_F * rand(rnd);
    Basis basis = makeBasis(rayDir);
    return costheta * rayDir + sintheta * (cos(phi) * basis.tW + sin(phi) * basis.bW);
  }

  // PT:379-441
  gfloat microfacetEval(vec3 m, gfloat roughness) {
    gfloat t2 = tanTheta2(m), c2 = cosTheta2(m);
    gfloat r2 = roughness * roughness;
    gfloat exponent = t2 / max(r2, gfloat(1.0e-9f));
    return exp(-exponent) / max(M_PI_F * r2 * c2 * c2, gfloat(1.0e-9f));
  }
  vec3 microfacetSample(vec4& rnd, gfloat roughness) {
    gfloat phiM = (2.0f * M_PI_F) * rand(rnd);
    gfloat cosPhiM = cos(phiM), sinPhiM = sin(phiM);
    gfloat tanThetaMSqr = -roughness * roughness * log(max(gfloat(1.0e-9f), rand(rnd)));
    gfloat cosThetaM = 1.0f / sqrt(1.0f + tanThetaMSqr);
    gfloat sinThetaM = sqrt(max(gfloat(0.0f), 1.0f - cosThetaM * cosThetaM));
    return safe_normalize(vec3(sinThetaM * cosPhiM, sinThetaM * sinPhiM, cosThetaM));
  }
  gfloat microfacetPDF(vec3 m, gfloat roughness) { return microfacetEval(m, roughness) * abs(cosTheta(m)); }
  gfloat smithG1(vec3 v, vec3 m, gfloat roughness) {
    gfloat tanThetaAbs = abs(tanTheta(v));
    if (tanThetaAbs < 1.0e-6f) return 1.0f;
    if (dot(v, m) * v.z <= 0.0f) return 0.0f;
    gfloat a = 1.0f / (max(roughness, gfloat(1.0e-6f)) * tanThetaAbs);
    if (a >= 1.6f) return 1.0f;
    gfloat aSqr = a * a;
    return (3.535f * a + 2.181f * aSqr) / (1.0f + 2.276f * a + 2.577f * aSqr);
  }
  gfloat smithG2(vec3 wo, vec3 wi, vec3 m, gfloat r) { return smithG1(wo, m, r) * smithG1(wi, m, r); }
  gfloat fresnelDielectricReflectance(gfloat cosi, gfloat eta_ti) {
    gfloat c = cosi;
    gfloat g = eta_ti * eta_ti - 1.0f + c * c;
    if (g > 0.0f) {
      g = sqrt(g);
      gfloat A = (g - c) / (g + c);
      gfloat B = (c * (g + c) - 1.0f) / (c * (g - c) + 1.0f);
      return 0.5f * A * A * (1.0f + B * B);
    }
    return 1.0f;
  }

  // ---- spectral material functions (js/materials.js IOR generators) --------------------------------
  gfloat lerpTable(const float* t, int n, gfloat u) {  // LINEAR + CLAMP_TO_EDGE texel lookup
    gfloat x = u * gfloat(float(n)) - 0.5f;
    gfloat x0 = floor(x);
    gfloat f = x - x0;
    int i0 = int(s_tofloat(x0)), i1 = i0 + 1;
    i0 = i0 < 0 ? 0 : (i0 >= n ? n - 1 : i0);
    i1 = i1 < 0 ? 0 : (i1 >= n ? n - 1 : i1);
    gfloat a = t[i0], b = t[i1];
    return a * (1.0f - f) + b * f;
  }
  gfloat IOR_METAL(gfloat wavelength_nm) {  // js/materials.js:646-650
    gfloat u = (wavelength_nm - 390.0f) * gfloat(float(1.0 / 360.0));
    return lerpTable(u_metalN(), SNELLY_METAL_SAMPLES, u);
  }
  gfloat K_METAL(gfloat wavelength_nm) {  // js/materials.js:651-655 (the intended k table)
    gfloat u = (wavelength_nm - 390.0f) * gfloat(float(1.0 / 360.0));
    return lerpTable(u_metalK(), SNELLY_METAL_SAMPLES, u);
  }
  const float* u_metalN() { return u.metalN; }
  const float* u_metalK() { return u.metalK; }
  gfloat IOR_DIELE(gfloat wavelength_nm) {
    const float* C = u.dieleCoeffs;
    switch (u.dieleModel) {
      case SNELLY_IOR_ABBE: {  // js/materials.js:847-861
        gfloat iorVal = C[0], abbe = C[1];
        if (abbe <= 0.0f) return iorVal;
        gfloat nD2 = 0.5893f; nD2 *= nD2;
        gfloat nF2 = 0.4861f; nF2 *= nF2;
        gfloat nC2 = 0.6563f; nC2 *= nC2;
        gfloat cauchyC = (iorVal - 1.0f) / abbe * (nC2 * nF2) / (nC2 - nF2);
        gfloat cauchyB = iorVal - cauchyC / nD2;
        gfloat l = 1.0e-3f * wavelength_nm;
        return cauchyB + cauchyC / (l * l);
      }
      case SNELLY_IOR_SELLMEIER:     // js/materials.js:905-930
      case SNELLY_IOR_SELLMEIER2: {  // js/materials.js:956-981
        gfloat wavelength_um = 1.0e-3f * wavelength_nm;
        gfloat l2 = wavelength_um * wavelength_um;
        gfloat n2 = 1.0f + gfloat(C[0]);
        int terms = (u.dieleNumCoeffs - 1) / 2;
        for (int t = 1; t <= terms; ++t) {
          gfloat B = C[2 * t - 1], Cc = C[2 * t];
          n2 = n2 + B * l2 / (l2 - (u.dieleModel == SNELLY_IOR_SELLMEIER ? Cc * Cc : Cc));
        }
        return max(sqrt(abs(n2)), gfloat(1.0e-3f));
      }
      case SNELLY_IOR_POLYANSKIY: {  // js/materials.js:1014-1034
        gfloat l = 1.0e-3f * wavelength_nm;
        gfloat n2 = gfloat(C[0]) + gfloat(C[1]) * pow(l, gfloat(C[2])) / (l * l - pow(gfloat(C[3]), gfloat(C[4])));
        return max(sqrt(abs(n2)), gfloat(1.0e-3f));
      }
      default: {  // Cauchy, js/materials.js:1064-1089
        gfloat l = 1.0e-3f * wavelength_nm;
        gfloat n = C[0];
        int terms = (u.dieleNumCoeffs - 1) / 2;
        for (int t = 1; t <= terms; ++t) n = n + gfloat(C[2 * t - 1]) * pow(l, gfloat(C[2 * t]));
        return max(n, gfloat(1.0e-3f));
      }
    }
  }

#include "pt_oracle_bsdf.inc"
#include "pt_oracle_integrator.inc"
#include "fh_oracle.inc"
#include "ps_oracle.inc"
};

}  // namespace oracle
