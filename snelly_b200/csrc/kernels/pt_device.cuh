// pt_device.cuh - device-side building blocks of the spectral SDF path tracer (sm_100a).
//
// Compiled by NVRTC together with one scene: glslcompat.h, then `namespace glsl { struct
// SceneUniforms; struct Scene; }` produced from the scene's GLSL, then this file. Compile-time
// configuration comes in as macros, mirroring the reference's shader defines
// (js/renderer.js:292-316): HAS_SURFACE, HAS_METAL, HAS_DIELECTRIC, HAS_GEOMETRY,
// HAS_ATMOSPHERE, HAS_FOG, HAS_VOLUME_EMISSION, HAS_SPHERE_LIGHT, HAS_NORMALMAP,
// HAS_{SURFACE,METAL,DIELECTRIC}_NORMALMAP, HAS_CUSTOM_CAMERA, DISPERSION_ENABLED,
// INTERACTIVE_MODE, and the loop bounds MAX_MARCH_STEPS, MAX_BOUNCES,
// MAX_ATMOSPHERE_SCATTERS, MAX_SAMPLES_PER_FRAME.
//
// Every estimator follows shaders/pathtracer-fragment-shader.glsl (cited as PT:line) so that
// the same random numbers are consumed in the same order as the reference; how the work is
// laid out on the GPU (kernels, queues, state in HBM) is in pt_kernels.cu.
#pragma once
#include "snelly_params.h"
#include "pt_rng.cuh"

#ifndef MAX_MARCH_STEPS
#define MAX_MARCH_STEPS 256
#endif
#ifndef MAX_BOUNCES
#define MAX_BOUNCES 3
#endif
#ifndef MAX_ATMOSPHERE_SCATTERS
#define MAX_ATMOSPHERE_SCATTERS 1
#endif
#ifndef MAX_SAMPLES_PER_FRAME
#define MAX_SAMPLES_PER_FRAME 1
#endif

#define SD_FN __device__ __forceinline__

namespace sdev {
using glsl::vec2;
using glsl::vec3;
using glsl::vec4;
using glsl::Scene;

#ifdef DISPERSION_ENABLED
typedef float Rad;  // one wavelength per path (PT:142-146)
#else
typedef vec3 Rad;
#endif

// PT:105-114
constexpr float kDenomTol = 1.0e-7f;
constexpr float kPdfEps = 1.0e-6f;
constexpr float kThroughputEps = 1.0e-5f;
constexpr float kRadianceEps = 1.0e-6f;
constexpr float kPi = 3.141592653589793f;
enum { MAT_INVAL = -1, MAT_DIELE = 0, MAT_METAL = 1, MAT_SURFA = 2 };

SD_FN vec3 v3(const float* a) { return vec3(a[0], a[1], a[2]); }
SD_FN float avg(float f) { return f; }
SD_FN float avg(const vec3& v) { return (v.x + v.y + v.z) / 3.0f; }
SD_FN float maxc(float f) { return f; }
SD_FN float maxc(const vec3& v) { return fmaxf(fmaxf(v.x, v.y), v.z); }

// ---- random numbers: pt_rng.cuh (Rng, rand01) -------------------------------------------------

// ---- tables (GL LINEAR + CLAMP_TO_EDGE 1-D lookups, texel centres at (i+0.5)/n) ---------------
SD_FN float table1(const float* t, int n, float u) {
  float x = u * float(n) - 0.5f;
  float x0 = glsl::s_floor(x);
  float f = x - x0;
  int i0 = int(x0), i1 = i0 + 1;
  i0 = i0 < 0 ? 0 : (i0 >= n ? n - 1 : i0);
  i1 = i1 < 0 ? 0 : (i1 >= n ? n - 1 : i1);
  float a = t[i0], b = t[i1];
  return a * (1.0f - f) + b * f;
}
SD_FN vec3 table_xyz(const float* t, float u) {
  const int n = SNELLY_XYZ_SAMPLES;
  float x = u * float(n) - 0.5f;
  float x0 = glsl::s_floor(x);
  float f = x - x0;
  int i0 = int(x0), i1 = i0 + 1;
  i0 = i0 < 0 ? 0 : (i0 >= n ? n - 1 : i0);
  i1 = i1 < 0 ? 0 : (i1 >= n ? n - 1 : i1);
  float4 a = __ldg(reinterpret_cast<const float4*>(t) + i0);
  float4 b = __ldg(reinterpret_cast<const float4*>(t) + i1);
  return vec3(a.x * (1.0f - f) + b.x * f, a.y * (1.0f - f) + b.y * f, a.z * (1.0f - f) + b.z * f);
}

// ---- local frames (PT:152-206) -----------------------------------------------------------------
struct Frame {
  vec3 n, t, b;  // normal (local z), tangent (local x), bitangent (local y)
};
SD_FN vec3 safe_normalize(const vec3& v) { return v / fmaxf(glsl::length(v), kDenomTol); }
SD_FN Frame make_frame(const vec3& n) {
  Frame f;
  f.n = n;
  if (fabsf(n.z) < fabsf(n.x)) f.t = vec3(n.z, 0.0f, -n.x);
  else f.t = vec3(0.0f, n.z, -n.y);
  f.t = safe_normalize(f.t);
  f.b = glsl::cross(n, f.t);
  return f;
}
SD_FN vec3 to_local(const vec3& v, const Frame& f) {
  return vec3(glsl::dot(v, f.t), glsl::dot(v, f.b), glsl::dot(v, f.n));
}
SD_FN vec3 to_world(const vec3& v, const Frame& f) { return f.t * v.x + f.b * v.y + f.n * v.z; }

SD_FN float cos2(const vec3& w) { return w.z * w.z; }
SD_FN float tan2(const vec3& w) {
  float c2 = cos2(w);
  return fmaxf(0.0f, 1.0f - c2) / fmaxf(c2, 1.0e-7f);
}
SD_FN float tanabs(const vec3& w) { return sqrtf(fmaxf(0.0f, tan2(w))); }

// ---- colour (PT:208-251) -----------------------------------------------------------------------
SD_FN vec3 xyz_to_rgb_normalized(const vec3& c) {
  vec3 o;
  o.x = 3.2404542f * c.x - 1.5371385f * c.y - 0.4985314f * c.z;
  o.y = -0.9692660f * c.x + 1.8760108f * c.y + 0.0415560f * c.z;
  o.z = 0.0556434f * c.x - 0.2040259f * c.y + 1.0572252f * c.z;
  float lift = -fminf(0.0f, fminf(fminf(o.x, o.y), o.z));  // bring out-of-gamut colours in
  o.x += lift;
  o.y += lift;
  o.z += lift;
  float sum = o.x + o.y + o.z;
  return o / sum;
}
SD_FN vec3 rgb_to_xyz(const vec3& c) {
  return vec3(0.4124564f * c.x + 0.3575761f * c.y + 0.1804375f * c.z,
              0.2126729f * c.x + 0.7151522f * c.y + 0.0721750f * c.z,
              0.0193339f * c.x + 0.1191920f * c.y + 0.9503041f * c.z);
}
// An RGB "albedo-like" colour seen by the current beam: at one wavelength, its projection on
// the normalised rgb colour-matching weights; in RGB mode, the colour itself.
#ifdef DISPERSION_ENABLED
SD_FN Rad albedo(const vec3& c, const vec3& w) { return glsl::dot(c, w); }
#else
SD_FN Rad albedo(const vec3& c, const vec3&) { return c; }
#endif

// ---- sampling (PT:301-372) ---------------------------------------------------------------------
// Note: the reference's uniform sphere sample returns (cos phi, sin phi, z) without the sin-theta
// scale (PT:303-309); it is reproduced as is.
SD_FN vec3 sample_sphere_ref(Rng& g) {
  float z = 1.0f - 2.0f * rand01(g);
  float phi = 2.0f * kPi * rand01(g);
  return vec3(cosf(phi), sinf(phi), z);
}
SD_FN vec3 sample_hemisphere_uniform(Rng& g) {
  float xi = rand01(g);
  float r = sqrtf(1.0f - xi * xi);
  float phi = 2.0f * kPi * rand01(g);
  return vec3(r * cosf(phi), r * sinf(phi), xi);
}
SD_FN vec3 sample_cosine(Rng& g, float& pdf) {
  float r = sqrtf(rand01(g));
  float th = 2.0f * kPi * rand01(g);
  float x = r * cosf(th), y = r * sinf(th);
  float z = sqrtf(fmaxf(0.0f, 1.0f - x * x - y * y));
  pdf = fabsf(z) / kPi;
  return vec3(x, y, z);
}
SD_FN float pdf_cosine(const vec3& w) { return w.z < 0.0f ? 0.0f : w.z / kPi; }
SD_FN float balance(float a, float b) { return a / (a + b); }  // PT:343 ("powerHeuristic")

SD_FN float hg_phase(float mu, float g) {
  float g2 = g * g;
  return (1.0f / (4.0f * kPi)) * (1.0f - g2) / powf(1.0f - 2.0f * g * mu + g2, 1.5f);
}
// PT:360-372 (the cosine formula is the reference's own, reproduced as is)
SD_FN vec3 sample_hg(const vec3& dir, float g, Rng& rng) {
  float ct;
  if (fabsf(g) < 1.0e-3f) ct = 1.0f - 2.0f * rand01(rng);
  else ct = 1.0f / (2.0f * g) * (1.0f + g * g - ((1.0f - g * g) * (1.0f - g + 2.0f * g * rand01(rng))));
  float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
  float phi = 2.0f * kPi * rand01(rng);
  Frame f = make_frame(dir);
  return ct * dir + st * (cosf(phi) * f.t + sinf(phi) * f.b);
}

// ---- Beckmann microfacets (PT:379-425) ---------------------------------------------------------
SD_FN float beckmann_D(const vec3& m, float alpha) {
  float t2 = tan2(m), c2 = cos2(m);
  float a2 = alpha * alpha;
  float e = t2 / fmaxf(a2, 1.0e-9f);
  return expf(-e) / fmaxf(kPi * a2 * c2 * c2, 1.0e-9f);
}
SD_FN vec3 beckmann_sample(Rng& g, float alpha) {
  float phi = (2.0f * kPi) * rand01(g);
  float cp = cosf(phi), sp = sinf(phi);
  float t2 = -alpha * alpha * logf(fmaxf(1.0e-9f, rand01(g)));
  float ct = 1.0f / sqrtf(1.0f + t2);
  float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
  return safe_normalize(vec3(st * cp, st * sp, ct));
}
SD_FN float beckmann_pdf(const vec3& m, float alpha) { return beckmann_D(m, alpha) * fabsf(m.z); }
SD_FN float smith_g1(const vec3& v, const vec3& m, float alpha) {
  float ta = fabsf(tanabs(v));
  if (ta < 1.0e-6f) return 1.0f;
  if (glsl::dot(v, m) * v.z <= 0.0f) return 0.0f;
  float a = 1.0f / (fmaxf(alpha, 1.0e-6f) * ta);
  if (a >= 1.6f) return 1.0f;
  float a2 = a * a;
  return (3.535f * a + 2.181f * a2) / (1.0f + 2.276f * a + 2.577f * a2);
}
SD_FN float smith_g2(const vec3& wo, const vec3& wi, const vec3& m, float alpha) {
  return smith_g1(wo, m, alpha) * smith_g1(wi, m, alpha);
}
SD_FN float fresnel_dielectric(float cosi, float eta) {
  float c = cosi;
  float g = eta * eta - 1.0f + c * c;
  if (g > 0.0f) {
    g = sqrtf(g);
    float A = (g - c) / (g + c);
    float B = (c * (g + c) - 1.0f) / (c * (g - c) + 1.0f);
    return 0.5f * A * A * (1.0f + B * B);
  }
  return 1.0f;  // total internal reflection
}

// ---- per-job parameters in constant memory ----------------------------------------------------
// One launch serves up to SNELLY_MAX_BATCH jobs of the same scene module. Scalars are read from
// the constant bank (broadcast when a warp works on one job); the lane-divergent table lookups
// (metal n,k) go to the global-memory copy of the same block.
}  // namespace sdev
#ifndef SNELLY_MAX_BATCH
#define SNELLY_MAX_BATCH 32
#endif
// Unmangled module globals: the runtime looks them up by name.
__constant__ SnellyParams c_params[SNELLY_MAX_BATCH];
__constant__ __align__(16) unsigned char c_uniforms[SNELLY_MAX_BATCH][sizeof(glsl::SceneUniforms)];
namespace sdev {
SD_FN const glsl::SceneUniforms& uniforms_of(int job) {
  return *reinterpret_cast<const glsl::SceneUniforms*>(c_uniforms[job]);
}

// ---- per-path context ----------------------------------------------------------------------------
// `sc` is this stage's instance of the scene (GLSL globals are per invocation; each kernel stage
// builds its own and runs INIT(), see scene_for()).
struct Ctx {
  const SnellyParams& P;   // constant-bank copy
  const SnellyParams* Pg;  // global-memory copy (lane-divergent table reads)
  Scene& sc;
  int job;
  float lambda;  // wavelength in nm
  vec3 cmf;      // normalised rgb colour-matching weights at lambda (zero in RGB mode)
  Frame sun;     // frame around sunDir (PT:1950)
};

// ---- spectral indices (js/materials.js:640-657, 842-861, 905-930, 956-981, 1014-1034, 1064-1089)
SD_FN float ior_dielectric(const Ctx& c) {
  const SnellyParams& P = c.P;
  const float* C = P.dieleCoeffs;
  float l = 1.0e-3f * c.lambda;
  switch (P.dieleModel) {
    case SNELLY_IOR_ABBE: {
      if (C[1] <= 0.0f) return C[0];
      float nD2 = 0.5893f; nD2 *= nD2;
      float nF2 = 0.4861f; nF2 *= nF2;
      float nC2 = 0.6563f; nC2 *= nC2;
      float cc = (C[0] - 1.0f) / C[1] * (nC2 * nF2) / (nC2 - nF2);
      float cb = C[0] - cc / nD2;
      return cb + cc / (l * l);
    }
    case SNELLY_IOR_SELLMEIER:
    case SNELLY_IOR_SELLMEIER2: {
      float l2 = l * l;
      float n2 = 1.0f + C[0];
      int terms = (P.dieleNumCoeffs - 1) / 2;
      for (int t = 1; t <= terms; ++t) {
        float pole = P.dieleModel == SNELLY_IOR_SELLMEIER ? C[2 * t] * C[2 * t] : C[2 * t];
        n2 = n2 + C[2 * t - 1] * l2 / (l2 - pole);
      }
      return fmaxf(sqrtf(fabsf(n2)), 1.0e-3f);
    }
    case SNELLY_IOR_POLYANSKIY: {
      float n2 = C[0] + C[1] * powf(l, C[2]) / (l * l - powf(C[3], C[4]));
      return fmaxf(sqrtf(fabsf(n2)), 1.0e-3f);
    }
    default: {  // Cauchy
      float n = C[0];
      int terms = (P.dieleNumCoeffs - 1) / 2;
      for (int t = 1; t <= terms; ++t) n = n + C[2 * t - 1] * powf(l, C[2 * t]);
      return fmaxf(n, 1.0e-3f);
    }
  }
}
SD_FN float metal_table_u(float lambda) { return (lambda - 390.0f) * float(1.0 / 360.0); }
SD_FN float ior_metal(const Ctx& c) { return table1(c.Pg->metalN, SNELLY_METAL_SAMPLES, metal_table_u(c.lambda)); }
SD_FN float k_metal(const Ctx& c) { return table1(c.Pg->metalK, SNELLY_METAL_SAMPLES, metal_table_u(c.lambda)); }

// ---- BSDFs (PT:447-852) ----------------------------------------------------------------------------
#ifdef HAS_DIELECTRIC
SD_FN bool refract_from_transmitted(const vec3& n, float eta, const vec3& wt, vec3& wi) {
  float wtn = glsl::dot(wt, n);
  float disc = 1.0f - eta * eta * (1.0f - wtn * wtn);
  if (disc < 0.0f) return false;
  wi = eta * wt - n * glsl::sign(wtn) * (eta * fabsf(wtn) - sqrtf(disc));
  return true;
}
SD_FN bool refract_from_incident(const vec3& n, float eta, const vec3& wi, vec3& wt) {
  float win = glsl::dot(wi, n);
  float disc = 1.0f - (1.0f - win * win) / (eta * eta);
  if (disc < 0.0f) return false;
  wt = wi / eta - n * glsl::sign(win) * (fabsf(win) / eta - sqrtf(disc));
  return true;
}
SD_FN Rad diele_albedo(const Ctx& c, const vec3& X, const vec3& wiL, const Frame& f) {
  vec3 wiW = to_world(wiL, f);
  return albedo(c.sc.DIELECTRIC_SPECULAR_REFLECTANCE(v3(c.P.dieleSpecAlbedoRGB), X, f.n, wiW), c.cmf);
}
SD_FN Rad diele_absorption(const Ctx& c, const vec3& X) {
  return albedo(c.sc.DIELECTRIC_ABSORPTION(v3(c.P.dieleAbsorptionRGB), X), c.cmf);
}
SD_FN Rad diele_eval(const Ctx& c, const vec3& X, const Frame& f, const vec3& wiL, const vec3& woL, bool fromCamera) {
  float ior = ior_dielectric(c);
  bool refl = woL.z * wiL.z > 0.0f;
  Rad alb = diele_albedo(c, X, wiL, f);
  vec3 inc = fromCamera ? -woL : -wiL;
  vec3 out = fromCamera ? wiL : woL;
  bool entering = inc.z < 0.0f;
  vec3 h = refl ? safe_normalize(woL + wiL) : (entering ? safe_normalize(inc - ior * out) : safe_normalize(ior * inc - out));
  if (h.z < 0.0f) h = h * -1.0f;
  float alpha = c.sc.DIELECTRIC_ROUGHNESS(c.P.dieleRoughness, X, f.n);
  float D = beckmann_D(h, alpha);
  float G = smith_g2(-inc, out, h, alpha);
  float eta = entering ? ior : 1.0f / ior;
  Rad Fr = alb * fresnel_dielectric(fabsf(wiL.z), eta);
  if (refl) return alb * Fr * D * G / fmaxf(4.0f * fabsf(woL.z) * fabsf(wiL.z), kDenomTol);
  float im = glsl::dot(-inc, h), om = glsl::dot(out, h);
  float sd = im + eta * om;
  float jac = eta * eta * fabsf(om) / fmaxf(sd * sd, kDenomTol);
  return (Rad(1.0f) - Fr) * G * D * fabsf(im) * jac / fmaxf(fabsf(woL.z) * fabsf(wiL.z), kDenomTol);
}
SD_FN float diele_pdf(const Ctx& c, const vec3& X, const Frame& f, const vec3& wiL, const vec3& woL, bool fromCamera) {
  float ior = ior_dielectric(c);
  bool refl = woL.z * wiL.z > 0.0f;
  Rad alb = diele_albedo(c, X, wiL, f);
  vec3 inc = fromCamera ? -woL : -wiL;
  vec3 out = fromCamera ? wiL : woL;
  bool entering = inc.z < 0.0f;
  float eta = entering ? ior : 1.0f / ior;
  Rad Fr = alb * fresnel_dielectric(fabsf(wiL.z), eta);
  vec3 h;
  float jac, pdf;
  if (refl) {
    h = safe_normalize(woL + wiL);
    jac = 1.0f / fmaxf(4.0f * fabsf(glsl::dot(wiL, h)), kDenomTol);
    pdf = avg(Fr);
  } else {
    h = entering ? safe_normalize(inc - ior * out) : safe_normalize(ior * inc - out);
    if (h.z < 0.0f) h = h * -1.0f;
    float im = glsl::dot(-inc, h), om = glsl::dot(out, h);
    float sd = im + eta * om;
    jac = eta * eta * fabsf(om) / fmaxf(sd * sd, kDenomTol);
    pdf = 1.0f - avg(Fr);
  }
  float alpha = c.sc.DIELECTRIC_ROUGHNESS(c.P.dieleRoughness, X, f.n);
  pdf *= beckmann_pdf(h, alpha);
  return fabsf(pdf * jac);
}
// `woL` is read before it is written on the transmission branch (PT:600): the caller's value is
// part of the reference's behaviour (zero for a fresh local, see the camera path).
SD_FN Rad diele_sample(const Ctx& c, const vec3& X, const Frame& f, const vec3& wiL, bool fromCamera, vec3& woL,
                       float& pdfOut, Rng& g) {
  float ior = ior_dielectric(c);
  Rad alb = diele_albedo(c, X, wiL, f);
  float eta_r = (wiL.z >= 0.0f) ? ior : 1.0f / ior;
  Rad Fr = alb * fresnel_dielectric(fabsf(wiL.z), eta_r);
  float alpha = c.sc.DIELECTRIC_ROUGHNESS(c.P.dieleRoughness, X, f.n);
  vec3 m = beckmann_sample(g, alpha);
  float mpdf = beckmann_pdf(m, alpha);
  float pr = avg(Fr);
  if (rand01(g) < pr) {
    woL = -wiL + 2.0f * glsl::dot(wiL, m) * m;
    if (woL.z * wiL.z < 0.0f) woL = woL * -1.0f;
    float D = beckmann_D(m, alpha);
    float G = smith_g2(wiL, woL, m, alpha);
    Rad fr = Fr * D * G / fmaxf(4.0f * fabsf(woL.z) * fabsf(wiL.z), kDenomTol);
    float jac = 1.0f / fmaxf(fabsf(4.0f * glsl::dot(wiL, m)), kDenomTol);
    pdfOut = mpdf * pr * jac;
    return fr;
  }
  vec3 inc = fromCamera ? -woL : -wiL;
  vec3 out = fromCamera ? wiL : woL;
  bool entering = inc.z < 0.0f;
  float eta = entering ? ior : 1.0f / ior;
  if (fromCamera) {
    if (!refract_from_transmitted(m, eta, out, inc)) return Rad(0.0f);
    woL = -inc;
  } else {
    inc = -wiL;
    if (!refract_from_incident(m, eta, inc, out)) return Rad(0.0f);
    woL = out;
  }
  float im = glsl::dot(-inc, m);
  Rad Frm = Rad(fresnel_dielectric(fabsf(im), eta));
  Rad Trm = Rad(1.0f) - alb * Frm;
  float D = beckmann_D(m, alpha);
  float G = smith_g2(-inc, out, m, alpha);
  float om = glsl::dot(out, m);
  float sd = im + eta * om;
  float jac = eta * eta * fabsf(om) / fmaxf(sd * sd, kDenomTol);
  Rad ft = Rad(fabsf(im) * jac * Trm * G * D) / fmaxf(fabsf(woL.z) * fabsf(wiL.z), kDenomTol);
  pdfOut = (1.0f - pr) * mpdf * fabsf(jac);
  return ft;
}
#endif  // HAS_DIELECTRIC

#ifdef HAS_METAL
SD_FN float fresnel_conductor(float cosi, float n, float k) {
  float c = fabsf(cosi), c2 = c * c;
  float nk = n * n + k * k, nkc = nk * c2, tnc = 2.0f * n * c;
  float rpar = (nkc - tnc + 1.0f) / (nkc + tnc + 1.0f);
  float rper = (nk - tnc + c2) / (nk + tnc + c2);
  return 0.5f * (rpar + rper);
}
SD_FN Rad metal_albedo(const Ctx& c, const vec3& X, const vec3& wiL, const Frame& f) {
  vec3 wiW = to_world(wiL, f);
  return albedo(c.sc.METAL_SPECULAR_REFLECTANCE(v3(c.P.metalSpecAlbedoRGB), X, f.n, wiW), c.cmf);
}
SD_FN Rad metal_eval(const Ctx& c, const vec3& X, const Frame& f, const vec3& wiL, const vec3& woL) {
  if (wiL.z < 0.0f) return Rad(0.0f);
  float Fr = fresnel_conductor(wiL.z, ior_metal(c), k_metal(c));
  vec3 h = glsl::normalize(woL + wiL);
  float alpha = c.sc.METAL_ROUGHNESS(c.P.metalRoughness, X, f.n);
  float D = beckmann_D(h, alpha);
  float G = smith_g2(wiL, woL, h, alpha);
  Rad a = metal_albedo(c, X, wiL, f);
  return a * Fr * D * G / fmaxf(4.0f * fabsf(woL.z) * fabsf(wiL.z), kDenomTol);
}
SD_FN float metal_pdf(const Ctx& c, const vec3& X, const Frame& f, const vec3& wiL, const vec3& woL) {
  if (wiL.z < 0.0f) return kPdfEps;
  vec3 h = safe_normalize(woL + wiL);
  float jac = 1.0f / fmaxf(fabsf(4.0f * glsl::dot(wiL, h)), kDenomTol);
  float alpha = c.sc.METAL_ROUGHNESS(c.P.metalRoughness, X, f.n);
  return beckmann_pdf(h, alpha) * jac;
}
SD_FN Rad metal_sample(const Ctx& c, const vec3& X, const Frame& f, const vec3& wiL, vec3& woL, float& pdfOut, Rng& g) {
  if (wiL.z < 0.0f) return Rad(0.0f);
  float Fr = fresnel_conductor(wiL.z, ior_metal(c), k_metal(c));
  float alpha = c.sc.METAL_ROUGHNESS(c.P.metalRoughness, X, f.n);
  vec3 m = beckmann_sample(g, alpha);
  woL = -wiL + 2.0f * glsl::dot(wiL, m) * m;
  if (woL.z < kDenomTol) woL.z *= -1.0f;
  float D = beckmann_D(m, alpha);
  float G = smith_g2(wiL, woL, m, alpha);
  Rad a = metal_albedo(c, X, wiL, f);
  Rad fr = a * Fr * D * G / fmaxf(4.0f * fabsf(woL.z) * fabsf(wiL.z), kDenomTol);
  float jac = 1.0f / fmaxf(fabsf(4.0f * glsl::dot(wiL, m)), kDenomTol);
  pdfOut = beckmann_pdf(m, alpha) * jac;
  return fr;
}
#endif  // HAS_METAL

#ifdef HAS_SURFACE
SD_FN Rad surf_diffuse(const Ctx& c, const vec3& X, const vec3& n, const vec3& wiW) {
  return albedo(c.sc.SURFACE_DIFFUSE_REFLECTANCE(v3(c.P.surfaceDiffuseAlbedoRGB), X, n, wiW), c.cmf);
}
SD_FN Rad surf_specular(const Ctx& c, const vec3& X, const vec3& n, const vec3& wiW) {
  return albedo(c.sc.SURFACE_SPECULAR_REFLECTANCE(v3(c.P.surfaceSpecAlbedoRGB), X, n, wiW), c.cmf);
}
SD_FN Rad subsurf_albedo(const Ctx& c, const vec3& X, const vec3& n) {
  return albedo(c.sc.SUBSURFACE_ALBEDO(v3(c.P.subsurfaceAlbedoRGB), X, n), c.cmf);
}
SD_FN Rad surf_eval(const Ctx& c, const vec3& X, const Frame& f, const vec3& wiL, const vec3& woL) {
  if (wiL.z < 0.0f) return Rad(0.0f);
  vec3 wiW = to_world(wiL, f);
  Rad dif = (1.0f - c.P.subsurface) * surf_diffuse(c, X, f.n, wiW);
  Rad spe = surf_specular(c, X, f.n, wiW);
  float ior = c.P.surfaceIor;
  float alpha = c.sc.SURFACE_ROUGHNESS(c.P.surfaceRoughness, X, f.n);
  float Fr = fresnel_dielectric(woL.z, ior);
  vec3 h = glsl::normalize(woL + wiL);
  float D = beckmann_D(h, alpha);
  float G = smith_g2(wiL, woL, h, alpha);
  Rad fr = Fr * spe * D * G / fmaxf(4.0f * fabsf(woL.z) * fabsf(wiL.z), kDenomTol);
  float E = fresnel_dielectric(wiL.z, ior);
  fr += (1.0f - E) * dif / kPi;
  return fr;
}
SD_FN float surf_pdf(const Ctx& c, const vec3& X, const Frame& f, const vec3& wiL, const vec3& woL) {
  if (wiL.z < 0.0f) return kPdfEps;
  vec3 wiW = to_world(wiL, f);
  Rad dif = (1.0f - c.P.subsurface) * surf_diffuse(c, X, f.n, wiW);
  Rad spe = surf_specular(c, X, f.n, wiW);
  float E = fresnel_dielectric(fabsf(wiL.z), c.P.surfaceIor);
  float ws = E * avg(spe);
  float wd = (1.0f - E) * avg(dif);
  float pspec = ws / fmaxf(ws + wd, kDenomTol);
  float alpha = c.sc.SURFACE_ROUGHNESS(c.P.surfaceRoughness, X, f.n);
  float pd = pdf_cosine(woL);
  vec3 h = safe_normalize(woL + wiL);
  float jac = 1.0f / fmaxf(fabsf(4.0f * glsl::dot(wiL, h)), kDenomTol);
  float ps = beckmann_pdf(h, alpha) * jac;
  return pspec * ps + (1.0f - pspec) * pd;
}
SD_FN Rad surf_sample(const Ctx& c, const vec3& X, const Frame& f, const vec3& wiL, vec3& woL, float& pdfOut, Rng& g) {
  if (wiL.z < 0.0f) return Rad(0.0f);
  vec3 wiW = to_world(wiL, f);
  Rad dif = (1.0f - c.P.subsurface) * surf_diffuse(c, X, f.n, wiW);
  Rad spe = surf_specular(c, X, f.n, wiW);
  float ior = c.P.surfaceIor;
  float alpha = c.sc.SURFACE_ROUGHNESS(c.P.surfaceRoughness, X, f.n);
  float E = fresnel_dielectric(fabsf(wiL.z), ior);
  float ws = E * avg(spe);
  float wd = (1.0f - E) * avg(dif);
  float pspec = ws / fmaxf(ws + wd, kDenomTol);
  if (rand01(g) >= pspec) {
    woL = sample_cosine(g, pdfOut);
    pdfOut *= (1.0f - pspec);
    return (1.0f - E) * dif / kPi;
  }
  vec3 m = beckmann_sample(g, alpha);
  woL = -wiL + 2.0f * glsl::dot(wiL, m) * m;
  pdfOut = pspec;
  if (woL.z < kDenomTol) return Rad(0.0f);
  float D = beckmann_D(m, alpha);
  float G = smith_g2(wiL, woL, m, alpha);
  float Fr = fresnel_dielectric(fabsf(wiL.z), ior);
  Rad fr = Fr * spe * D * G / fmaxf(4.0f * fabsf(woL.z) * fabsf(wiL.z), kDenomTol);
  float jac = 1.0f / fmaxf(fabsf(4.0f * glsl::dot(wiL, m)), kDenomTol);
  pdfOut *= beckmann_pdf(m, alpha) * jac;
  return fr;
}
#endif  // HAS_SURFACE

SD_FN Rad bsdf_eval(const Ctx& c, const vec3& X, const Frame& f, const vec3& wiL, const vec3& woL, int mat) {
#ifdef HAS_SURFACE
  if (mat == MAT_SURFA) return surf_eval(c, X, f, wiL, woL);
#endif
#ifdef HAS_METAL
  if (mat == MAT_METAL) return metal_eval(c, X, f, wiL, woL);
#endif
#ifdef HAS_DIELECTRIC
  if (mat == MAT_DIELE) return diele_eval(c, X, f, wiL, woL, true);
#endif
  return Rad(0.0f);
}
SD_FN float bsdf_pdf(const Ctx& c, const vec3& X, const Frame& f, const vec3& wiL, const vec3& woL, int mat) {
#ifdef HAS_SURFACE
  if (mat == MAT_SURFA) return surf_pdf(c, X, f, wiL, woL);
#endif
#ifdef HAS_METAL
  if (mat == MAT_METAL) return metal_pdf(c, X, f, wiL, woL);
#endif
#ifdef HAS_DIELECTRIC
  if (mat == MAT_DIELE) return diele_pdf(c, X, f, wiL, woL, true);
#endif
  return 0.0f;
}
SD_FN Rad bsdf_sample(const Ctx& c, const vec3& X, const Frame& f, const vec3& wiL, int mat, vec3& woL, float& pdf, Rng& g) {
#ifdef HAS_SURFACE
  if (mat == MAT_SURFA) return surf_sample(c, X, f, wiL, woL, pdf, g);
#endif
#ifdef HAS_METAL
  if (mat == MAT_METAL) return metal_sample(c, X, f, wiL, woL, pdf, g);
#endif
#ifdef HAS_DIELECTRIC
  if (mat == MAT_DIELE) return diele_sample(c, X, f, wiL, true, woL, pdf, g);
#endif
  return Rad(0.0f);
}

// ---- homogeneous atmosphere coefficients (PT:856-874) ---------------------------------------------
SD_FN Rad vol_scattering(const Ctx& c) {
  return albedo(v3(c.P.atmosphereScatteringCoeffRGB) / (c.P.atmosphereMFP * c.P.lengthScale), c.cmf);
}
SD_FN Rad vol_extinction(const Ctx& c) {
  return albedo(v3(c.P.atmosphereExtinctionCoeffRGB) / (c.P.atmosphereMFP * c.P.lengthScale), c.cmf);
}
#ifdef HAS_VOLUME_EMISSION
SD_FN Rad vol_emission(const Ctx& c, const vec3& X) {
  return albedo(c.sc.VOLUME_EMISSION(v3(c.P.volumeEmissionColorRGB) * c.P.volumeEmission, X), c.cmf);
}
#endif

// ---- sphere tracing (PT:881-920) ------------------------------------------------------------------
struct Hit {
  vec3 p;
  int mat;
  bool hit;
};
// Marches along `dir` by the smallest unsigned distance to any of the scene's SDFs; a hit is a
// distance below minLengthScale, tested in the order surface, metal, dielectric. Not inlined (it
// is called from every tracing site); it builds its own scene instance so the SDF code and the
// scene's INIT() state live in registers, with uniforms read from the constant bank.
__device__ __noinline__ Hit march_ray(int job, vec3 start, vec3 dir, float maxDist) {
  const SnellyParams& P = c_params[job];
  Scene sc(uniforms_of(job));
  sc.INIT();
  Hit h;
  h.mat = MAT_INVAL;
  h.hit = false;
  const float minMarch = P.minLengthScale;
  float sdf = 1.0e20f;
#ifdef HAS_SURFACE
  sdf = fminf(sdf, fabsf(sc.SDF_SURFACE(start)));
#endif
#ifdef HAS_METAL
  sdf = fminf(sdf, fabsf(sc.SDF_METAL(start)));
#endif
#ifdef HAS_DIELECTRIC
  sdf = fminf(sdf, fabsf(sc.SDF_DIELECTRIC(start)));
#endif
  const float sgn = glsl::sign(sdf);
  float t = sgn * sdf;
  if (fabsf(t) >= maxDist) return h;
  for (int n = 0; n < MAX_MARCH_STEPS; ++n) {
    vec3 p = start + t * dir;
    sdf = 1.0e20f;
    // every SDF, then the hit: the first of surface, metal, dielectric below the threshold (the
    // reference returns at the first, PT:906-912; the others' values are not used then)
    int m = MAT_INVAL;
#ifdef HAS_DIELECTRIC
    const float d3 = fabsf(sc.SDF_DIELECTRIC(p));
    m = d3 < minMarch ? MAT_DIELE : m;
    sdf = fminf(sdf, d3);
#endif
#ifdef HAS_METAL
    const float d2 = fabsf(sc.SDF_METAL(p));
    m = d2 < minMarch ? MAT_METAL : m;
    sdf = fminf(sdf, d2);
#endif
#ifdef HAS_SURFACE
    const float d1 = fabsf(sc.SDF_SURFACE(p));
    m = d1 < minMarch ? MAT_SURFA : m;
    sdf = fminf(sdf, d1);
#endif
    if (m != MAT_INVAL) {
      h.mat = m;
      h.p = start + t * dir;
      h.hit = true;
      return h;
    }
    t += sgn * sdf;
    if (fabsf(t) >= maxDist) return h;
  }
  // Out of steps: a hit when maxStepsIsMiss is off, at the zero-initialised position (PT:919).
  h.hit = !P.maxStepsIsMiss;
  return h;
}

// Central-difference SDF gradient of the hit material (PT:922-940).
__device__ __noinline__ vec3 sdf_normal(int job, vec3 p, int mat) {
  const SnellyParams& P = c_params[job];
  Scene sc(uniforms_of(job));
  sc.INIT();
  const float e = 2.0f * P.minLengthScale;
  vec3 xp = p + vec3(e, 0.0f, 0.0f), xn = p - vec3(e, 0.0f, 0.0f);
  vec3 yp = p + vec3(0.0f, e, 0.0f), yn = p - vec3(0.0f, e, 0.0f);
  vec3 zp = p + vec3(0.0f, 0.0f, e), zn = p - vec3(0.0f, 0.0f, e);
  vec3 N(0.0f);
#ifdef HAS_SURFACE
  if (mat == MAT_SURFA)
    N = vec3(sc.SDF_SURFACE(xp) - sc.SDF_SURFACE(xn), sc.SDF_SURFACE(yp) - sc.SDF_SURFACE(yn),
             sc.SDF_SURFACE(zp) - sc.SDF_SURFACE(zn));
#endif
#ifdef HAS_METAL
  if (mat == MAT_METAL)
    N = vec3(sc.SDF_METAL(xp) - sc.SDF_METAL(xn), sc.SDF_METAL(yp) - sc.SDF_METAL(yn),
             sc.SDF_METAL(zp) - sc.SDF_METAL(zn));
#endif
#ifdef HAS_DIELECTRIC
  if (mat == MAT_DIELE)
    N = vec3(sc.SDF_DIELECTRIC(xp) - sc.SDF_DIELECTRIC(xn), sc.SDF_DIELECTRIC(yp) - sc.SDF_DIELECTRIC(yn),
             sc.SDF_DIELECTRIC(zp) - sc.SDF_DIELECTRIC(zn));
#endif
  if (mat == MAT_INVAL) return N;
  return safe_normalize(N);
}

#ifdef HAS_NORMALMAP
// PT:943-967
SD_FN vec3 perturb_normal(const Ctx& c, const vec3& X, const Frame& f, int mat) {
#ifdef HAS_SURFACE_NORMALMAP
  if (mat == MAT_SURFA) return to_world(glsl::normalize(c.sc.SURFACE_NORMAL_MAP(X, f.n)), f);
#endif
#ifdef HAS_METAL_NORMALMAP
  if (mat == MAT_METAL) return to_world(glsl::normalize(c.sc.METAL_NORMAL_MAP(X, f.n)), f);
#endif
#ifdef HAS_DIELECTRIC_NORMALMAP
  if (mat == MAT_DIELE) return to_world(glsl::normalize(c.sc.DIELECTRIC_NORMAL_MAP(X, f.n)), f);
#endif
  return f.n;
}
#endif

// ---- atmosphere slab (PT:971-1026) --------------------------------------------------------------
#if defined(HAS_ATMOSPHERE) || defined(HAS_HETERO_VOLUME)
SD_FN bool atmosphere_segment(const Ctx& c, const vec3& p, const vec3& d, float len, float& t0, float& t1) {
  vec3 inv = 1.0f / d;
  vec3 lo = (v3(c.P.atmosphereBoundsMin) * c.P.lengthScale - p) * inv;
  vec3 hi = (v3(c.P.atmosphereBoundsMax) * c.P.lengthScale - p) * inv;
  vec3 mn = glsl::min(lo, hi);
  hi = lo + hi - mn;
  lo = mn;
  bool hit = !(lo.x > hi.y || lo.y > hi.x || lo.x > hi.z || lo.z > hi.x || lo.y > hi.z || lo.z > hi.y);
  t0 = fmaxf(fmaxf(lo.x, lo.y), lo.z);
  t1 = fminf(fminf(hi.x, hi.y), hi.z);
  if (!hit) return false;
  t0 = fmaxf(0.0f, t0);
  if (t1 < 0.0f || len < t0) return false;
  t1 = fminf(len, t1);
  return true;
}
#endif

#ifdef HAS_HETERO_VOLUME
// ---- heterogeneous medium (an extension of this build) ----------------------------------------
// The reference appends default bodies for VOLUME_EXTINCTION, VOLUME_EXTINCTION_MAX,
// VOLUME_SCATTERING_COLOR, VOLUME_ABSORPTION_COLOR and VOLUME_ANISOTROPY (js/renderer.js:258-262)
// but its path tracer never calls them. When a scene defines VOLUME_EXTINCTION itself, the
// atmosphere's box holds a medium with grey extinction VOLUME_EXTINCTION(e, X), e the atmosphere's
// extinction per unit length (the rgb mean of atmosphereExtinctionCoeffRGB / (atmosphereMFP *
// lengthScale)), bounded by the majorant VOLUME_EXTINCTION_MAX(e); single-scattering albedo
// sc / (sc + ab) of the two colour hooks (given the atmosphere's scattering and absorption
// coefficients), projected on the beam's wavelength; Henyey-Greenstein phase function with
// g = VOLUME_ANISOTROPY(atmosphereAnisotropy, X). It takes the homogeneous atmosphere's place.
// Collisions are found by delta tracking with the path's random numbers; transmittance along
// shadow rays is estimated by ratio tracking with random numbers hashed from the shadow ray's own
// origin and direction, so the estimate does not depend on when the ray is resolved.
#define HV_MAX_STEPS 4096
SD_FN float hv_extinction_ui(const Ctx& c) {
  const vec3 e = v3(c.P.atmosphereExtinctionCoeffRGB);
  return (e.x + e.y + e.z) / 3.0f / (c.P.atmosphereMFP * c.P.lengthScale);
}
// An xorshift-multiply integer mix (two rounds), for the ratio-tracking streams.
SD_FN unsigned hv_mix(unsigned x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
// The seed of a shadow ray's stream: its origin and direction with the 10 lowest mantissa bits
// dropped (about 1e-4 relative), so that builds whose arithmetic differs in the last bits (the
// CPU oracle's transcendentals) draw the same numbers for the same ray.
SD_FN unsigned hv_seed(const vec3& p, const vec3& d) {
  unsigned h = 0x2545f491u;
  const float v[6] = {p.x, p.y, p.z, d.x, d.y, d.z};
  for (int k = 0; k < 6; ++k) h = hv_mix(h ^ ((unsigned)__float_as_int(v[k]) & 0xfffffc00u));
  return h;
}
SD_FN float hv_uniform(unsigned& h) {  // in [0, 1), 24 bits
  h = hv_mix(h + 0x9e3779b9u);
  return float(h >> 8) * (1.0f / 16777216.0f);
}
// Ratio-tracking estimate of the medium's transmittance along [p, p + len d] (Russian roulette
// once it falls below 0.1 keeps it unbiased and bounded).
SD_FN float hv_transmittance(const Ctx& c, const vec3& p, const vec3& d, float len) {
  float t0, t1;
  if (!atmosphere_segment(c, p, d, len, t0, t1)) return 1.0f;
  const float e = hv_extinction_ui(c);
  const float mx = c.sc.VOLUME_EXTINCTION_MAX(e);
  if (!(mx > 0.0f)) return 1.0f;
  unsigned h = hv_seed(p, d);
  float T = 1.0f, t = t0;
  for (int k = 0; k < HV_MAX_STEPS; ++k) {
    t -= logf(1.0f - hv_uniform(h)) / mx;
    if (t >= t1) break;
    T *= 1.0f - glsl::clamp(c.sc.VOLUME_EXTINCTION(e, p + t * d) / mx, 0.0f, 1.0f);
    if (T < 0.1f) {
      if (hv_uniform(h) < 0.5f) return 0.0f;
      T *= 2.0f;
    }
  }
  return T;
}
// Delta tracking along [p, p + len d] with the path's random numbers: true and the collision
// point when the path scatters in the medium before the segment's end.
SD_FN bool hv_collision(const Ctx& c, const vec3& p, const vec3& d, float len, Rng& g, vec3& ps) {
  float t0, t1;
  if (!atmosphere_segment(c, p, d, len, t0, t1)) return false;
  const float e = hv_extinction_ui(c);
  const float mx = c.sc.VOLUME_EXTINCTION_MAX(e);
  if (!(mx > 0.0f)) return false;
  float t = t0;
  for (int k = 0; k < HV_MAX_STEPS; ++k) {
    t -= logf(1.0f - rand01(g)) / mx;
    if (t >= t1) return false;
    const vec3 x = p + t * d;
    if (rand01(g) * mx < c.sc.VOLUME_EXTINCTION(e, x)) {
      ps = x;
      return true;
    }
  }
  return false;
}
// Henyey-Greenstein direction about `dir` by inversion of its distribution (pdf hg_phase).
SD_FN vec3 hv_sample_hg(const vec3& dir, float g, Rng& rng) {
  float ct;
  const float u = rand01(rng);
  if (fabsf(g) < 1.0e-3f) {
    ct = 1.0f - 2.0f * u;
  } else {
    const float q = (1.0f - g * g) / (1.0f - g + 2.0f * g * u);
    ct = glsl::clamp((1.0f + g * g - q * q) / (2.0f * g), -1.0f, 1.0f);
  }
  const float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
  const float phi = 2.0f * kPi * rand01(rng);
  Frame f = make_frame(dir);
  return ct * dir + st * (cosf(phi) * f.t + sinf(phi) * f.b);
}
// Uniform direction on the sphere (pdf 1 / 4 pi).
SD_FN vec3 hv_sample_sphere(Rng& g) {
  const float z = 1.0f - 2.0f * rand01(g);
  const float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
  const float phi = 2.0f * kPi * rand01(g);
  return vec3(r * cosf(phi), r * sinf(phi), z);
}
#endif

// Transmittance along a segment known to be free of geometry (PT:1003-1026). `medium`: include
// the heterogeneous medium's ratio-tracking estimate (shadow rays); the path's own segments leave
// it out, since delta tracking has already decided whether the path crosses the medium.
SD_FN Rad transmittance_free(const Ctx& c, const vec3& p, const vec3& d, float len, bool medium = true) {
  Rad Tr = Rad(1.0f);
#ifdef HAS_HETERO_VOLUME
  if (medium) Tr = Rad(hv_transmittance(c, p, d, len));
#else
  (void)medium;
#endif
#ifdef HAS_ATMOSPHERE
  Rad ext = vol_extinction(c);
  if (glsl::length(ext) == 0.0f) return Rad(1.0f);
  float t0, t1;
  if (!atmosphere_segment(c, p, d, len, t0, t1)) return Rad(1.0f);
  Tr = glsl::exp(-((t1 - t0) * ext));
#endif
#ifdef HAS_FOG
  if (c.P.fogEnable) {
    vec3 fa = vec3(1.0f) - v3(c.P.fogTint);
    vec3 od = c.P.fogMaxOpticalDepth * (vec3(1.0f) - glsl::exp(-len * fa / c.P.fogMFP));
    Tr *= glsl::exp(-albedo(od, c.cmf));
  }
#endif
  return Tr;
}
// Zero if geometry blocks the segment (PT:1030-1039).
SD_FN Rad transmittance(const Ctx& c, const vec3& p, const vec3& d, float len) {
  if (march_ray(c.job, p, d, len).hit) return Rad(0.0f);
  return transmittance_free(c, p, d, len);
}

// ---- lights (PT:1051-1212) ---------------------------------------------------------------------
SD_FN vec3 sky_rgb(const Ctx& c, const vec3& dir) {
  const SnellyParams& P = c.P;
  float rot_theta = kPi * P.envMapThetaRotation / 180.0f;
  vec3 pole(sinf(rot_theta), cosf(rot_theta), 0.0f);
  vec3 rgb(1.0f);
  if (P.haveEnvMap) {
    float rot_phi = kPi * P.envMapPhiRotation / 180.0f;
    vec3 dl = to_local(dir, make_frame(pole));
    float phi = atan2f(dl.y, dl.x) + kPi + rot_phi;
    phi -= 2.0f * kPi * glsl::s_floor(phi / (2.0f * kPi));
    float theta = acosf(dl.z);
    glsl::sampler2D env{P.envMap, P.envMapW, P.envMapH, 3, 2, 1, 1};
    vec4 tx = glsl::texture(env, vec2(phi / (2.0f * kPi), theta / kPi));
    rgb = vec3(tx.x, tx.y, tx.z);
  }
  float t = glsl::dot(dir, pole);
  float tt = P.envMapTransitionAngle / 180.0f;
  rgb *= P.skyPower * glsl::mix(v3(P.skyTintDown), v3(P.skyTintUp), glsl::smoothstep(-tt, tt, t));
  return rgb;
}
SD_FN Rad sky_radiance(const Ctx& c, const vec3& dir) { return albedo(sky_rgb(c, dir), c.cmf); }

SD_FN vec3 sample_sun_dir(const Ctx& c, Rng& g, float& pdf) {
  float tmax = c.P.sunAngularSize * kPi / 180.0f;
  float th = tmax * sqrtf(rand01(g));
  float ct = cosf(th);
  float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
  float phi = 2.0f * kPi * rand01(g);
  float cp = cosf(phi), sp = sinf(phi);
  float sa = 2.0f * kPi * (1.0f - cosf(tmax));
  pdf = 1.0f / sa;
  return to_world(vec3(st * cp, st * sp, ct), c.sun);
}
SD_FN Rad sun_radiance(const Ctx& c, const vec3& dir) {
  float tmax = c.P.sunAngularSize * kPi / 180.0f;
  if (glsl::dot(dir, v3(c.P.sunDir)) < cosf(tmax)) return Rad(0.0f);
  return albedo(c.P.sunPower * v3(c.P.sunColor), c.cmf);
}

#ifdef HAS_SPHERE_LIGHT
SD_FN Rad sphere_light_hit(const Ctx& c, const vec3& p, const vec3& d, vec3& pHit) {
  const SnellyParams& P = c.P;
  vec3 m = p - v3(P.sphereLightPosition);
  float b = glsl::dot(m, d);
  float cc = glsl::dot(m, m) - P.sphereLightRadius * P.sphereLightRadius;
  if (cc > 0.0f && b > 0.0f) return Rad(0.0f);
  float disc = b * b - cc;
  if (disc < 0.0f) return Rad(0.0f);
  float t = fmaxf(-b - sqrtf(disc), 0.0f);
  pHit = p + t * d;
  return albedo(P.sphereLightPower * v3(P.sphereLightColor), c.cmf);
}
SD_FN Rad sample_sphere_light(const Ctx& c, Rng& g, const vec3& p, vec3& pHit, float& pdfDir) {
  const SnellyParams& P = c.P;
  if (P.sphereLightPower < kRadianceEps) return Rad(0.0f);
  vec3 cp = glsl::normalize(p - v3(P.sphereLightPosition));
  Frame hf = make_frame(cp);
  vec3 vW = to_world(sample_hemisphere_uniform(g), hf);
  float pdfA = 1.0f / (2.0f * kPi * P.sphereLightRadius * P.sphereLightRadius);
  pHit = v3(P.sphereLightPosition) + P.sphereLightRadius * vW;
  vec3 dh = pHit - p;
  float d2 = glsl::dot(dh, dh);
  dh = glsl::normalize(dh);
  vec3 nh = glsl::normalize(pHit - v3(P.sphereLightPosition));
  float ct = fabsf(glsl::dot(nh, dh));
  pdfDir = pdfA * d2 / fmaxf(kDenomTol, ct);
  return albedo(P.sphereLightPower * v3(P.sphereLightColor), c.cmf);
}
#endif

// Occlusion-scaled incident radiance (PT:1237 and siblings).
SD_FN Rad shadow_scale(const Ctx& c, const Rad& Li, const Rad& Tr) {
  return Li * glsl::abs(Rad(1.0f) - c.P.shadowStrength * (Rad(1.0f) - Tr));
}

}  // namespace sdev
