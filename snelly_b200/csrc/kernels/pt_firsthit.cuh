// pt_firsthit.cuh - the reference's first-hit render modes: surface normals
// (shaders/normals-fragment-shader.glsl, cited NM:line), ambient occlusion under the sky and sun
// (shaders/ao-fragment-shader.glsl, AO:line) and first-hit distance and material
// (shaders/pick-fragment-shader.glsl, PK:line), one thread per pixel.
//
// These programs have their own marcher (traceDistance: the distance starts at zero and the hit
// point is taken after the loop) and use normalize() where the path tracer uses safe_normalize();
// both are followed here.
#pragma once
#include "pt_integrator.cuh"
#include "pt_launch.h"

namespace sdev {

// NM:70-114, AO:100-143, PK:58-108
SD_FN bool trace_distance(Scene& sc, const SnellyParams& P, const vec3& start, const vec3& dir, float maxDist, vec3& hit,
                          int& mat) {
  mat = MAT_INVAL;
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
  float t = 0.0f;
  int iters = 0;
  for (int n = 0; n < MAX_MARCH_STEPS; n++) {
    t += sgn * sdf;
    if (t >= maxDist) break;
    vec3 p = start + t * dir;
    sdf = 1.0e20f;
    bool stop = false;
#ifdef HAS_SURFACE
    {
      float d = fabsf(sc.SDF_SURFACE(p));
      if (d < minMarch) { mat = MAT_SURFA; stop = true; }
      else sdf = fminf(sdf, d);
    }
#endif
#ifdef HAS_METAL
    if (!stop) {
      float d = fabsf(sc.SDF_METAL(p));
      if (d < minMarch) { mat = MAT_METAL; stop = true; }
      else sdf = fminf(sdf, d);
    }
#endif
#ifdef HAS_DIELECTRIC
    if (!stop) {
      float d = fabsf(sc.SDF_DIELECTRIC(p));
      if (d < minMarch) { mat = MAT_DIELE; stop = true; }
      else sdf = fminf(sdf, d);
    }
#endif
    if (stop) break;
    iters++;
  }
  hit = start + t * dir;
  if (t >= maxDist) return false;
  if (P.maxStepsIsMiss && iters >= MAX_MARCH_STEPS) return false;
  return true;
}

// NM:134-150 (normalize, not safe_normalize; no branch for an invalid material: zero vector)
SD_FN vec3 fh_normal(Scene& sc, const SnellyParams& P, const vec3& p, int mat) {
  const float e = 2.0f * P.minLengthScale;
  vec3 xp = p + vec3(e, 0.0f, 0.0f), xn = p - vec3(e, 0.0f, 0.0f);
  vec3 yp = p + vec3(0.0f, e, 0.0f), yn = p - vec3(0.0f, e, 0.0f);
  vec3 zp = p + vec3(0.0f, 0.0f, e), zn = p - vec3(0.0f, 0.0f, e);
#ifdef HAS_SURFACE
  if (mat == MAT_SURFA)
    return glsl::normalize(vec3(sc.SDF_SURFACE(xp) - sc.SDF_SURFACE(xn), sc.SDF_SURFACE(yp) - sc.SDF_SURFACE(yn),
                                sc.SDF_SURFACE(zp) - sc.SDF_SURFACE(zn)));
#endif
#ifdef HAS_METAL
  if (mat == MAT_METAL)
    return glsl::normalize(vec3(sc.SDF_METAL(xp) - sc.SDF_METAL(xn), sc.SDF_METAL(yp) - sc.SDF_METAL(yn),
                                sc.SDF_METAL(zp) - sc.SDF_METAL(zn)));
#endif
#ifdef HAS_DIELECTRIC
  if (mat == MAT_DIELE)
    return glsl::normalize(vec3(sc.SDF_DIELECTRIC(xp) - sc.SDF_DIELECTRIC(xn), sc.SDF_DIELECTRIC(yp) - sc.SDF_DIELECTRIC(yn),
                                sc.SDF_DIELECTRIC(zp) - sc.SDF_DIELECTRIC(zn)));
#endif
  return vec3(0.0f);
}

SD_FN Frame fh_basis(const vec3& n) {
  Frame f;
  f.n = n;
  if (fabsf(n.z) < fabsf(n.x)) f.t = vec3(n.z, 0.0f, -n.x);
  else f.t = vec3(0.0f, n.z, -n.y);
  f.t = glsl::normalize(f.t);
  f.b = glsl::cross(n, f.t);
  return f;
}

// Primary ray of the first-hit programs (NM:270-291, AO:373-393): as the path tracer's, with
// normalize() for the directions.
SD_FN void fh_primary_ray(const SnellyParams& P, const vec2& pixel, Rng& g, vec3& start, vec3& dir) {
  vec2 ndc = -1.0f + 2.0f * (pixel / vec2(P.resolution[0], P.resolution[1]));
  float fh = tanf(0.5f * glsl::radians(P.camFovy));
  float fw = P.camAspect * fh;
  vec3 s = -fw * ndc.x * v3(P.camX) + fh * ndc.y * v3(P.camY);
  dir = glsl::normalize(v3(P.camDir) + s);
  if (P.camAperture <= 0.0f) {
    start = v3(P.camPos);
    return;
  }
  vec3 focal = v3(P.camPos) + P.camFocalDistance * dir / glsl::dot(dir, v3(P.camDir));
  float rad = P.camAperture * sqrtf(rand01(g));
  float th = 2.0f * kPi * rand01(g);
  vec3 lens = v3(P.camPos) + rad * (-v3(P.camX) * cosf(th) + v3(P.camY) * sinf(th));
  start = lens;
  dir = glsl::normalize(focal - lens);
}

// AO:423-427: the ambient-occlusion program honours a scene's CONSTRUCT_PRIMARY_RAY hook (the
// normals program does not).
SD_FN void fh_camera(const Ctx& c, const vec2& pixel, Rng& g, vec3& start, vec3& dir) {
#ifdef HAS_CUSTOM_CAMERA
  primary_ray_hook(c, pixel, g, start, dir);
#else
  fh_primary_ray(c.P, pixel, g, start, dir);
#endif
}

// NM:248-268: the normals program's environment term (XYZ); its rotation uniform is never set by
// the host, i.e. zero.
SD_FN vec3 fh_env_xyz(const SnellyParams& P, const vec3& dir) {
  if (P.haveEnvMap) {
    float phi = atan2f(dir.x, dir.z) + kPi;
    phi -= 2.0f * kPi * glsl::s_floor(phi / (2.0f * kPi));
    float theta = acosf(dir.y);
    glsl::sampler2D env{P.envMap, P.envMapW, P.envMapH, 3, 2, 1, 1};
    vec4 tx = glsl::texture(env, vec2(phi / (2.0f * kPi), theta / kPi));
    return rgb_to_xyz(vec3(tx.x, tx.y, tx.z) * P.skyPower);
  }
  return P.skyPower * vec3(1.0f);
}

// AO:265-296: the sky term of the AO program (RGB; its basis uses normalize()).
SD_FN vec3 fh_sky_rgb(const SnellyParams& P, const vec3& dir) {
  float rot_theta = kPi * P.envMapThetaRotation / 180.0f;
  vec3 pole(sinf(rot_theta), cosf(rot_theta), 0.0f);
  vec3 rgb(1.0f);
  if (P.haveEnvMap) {
    float rot_phi = kPi * P.envMapPhiRotation / 180.0f;
    vec3 dl = to_local(dir, fh_basis(pole));
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

// One frame of the normals program (NM:293-346): XYZ.
SD_FN vec3 fh_normals(const Ctx& c, const vec2& pixel, Rng& g) {
  const SnellyParams& P = c.P;
  vec3 xyz(0.0f);
  for (int n = 0; n < MAX_SAMPLES_PER_FRAME; ++n) {
    float jx = rand01(g);
    float jy = rand01(g);
    vec2 pj = pixel + (-0.5f + vec2(jx, jy));
    vec3 start, dir;
    fh_primary_ray(P, pj, g, start, dir);
    vec3 pW;
    int mat;
    if (trace_distance(c.sc, P, start, dir, P.maxLengthScale, pW, mat)) {
      vec3 nW = fh_normal(c.sc, P, pW, mat);
#ifdef HAS_SURFACE_NORMALMAP
      vec3 ngW = nW;
      Frame b = fh_basis(nW);
      if (mat == MAT_SURFA) nW = to_world(glsl::normalize(c.sc.SURFACE_NORMAL_MAP(pW, b.n)), b);
      if (glsl::dot(nW, dir) > 0.0f && mat != MAT_DIELE) nW = 2.0f * ngW * glsl::dot(ngW, nW) - nW;
#endif
      xyz += rgb_to_xyz(0.5f * (nW + vec3(1.0f)));
    } else if (P.envMapVisible) {
      xyz += fh_env_xyz(P, dir);
    }
  }
  return xyz / float(MAX_SAMPLES_PER_FRAME);
}

// One frame of the ambient-occlusion program (AO:395-488): XYZ. Its radiance threshold is
// RADIANCE_EPSILON = 1e-5 (AO:62), ten times the path tracer's.
SD_FN vec3 fh_ao(const Ctx& c, const vec2& pixel, Rng& g) {
  const SnellyParams& P = c.P;
  const float kAoRadianceEps = 1.0e-5f;
  Frame sun = fh_basis(v3(P.sunDir));
  vec3 rgb(0.0f);
  for (int n = 0; n < MAX_SAMPLES_PER_FRAME; ++n) {
    float jx = rand01(g);
    float jy = rand01(g);
    vec2 pj = pixel + (-0.5f + vec2(jx, jy));
    vec3 start, dir;
    fh_camera(c, pj, g, start, dir);
    vec3 woW = -dir;
    vec3 pW;
    int mat;
    if (trace_distance(c.sc, P, start, dir, P.maxLengthScale, pW, mat)) {
      vec3 nW = fh_normal(c.sc, P, pW, mat);
      Frame b = fh_basis(nW);
#ifdef HAS_SURFACE_NORMALMAP
      if (mat == MAT_SURFA) nW = to_world(glsl::normalize(c.sc.SURFACE_NORMAL_MAP(pW, b.n)), b);
      b = fh_basis(nW);
#endif
      vec3 f = c.sc.SURFACE_DIFFUSE_REFLECTANCE(v3(P.surfaceDiffuseAlbedoRGB), pW, nW, woW) / kPi;
      vec3 Ld(0.0f);
      vec3 off = 3.0f * P.minLengthScale * nW;
      if (P.skyPower > kAoRadianceEps) {
        float pdf;
        vec3 woL = sample_cosine(g, pdf);
        vec3 wo = to_world(woL, b);
        vec3 Li = fh_sky_rgb(P, wo);
        vec3 h;
        int m;
        Li *= trace_distance(c.sc, P, pW + off, wo, P.maxLengthScale, h, m) ? 0.0f : 1.0f;
        Ld += f * Li / fmaxf(kPdfEps, pdf) * fabsf(glsl::dot(wo, nW));
      }
      if (P.sunPower > kAoRadianceEps) {
        float tmax = P.sunAngularSize * kPi / 180.0f;
        float th = tmax * sqrtf(rand01(g));
        float ct = cosf(th);
        float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
        float phi = 2.0f * kPi * rand01(g);
        float cp = cosf(phi), sp = sinf(phi);
        float pdf = 1.0f / (2.0f * kPi * (1.0f - cosf(tmax)));
        vec3 wo = to_world(vec3(st * cp, st * sp, ct), sun);
        vec3 Li(0.0f);
        if (to_local(wo, b).z >= 0.0f && glsl::dot(wo, v3(P.sunDir)) >= cosf(tmax)) Li = P.sunPower * v3(P.sunColor);
        if (avg(Li) > kAoRadianceEps) {
          vec3 h;
          int m;
          Li *= trace_distance(c.sc, P, pW + off, wo, P.maxLengthScale, h, m) ? 0.0f : 1.0f;
          Ld += f * Li / fmaxf(kPdfEps, pdf) * fabsf(glsl::dot(wo, nW));
        }
      }
      rgb += Ld;
    } else if (P.envMapVisible) {
      rgb += fh_sky_rgb(P, dir);
    }
  }
  rgb /= float(MAX_SAMPLES_PER_FRAME);
  return rgb_to_xyz(rgb);
}

// The pick program at one pixel (PK:114-151): first-hit distance along the pinhole ray through
// the pixel, or maxLengthScale, and the material id.
SD_FN vec2 fh_pick(const Ctx& c, const vec2& pixel) {
  const SnellyParams& P = c.P;
  vec2 ndc = -1.0f + 2.0f * (pixel / vec2(P.resolution[0], P.resolution[1]));
  float fh = tanf(0.5f * glsl::radians(P.camFovy));
  float fw = P.camAspect * fh;
  vec3 s = -fw * ndc.x * v3(P.camX) + fh * ndc.y * v3(P.camY);
  vec3 dir = glsl::normalize(v3(P.camDir) + s);
  vec3 start = v3(P.camPos);
  vec3 pW;
  int mat;
  bool hit = trace_distance(c.sc, P, start, dir, P.maxLengthScale, pW, mat);
  float d = hit ? glsl::length(pW - start) : P.maxLengthScale;
  return vec2(d, float(mat));
}

}  // namespace sdev

// One frame of a first-hit mode (JobRec.mode) for every pixel of the job.
extern "C" __global__ void __launch_bounds__(SNELLY_BLOCK) snelly_firsthit(const JobRec* __restrict__ jobs,
                                                                        const int* __restrict__ block_start, int njobs,
                                                                        const SnellyParams* __restrict__ gparams) {
  using namespace sdev;
  int j = job_of_block(block_start, njobs, blockIdx.x);
  const JobRec& J = jobs[j];
  long long i = (long long)(blockIdx.x - block_start[j]) * blockDim.x + threadIdx.x + J.pixel_begin;
  if (i >= (long long)J.pixel_begin + J.pixel_count) return;
  const int slot = J.slot;
  const SnellyParams& P = c_params[slot];
  const int W = J.width;
  const vec2 pixel = J.pick_at ? vec2(J.pick_x, J.pick_y) : vec2(float(int(i % W)) + 0.5f, float(int(i / W)) + 0.5f);
  uint4 r4 = J.rng[i];
  Rng g;
  g.s[0] = r4.x; g.s[1] = r4.y; g.s[2] = r4.z; g.s[3] = r4.w;
  if (J.mode == JOB_MODE_AO) {
#ifdef INTERACTIVE_MODE
    if (rand01(g) < P.skipProbability) {
      J.rng[i] = make_uint4(g.s[0], g.s[1], g.s[2], g.s[3]);
      return;
    }
#endif
  }
  Scene sc(uniforms_of(slot));
  sc.INIT();
  Ctx c{P, gparams + slot, sc, slot, 0.0f, vec3(0.0f), Frame()};
  if (J.mode == JOB_MODE_PICK) {
    vec2 r = fh_pick(c, pixel);
    J.acc[i] = make_float4(r.x, r.y, 0.0f, 1.0f);
    J.comp[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    return;
  }
  vec3 xyz = J.mode == JOB_MODE_AO ? fh_ao(c, pixel, g) : fh_normals(c, pixel, g);
  J.rng[i] = make_uint4(g.s[0], g.s[1], g.s[2], g.s[3]);
  float4 s = J.acc[i], cp = J.comp[i];
  kahan_add(s, cp, xyz);
  J.acc[i] = s;
  J.comp[i] = cp;
}
