// pt_simple.cuh - the reference's simplified path tracer, renderMode 'ptsimple'
// (shaders/simplepathtracer-fragment-shader.glsl, cited SP:line): RGB radiance, the Surface
// material only (the metal and dielectric distance functions are not traced), sky and sun
// lights with MIS, the homogeneous fog model, subsurface random walks. One thread per pixel.
//
// It shares the building blocks of the spectral path tracer where the two programs agree (the RNG,
// bases, Beckmann and Fresnel formulas, cosine and Henyey-Greenstein sampling, the sky and sun
// models) and restates the rest from the simplified program.
#pragma once
#include "pt_integrator.cuh"
#include "pt_launch.h"

namespace sdev {

// SP:508-534: sphere tracing against the surface distance function only. Running out of steps
// reports a hit (unless maxStepsIsMiss) without a position: the caller's zero-initialised one.
SD_FN bool ps_trace(Scene& sc, const SnellyParams& P, const vec3& start, const vec3& dir, float maxDist, vec3& hit,
                    int& mat) {
  mat = MAT_INVAL;
  const float minMarch = P.minLengthScale;
  float sdf = 1.0e20f;
#ifdef HAS_SURFACE
  sdf = fminf(sdf, fabsf(sc.SDF_SURFACE(start)));
#endif
  const float sgn = glsl::sign(sdf);
  float t = sgn * sdf;
  if (fabsf(t) >= maxDist) return false;
  for (int n = 0; n < MAX_MARCH_STEPS; ++n) {
    const vec3 p = start + t * dir;
    sdf = 1.0e20f;
#ifdef HAS_SURFACE
    {
      float d = fabsf(sc.SDF_SURFACE(p));
      if (d < minMarch) {
        mat = MAT_SURFA;
        hit = start + t * dir;
        return true;
      }
      sdf = fminf(sdf, d);
    }
#endif
    t += sgn * sdf;
    if (fabsf(t) >= maxDist) return false;
  }
  return !P.maxStepsIsMiss;
}

// SP:536-549 (safe_normalize of the surface gradient; no material: the zero vector, where the
// reference function ends without a return value)
SD_FN vec3 ps_normal(Scene& sc, const SnellyParams& P, const vec3& p, int mat) {
#ifdef HAS_SURFACE
  if (mat == MAT_SURFA) {
    const float e = 2.0f * P.minLengthScale;
    vec3 xp = p + vec3(e, 0.0f, 0.0f), xn = p - vec3(e, 0.0f, 0.0f);
    vec3 yp = p + vec3(0.0f, e, 0.0f), yn = p - vec3(0.0f, e, 0.0f);
    vec3 zp = p + vec3(0.0f, 0.0f, e), zn = p - vec3(0.0f, 0.0f, e);
    return safe_normalize(vec3(sc.SDF_SURFACE(xp) - sc.SDF_SURFACE(xn), sc.SDF_SURFACE(yp) - sc.SDF_SURFACE(yn),
                               sc.SDF_SURFACE(zp) - sc.SDF_SURFACE(zn)));
  }
#endif
  return vec3(0.0f);
}

// SP:551-565
SD_FN vec3 ps_perturb(Scene& sc, const vec3& X, const Frame& b, int mat) {
#ifdef HAS_SURFACE_NORMALMAP
  if (mat == MAT_SURFA) return to_world(glsl::normalize(sc.SURFACE_NORMAL_MAP(X, b.n)), b);
#endif
  return b.n;
}

// SP:570-582: fog transmittance over a segment free of geometry
SD_FN vec3 ps_tr_free(const SnellyParams& P, float len) {
  vec3 Tr(1.0f);
#ifdef HAS_FOG
  if (P.fogEnable) {
    vec3 absorption = vec3(1.0f) - v3(P.fogTint);
    vec3 depth = P.fogMaxOpticalDepth * (vec3(1.0f) - glsl::exp(-len * absorption / P.fogMFP));
    Tr *= glsl::exp(-depth);
  }
#endif
  return Tr;
}

// SP:584-597
SD_FN vec3 ps_tr_segment(Scene& sc, const SnellyParams& P, const vec3& p, const vec3& dir, float len) {
  vec3 h(0.0f);
  int m;
  if (ps_trace(sc, P, p, dir, len, h, m)) return vec3(0.0f);
#ifdef HAS_FOG
  return ps_tr_free(P, len);
#else
  return vec3(1.0f);
#endif
}

// SP:599-604
SD_FN vec3 ps_inscatter(const SnellyParams& P, const vec3& Tr) {
  if (!P.fogEnable) return vec3(0.0f);
  return (1.0f - Tr) * v3(P.fogEmission);
}

// SP:688-694
SD_FN vec3 ps_sun_radiance(const SnellyParams& P, const vec3& dir) {
  float tmax = P.sunAngularSize * kPi / 180.0f;
  if (glsl::dot(dir, v3(P.sunDir)) < cosf(tmax)) return vec3(0.0f);
  return P.sunPower * v3(P.sunColor);
}

#ifdef HAS_SURFACE
SD_FN vec3 ps_diffuse(Scene& sc, const SnellyParams& P, const vec3& X, const vec3& n, const vec3& wiW) {
  return sc.SURFACE_DIFFUSE_REFLECTANCE(v3(P.surfaceDiffuseAlbedoRGB), X, n, wiW);
}
SD_FN vec3 ps_specular(Scene& sc, const SnellyParams& P, const vec3& X, const vec3& n, const vec3& wiW) {
  return sc.SURFACE_SPECULAR_REFLECTANCE(v3(P.surfaceSpecAlbedoRGB), X, n, wiW);
}

// SP:388-404
SD_FN vec3 ps_surf_eval(Scene& sc, const SnellyParams& P, const vec3& X, const Frame& f, const vec3& wiL,
                        const vec3& woL) {
  if (wiL.z < 0.0f) return vec3(0.0f);
  vec3 wiW = to_world(wiL, f);
  vec3 diffuse = (1.0f - P.subsurface) * ps_diffuse(sc, P, X, f.n, wiW);
  vec3 spec = ps_specular(sc, P, X, f.n, wiW);
  float ior = P.surfaceIor;
  float rough = sc.SURFACE_ROUGHNESS(P.surfaceRoughness, X, f.n);
  float Fr = fresnel_dielectric(woL.z, ior);
  vec3 h = glsl::normalize(woL + wiL);
  float D = beckmann_D(h, rough);
  float G = smith_g2(wiL, woL, h, rough);
  vec3 r = Fr * spec * D * G / fmaxf(4.0f * fabsf(woL.z) * fabsf(wiL.z), kDenomTol);
  float E = fresnel_dielectric(wiL.z, ior);
  r += (1.0f - E) * diffuse / kPi;
  return r;
}

// SP:406-424
SD_FN float ps_surf_pdf(Scene& sc, const SnellyParams& P, const vec3& X, const Frame& f, const vec3& wiL,
                        const vec3& woL) {
  if (wiL.z < 0.0f) return kPdfEps;
  vec3 wiW = to_world(wiL, f);
  vec3 diffuse = (1.0f - P.subsurface) * ps_diffuse(sc, P, X, f.n, wiW);
  vec3 spec = ps_specular(sc, P, X, f.n, wiW);
  float ior = P.surfaceIor;
  float E = fresnel_dielectric(fabsf(wiL.z), ior);
  float specW = E * avg(spec);
  float diffW = (1.0f - E) * avg(diffuse);
  float wsum = fmaxf(specW + diffW, kDenomTol);
  float specProb = specW / wsum;
  float rough = sc.SURFACE_ROUGHNESS(P.surfaceRoughness, X, f.n);
  float diffPdf = pdf_cosine(woL);
  vec3 h = safe_normalize(woL + wiL);
  float dwh = 1.0f / fmaxf(fabsf(4.0f * glsl::dot(wiL, h)), kDenomTol);
  float specPdf = beckmann_pdf(h, rough) * dwh;
  return specProb * specPdf + (1.0f - specProb) * diffPdf;
}

// SP:426-464
SD_FN vec3 ps_surf_sample(Scene& sc, const SnellyParams& P, const vec3& X, const Frame& f, const vec3& wiL, vec3& woL,
                          float& pdfOut, Rng& g) {
  if (wiL.z < 0.0f) return vec3(0.0f);
  vec3 wiW = to_world(wiL, f);
  vec3 diffuse = (1.0f - P.subsurface) * ps_diffuse(sc, P, X, f.n, wiW);
  vec3 spec = ps_specular(sc, P, X, f.n, wiW);
  float ior = P.surfaceIor;
  float rough = sc.SURFACE_ROUGHNESS(P.surfaceRoughness, X, f.n);
  float E = fresnel_dielectric(fabsf(wiL.z), ior);
  float specW = E * avg(spec);
  float diffW = (1.0f - E) * avg(diffuse);
  float wsum = fmaxf(specW + diffW, kDenomTol);
  float specProb = specW / wsum;
  if (rand01(g) >= specProb) {
    woL = sample_cosine(g, pdfOut);
    pdfOut *= (1.0f - specProb);
    return (1.0f - E) * diffuse / kPi;
  }
  vec3 m = beckmann_sample(g, rough);
  woL = -wiL + 2.0f * glsl::dot(wiL, m) * m;
  pdfOut = specProb;
  if (woL.z < kDenomTol) return vec3(0.0f);
  float D = beckmann_D(m, rough);
  float G = smith_g2(wiL, woL, m, rough);
  float Fr = fresnel_dielectric(fabsf(wiL.z), ior);
  vec3 r = Fr * spec * D * G / fmaxf(4.0f * fabsf(woL.z) * fabsf(wiL.z), kDenomTol);
  float dwh = 1.0f / fmaxf(fabsf(4.0f * glsl::dot(wiL, m)), kDenomTol);
  pdfOut *= beckmann_pdf(m, rough) * dwh;
  return r;
}
#endif

// SP:467-490: only the Surface material has a BSDF in this program (none: zero).
SD_FN vec3 ps_bsdf_eval(Scene& sc, const SnellyParams& P, const vec3& X, const Frame& f, const vec3& wiL,
                        const vec3& woL, int mat) {
#ifdef HAS_SURFACE
  if (mat == MAT_SURFA) return ps_surf_eval(sc, P, X, f, wiL, woL);
#endif
  return vec3(0.0f);
}
SD_FN float ps_bsdf_pdf(Scene& sc, const SnellyParams& P, const vec3& X, const Frame& f, const vec3& wiL,
                        const vec3& woL, int mat) {
#ifdef HAS_SURFACE
  if (mat == MAT_SURFA) return ps_surf_pdf(sc, P, X, f, wiL, woL);
#endif
  return 0.0f;
}
SD_FN vec3 ps_bsdf_sample(Scene& sc, const SnellyParams& P, const vec3& X, const Frame& f, const vec3& wiL, int mat,
                          vec3& woL, float& pdf, Rng& g) {
#ifdef HAS_SURFACE
  if (mat == MAT_SURFA) return ps_surf_sample(sc, P, X, f, wiL, woL, pdf, g);
#endif
  return vec3(0.0f);
}

// SP:713-760: next-event estimate of sky and sun at a surface vertex, clamped.
SD_FN vec3 ps_direct(const Ctx& c, const vec3& pW, const Frame& b, const vec3& wiW, int mat, Rng& g, float& skyPdf,
                     float& sunPdf) {
  const SnellyParams& P = c.P;
  const vec3 wiL = to_local(wiW, b);
  vec3 Ld(0.0f);
  if (P.skyPower > kRadianceEps) {
    vec3 Li(0.0f), woL(0.0f), woW(0.0f);
    if (!(P.skyPower < kRadianceEps)) {  // SP:648-657
      woL = sample_cosine(g, skyPdf);
      woW = to_world(woL, b);
      Li = sky_rgb(c, woW);
    }
    if (avg(Li) > kRadianceEps) {
      Li *= ps_tr_segment(c.sc, P, pW, woW, P.maxLengthScale);
      if (avg(Li) > kRadianceEps) {
        float bsdfPdf = fmaxf(kPdfEps, ps_bsdf_pdf(c.sc, P, pW, b, wiL, woL, mat));
        vec3 f = ps_bsdf_eval(c.sc, P, pW, b, wiL, woL, mat);
        float w = balance(skyPdf, bsdfPdf);
        Ld += f * Li / fmaxf(kPdfEps, skyPdf) * fabsf(glsl::dot(woW, b.n)) * w;
      }
    }
  }
  if (P.sunPower > kRadianceEps) {
    vec3 Li(0.0f), woL(0.0f), woW(0.0f);
    if (!(P.sunPower < kRadianceEps)) {  // SP:696-705
      woW = sample_sun_dir(c, g, sunPdf);
      woL = to_local(woW, b);
      if (!(woL.z < 0.0f)) Li = ps_sun_radiance(P, woW);
    }
    if (avg(Li) > kRadianceEps) {
      Li *= ps_tr_segment(c.sc, P, pW, woW, P.maxLengthScale);
      if (avg(Li) > kRadianceEps) {
        float bsdfPdf = fmaxf(kPdfEps, ps_bsdf_pdf(c.sc, P, pW, b, wiL, woL, mat));
        vec3 f = ps_bsdf_eval(c.sc, P, pW, b, wiL, woL, mat);
        float w = balance(sunPdf, bsdfPdf);
        Ld += f * Li / fmaxf(kPdfEps, sunPdf) * fabsf(glsl::dot(woW, b.n)) * w;
      }
    }
  }
  return glsl::min(vec3(P.radianceClamp), Ld);
}

#ifdef HAS_SURFACE
// SP:765-818: random walk inside the surface (at most 256 steps, Russian roulette after 4).
SD_FN bool ps_sss_walk(const Ctx& c, const vec3& pW, const Frame& b, Rng& g, float mfp, const vec3& albedo,
                       vec3& walkThr, vec3& pExit) {
  const SnellyParams& P = c.P;
  vec3 pWalk = pW;
  pWalk -= 3.0f * P.minLengthScale * b.n;
  float pdfDir;
  vec3 dL = sample_cosine(g, pdfDir);
  vec3 dW = -to_world(dL, b);
  walkThr = vec3(1.0f);
  for (int n = 0; n < 256; ++n) {
    if (n > P.maxSSSSteps) break;
    float step = -logf(rand01(g)) * mfp * P.lengthScale;
    vec3 pHit(0.0f);
    int m;
    if (ps_trace(c.sc, P, pWalk, dW, step, pHit, m)) {
      pExit = pHit;
      return true;
    }
    if (n > 4) {
      float cont = glsl::clamp(10.0f * maxc(walkThr), 0.0f, 1.0f);
      if (rand01(g) < 1.0f - cont) break;
      walkThr /= cont;
    }
    dW = sample_hg(dW, P.subsurfaceAnisotropy, g);
    pWalk += step * dW;
    walkThr *= albedo;
  }
  return false;
}

// SP:820-866: sky and sun next-event estimate at the walk's exit, for a Lambertian lobe.
SD_FN vec3 ps_sss_exit(const Ctx& c, const vec3& pW, const Frame& b, Rng& g, const vec3& albedoExit, float& skyPdf,
                       float& sunPdf) {
  const SnellyParams& P = c.P;
  vec3 Ld(0.0f);
  vec3 f = glsl::mix(vec3(1.0f), albedoExit, P.subsurfaceDiffuseWeight) / kPi;
  if (P.skyPower > kRadianceEps) {
    vec3 Li(0.0f), woL(0.0f), woW(0.0f);
    if (!(P.skyPower < kRadianceEps)) {
      woL = sample_cosine(g, skyPdf);
      woW = to_world(woL, b);
      Li = sky_rgb(c, woW);
    }
    Li *= ps_tr_segment(c.sc, P, pW, woW, P.maxLengthScale);
    if (avg(Li) > kRadianceEps) {
      float bsdfPdf = pdf_cosine(woL);
      float w = balance(skyPdf, bsdfPdf);
      Ld += f * Li / fmaxf(kPdfEps, skyPdf) * fabsf(glsl::dot(woW, b.n)) * w;
    }
  }
  if (P.sunPower > kRadianceEps) {
    vec3 Li(0.0f), woL(0.0f), woW(0.0f);
    if (!(P.sunPower < kRadianceEps)) {
      woW = sample_sun_dir(c, g, sunPdf);
      woL = to_local(woW, b);
      if (!(woL.z < 0.0f)) Li = ps_sun_radiance(P, woW);
    }
    Li *= ps_tr_segment(c.sc, P, pW, woW, P.maxLengthScale);
    if (avg(Li) > kRadianceEps) {
      float bsdfPdf = pdf_cosine(woL);
      float w = balance(sunPdf, bsdfPdf);
      Ld += f * Li / fmaxf(kPdfEps, sunPdf) * fabsf(glsl::dot(woW, b.n)) * w;
    }
  }
  return glsl::min(vec3(P.radianceClamp), Ld);
}
#endif

// SP:892-1075: the camera path in RGB.
SD_FN vec3 ps_camera_path(const Ctx& c, vec3 pW, vec3 rayDir, Rng& g) {
  const SnellyParams& P = c.P;
  vec3 L(0.0f);
  float misSky = 1.0f, misSun = 1.0f;
  vec3 thr(1.0f);
  for (int vertex = 0; vertex <= MAX_BOUNCES; ++vertex) {
    if (maxc(thr) < kThroughputEps) break;
    vec3 pNext(0.0f);
    int mat;
    const bool hit = ps_trace(c.sc, P, pW, rayDir, P.maxLengthScale, pNext, mat);
    vec3 Tr;
    if (hit) {
      Tr = ps_tr_free(P, glsl::length(pNext - pW));
    } else {
      Tr = ps_tr_free(P, P.maxLengthScale);
#ifdef HAS_FOG
      if (avg(Tr) > kRadianceEps)
#endif
      {
        if (!(vertex == 0 && !P.envMapVisible) && misSky > 0.0f) L += thr * Tr * misSky * sky_rgb(c, rayDir);
        if (!(vertex == 0 && !P.sunVisibleDirectly) && misSun > 0.0f)
          L += thr * Tr * misSun * ps_sun_radiance(P, rayDir);
      }
#ifdef HAS_FOG
      if (vertex < 2) L += thr * ps_inscatter(P, Tr);
#endif
      break;
    }
#ifdef HAS_FOG
    if (vertex < 2) L += thr * ps_inscatter(P, Tr);
    thr *= Tr;
#endif
    pW = pNext;
    vec3 nW = ps_normal(c.sc, P, pW, mat);
    const vec3 ngW = nW;
    Frame b = make_frame(nW);
#ifdef HAS_NORMALMAP
    nW = ps_perturb(c.sc, pW, b, mat);
    if (glsl::dot(nW, rayDir) > 0.0f && mat != MAT_DIELE) nW = 2.0f * ngW * glsl::dot(ngW, nW) - nW;
    b = make_frame(nW);
#endif
    bool sss = false;
    float probSss = 0.0f;
    vec3 sssAlbedo(0.0f);
#ifdef HAS_SURFACE
    if (P.subsurfaceMFP > 0.0f) {
      sssAlbedo = c.sc.SUBSURFACE_ALBEDO(v3(P.subsurfaceAlbedoRGB), pW, b.n);
      float dw = (1.0f - P.subsurface) * avg(ps_diffuse(c.sc, P, pW, b.n, -rayDir));
      float sw = avg(ps_specular(c.sc, P, pW, b.n, -rayDir));
      float ssw = P.subsurface * avg(sssAlbedo) * 3.0f;
      float total = dw + sw + ssw;
      probSss = ssw / (total + kDenomTol);
      probSss = glsl::clamp(probSss, 0.0f, 1.0f - kPdfEps);
      sss = rand01(g) < probSss;
    }
#endif
    if (!sss) {
      const vec3 wiW = -rayDir;
      const vec3 wiL = to_local(wiW, b);
      vec3 woL(0.0f);
      float bsdfPdf = 0.0f;
      vec3 f = ps_bsdf_sample(c.sc, P, pW, b, wiL, mat, woL, bsdfPdf, g);
      vec3 woW = to_world(woL, b);
#ifdef HAS_VOLUME_EMISSION
      L += thr * c.sc.VOLUME_EMISSION(v3(P.volumeEmissionColorRGB) * P.volumeEmission, pW);
#endif
      rayDir = woW;
      pW += ngW * glsl::sign(glsl::dot(rayDir, ngW)) * 3.0f * P.minLengthScale;
      float skyPdf = 0.0f, sunPdf = 0.0f;
      L += thr * ps_direct(c, pW, b, wiW, mat, g, skyPdf, sunPdf);
      vec3 fOverPdf = glsl::min(vec3(P.radianceClamp), f / fmaxf(kPdfEps, bsdfPdf));
      vec3 st = fOverPdf * fabsf(glsl::dot(woW, nW)) / fmaxf(kPdfEps, 1.0f - probSss);
      thr *= st;
      misSky = balance(bsdfPdf, skyPdf);
      misSun = balance(bsdfPdf, sunPdf);
    }
#ifdef HAS_SURFACE
    else {
      vec3 albedoEntry = ps_diffuse(c.sc, P, pW, b.n, -rayDir);
      vec3 walkThr(0.0f), pExit(0.0f);
      Frame bw = b;
      bw.n = ngW;  // the walk enters with the geometric normal (SP:1029)
      if (!ps_sss_walk(c, pW, bw, g, P.subsurfaceMFP, sssAlbedo, walkThr, pExit)) break;
      pW = pExit;
      nW = ps_normal(c.sc, P, pExit, MAT_SURFA);
      Frame be = make_frame(nW);
      float bsdfPdf;
      vec3 dL = sample_cosine(g, bsdfPdf);
      vec3 woW = to_world(dL, be);
      rayDir = woW;
      thr *= walkThr;
      float skyPdf = 0.0f, sunPdf = 0.0f;
      vec3 albedoExit = ps_diffuse(c.sc, P, pW, nW, -rayDir);
      L += thr * ps_sss_exit(c, pExit, be, g, albedoExit, skyPdf, sunPdf);
      misSky = balance(bsdfPdf, skyPdf);
      misSun = balance(bsdfPdf, sunPdf);
      vec3 f = glsl::mix(vec3(1.0f), albedoExit, P.subsurfaceDiffuseWeight) / kPi;
      vec3 fOverPdf = glsl::min(vec3(P.radianceClamp), f / fmaxf(kPdfEps, bsdfPdf));
      vec3 st = fOverPdf * fabsf(glsl::dot(woW, nW));
      thr *= st / fmaxf(kPdfEps, probSss);
      pW += nW * glsl::sign(glsl::dot(rayDir, nW)) * 3.0f * P.minLengthScale;
    }
#endif
  }
  return L;
}

}  // namespace sdev

// One frame of the simplified path tracer (SP:1083-1130) for every pixel of the job: XYZ of the RGB
// estimate, added to the pixel's Kahan sums.
extern "C" __global__ void __launch_bounds__(SNELLY_BLOCK) snelly_ptsimple(const JobRec* __restrict__ jobs,
                                                                        const int* __restrict__ block_start, int njobs,
                                                                        const SnellyParams* __restrict__ gparams) {
  using namespace sdev;
  int j = job_of_block(block_start, njobs, blockIdx.x);
  const JobRec& J = jobs[j];
  long long i = (long long)(blockIdx.x - block_start[j]) * blockDim.x + threadIdx.x + J.pixel_begin;
  if (i >= (long long)J.pixel_begin + J.pixel_count) return;
  const int slot = J.slot;
  const SnellyParams& P = c_params[slot];
  uint4 r4 = J.rng[i];
  Rng g;
  g.s[0] = r4.x; g.s[1] = r4.y; g.s[2] = r4.z; g.s[3] = r4.w;
  Scene sc(uniforms_of(slot));
  sc.INIT();
  Ctx c{P, gparams + slot, sc, slot, 570.0f, vec3(0.0f), make_frame(v3(P.sunDir))};
  const int W = J.width;
  const vec2 pixel(float(int(i % W)) + 0.5f, float(int(i / W)) + 0.5f);
  vec3 L(0.0f);
  for (int n = 0; n < MAX_SAMPLES_PER_FRAME; ++n) {
    float jx = 0.5f * P.filterRadius * tent(rand01(g));
    float jy = 0.5f * P.filterRadius * tent(rand01(g));
    vec3 start, dir;
    primary_ray_hook(c, pixel + vec2(jx, jy), g, start, dir);
    L += ps_camera_path(c, start, dir, g);
  }
  L /= float(MAX_SAMPLES_PER_FRAME);
  vec3 xyz = rgb_to_xyz(L);
  J.rng[i] = make_uint4(g.s[0], g.s[1], g.s[2], g.s[3]);
  float4 s = J.acc[i], cp = J.comp[i];
  kahan_add(s, cp, xyz);
  J.acc[i] = s;
  J.comp[i] = cp;
}
