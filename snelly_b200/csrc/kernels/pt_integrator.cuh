// pt_integrator.cuh - the per-sample estimator: next-event estimation, homogeneous atmosphere,
// subsurface random walk and the camera path (PT:1221-1989), on top of pt_device.cuh.
//
// Used as is by the path-per-thread kernel, and piecewise by the wavefront stages.
#pragma once
#include "pt_device.cuh"

namespace sdev {

// Next-event estimation at a surface vertex (PT:1221-1295).
SD_FN Rad direct_surface(const Ctx& c, const vec3& pW, const Frame& f, const vec3& wiW, int mat, Rng& g,
                         float& skyPdf, float& sunPdf, float& sphPdf) {
  const SnellyParams& P = c.P;
  vec3 wiL = to_local(wiW, f);
  Rad Ld = Rad(0.0f);
  if (P.skyPower > kRadianceEps) {
    vec3 woL = sample_cosine(g, skyPdf);
    vec3 woW = to_world(woL, f);
    Rad Li = sky_radiance(c, woW);
    if (avg(Li) > kRadianceEps) {
      Li = shadow_scale(c, Li, transmittance(c, pW, woW, P.maxLengthScale));
      if (avg(Li) > kRadianceEps) {
        float bp = fmaxf(kPdfEps, bsdf_pdf(c, pW, f, wiL, woL, mat));
        Rad fv = bsdf_eval(c, pW, f, wiL, woL, mat);
        float w = balance(skyPdf, bp);
        Ld += fv * Li / fmaxf(kPdfEps, skyPdf) * fabsf(glsl::dot(woW, f.n)) * w;
      }
    }
  }
  if (P.sunPower > kRadianceEps) {
    vec3 woW = sample_sun_dir(c, g, sunPdf);
    vec3 woL = to_local(woW, f);
    Rad Li = woL.z < 0.0f ? Rad(0.0f) : sun_radiance(c, woW);
    if (avg(Li) > kRadianceEps) {
      Li = shadow_scale(c, Li, transmittance(c, pW, woW, P.maxLengthScale));
      if (avg(Li) > kRadianceEps) {
        float bp = fmaxf(kPdfEps, bsdf_pdf(c, pW, f, wiL, woL, mat));
        Rad fv = bsdf_eval(c, pW, f, wiL, woL, mat);
        float w = balance(sunPdf, bp);
        Ld += fv * Li / fmaxf(kPdfEps, sunPdf) * fabsf(glsl::dot(woW, f.n)) * w;
      }
    }
  }
#ifdef HAS_SPHERE_LIGHT
  if (P.sphereLightPower > kRadianceEps &&
      glsl::dot(pW - v3(P.sphereLightPosition), f.n) <= P.sphereLightRadius) {
    vec3 pHit;
    Rad Li = sample_sphere_light(c, g, pW, pHit, sphPdf);
    if (avg(Li) > kRadianceEps) {
      float dist = fmaxf(0.0f, glsl::length(pHit - pW) - 3.0f * P.minLengthScale);
      vec3 woW = glsl::normalize(pHit - pW);
      vec3 woL = to_local(woW, f);
      Li = shadow_scale(c, Li, transmittance(c, pW, woW, dist));
      if (avg(Li) > kRadianceEps) {
        float bp = fmaxf(kPdfEps, bsdf_pdf(c, pW, f, wiL, woL, mat));
        Rad fv = bsdf_eval(c, pW, f, wiL, woL, mat);
        float w = balance(sphPdf, bp);
        Ld += fv * Li / fmaxf(kPdfEps, sphPdf) * fabsf(glsl::dot(woW, f.n)) * w;
      }
    }
  }
#endif
  return glsl::min(Rad(P.radianceClamp), Ld);
}

#ifdef HAS_ATMOSPHERE
// Light scattered towards -rayDir at a point of the atmosphere (PT:1299-1363).
SD_FN Rad direct_volume(const Ctx& c, const vec3& pW, const vec3& rayDir, Rng& g) {
  const SnellyParams& P = c.P;
  Rad Ld = Rad(0.0f);
  if (P.skyPower > kRadianceEps) {
    vec3 woW = sample_sphere_ref(g);
    float pdf = 1.0f / (4.0f * kPi);
    Rad Li = sky_radiance(c, woW);
    if (avg(Li) > kRadianceEps) {
      Li = shadow_scale(c, Li, transmittance(c, pW, woW, P.maxLengthScale));
      if (avg(Li) > kRadianceEps) {
        float ph = hg_phase(glsl::dot(-rayDir, -woW), P.atmosphereAnisotropy);
        Ld += ph * Li / fmaxf(kPdfEps, pdf);
      }
    }
  }
  if (P.sunPower > kRadianceEps) {
    float pdf;
    vec3 woW = sample_sun_dir(c, g, pdf);
    Rad Li = sun_radiance(c, woW);
    if (avg(Li) > kRadianceEps) {
      Li = shadow_scale(c, Li, transmittance(c, pW, woW, P.maxLengthScale));
      if (avg(Li) > kRadianceEps) {
        float ph = hg_phase(glsl::dot(-rayDir, -woW), P.atmosphereAnisotropy);
        Ld += ph * Li / fmaxf(kPdfEps, pdf);
      }
    }
  }
#ifdef HAS_SPHERE_LIGHT
  if (P.sphereLightPower > kRadianceEps) {
    float pdf;
    vec3 pHit;
    Rad Li = sample_sphere_light(c, g, pW, pHit, pdf);
    if (avg(Li) > kRadianceEps) {
      float dist = fmaxf(0.0f, glsl::length(pHit - pW) - 3.0f * P.minLengthScale);
      vec3 woW = glsl::normalize(pHit - pW);
      Li = shadow_scale(c, Li, transmittance(c, pW, woW, dist));
      if (avg(Li) > kRadianceEps) {
        float ph = hg_phase(glsl::dot(-rayDir, -woW), P.atmosphereAnisotropy);
        Ld += ph * Li / fmaxf(kPdfEps, pdf);
      }
    }
  }
#endif
  return glsl::min(Rad(P.radianceClamp), Ld);
}

// Single-scattering estimate over a segment (PT:1365-1417).
SD_FN Rad atm_inscatter(const Ctx& c, const vec3& pW, const vec3& d, float len, Rng& g) {
  const SnellyParams& P = c.P;
  Rad Ls = Rad(0.0f);
#ifdef HAS_FOG
  if (P.fogEnable) {
    Rad TrFog = transmittance_free(c, pW, d, len);
    Ls = (Rad(1.0f) - TrFog) * albedo(v3(P.fogEmission), c.cmf);
  }
#endif
  Rad ext = vol_extinction(c), sca = vol_scattering(c);
  float en = avg(ext), sn = avg(sca);
  if (en < kRadianceEps || sn < kRadianceEps) return Ls;
  float t0, t1;
  if (!atmosphere_segment(c, pW, d, len, t0, t1)) return Ls;
  float T01 = expf(-(t1 - t0) * en);
  float ts = t0 - logf(1.0f - rand01(g) * (1.0f - T01)) / en;
  vec3 ps = pW + ts * d;
  Rad od = (ts - t0) * ext;
  Rad Trp = glsl::exp(-od);
  float inv = (1.0f - T01) * expf(avg(od)) / en;
  Rad Li = direct_volume(c, ps, d, g);
  Ls += Trp * sca * Li * inv;
#ifdef HAS_VOLUME_EMISSION
  vec3 wo = sample_hg(d, P.atmosphereAnisotropy, g);
  Hit h = march_ray(c.job, ps, wo, P.maxLengthScale);
  if (h.hit) Ls += Trp * sca * vol_emission(c, h.p) * inv;
#endif
  return Ls;
}

// Scatter-point and direction sample for a continuing path (PT:1419-1442).
SD_FN Rad atm_scatter_sample(const Ctx& c, const vec3& pW, const vec3& d, float len, Rng& g, vec3& ps, vec3& wo) {
  Rad ext = vol_extinction(c), sca = vol_scattering(c);
  float en = avg(ext);
  float t0, t1;
  if (!atmosphere_segment(c, pW, d, len, t0, t1)) return Rad(0.0f);
  float T01 = expf(-(t1 - t0) * en);
  float ts = t0 - logf(1.0f - rand01(g) * (1.0f - T01)) / en;
  ps = pW + ts * d;
  Rad od = (ts - t0) * ext;
  Rad Trp = glsl::exp(-od);
  float inv = (1.0f - T01) * expf(avg(od)) / en;
  wo = sample_hg(d, c.P.atmosphereAnisotropy, g);
  return sca * Trp * inv;
}
#endif  // HAS_ATMOSPHERE

// PT:1446-1457
SD_FN float scatter_prob(const Ctx& c, const Rad& Tr) {
#ifdef HAS_ATMOSPHERE
  Rad ext = vol_extinction(c), sca = vol_scattering(c);
  return avg(sca / ext) * (1.0f - avg(Tr));
#else
  (void)c;
  (void)Tr;
  return 0.0f;
#endif
}

#ifdef HAS_SURFACE
// Subsurface random walk inside SDF_SURFACE (PT:1464-1518), as a start and single steps so that a
// persistent walker can interleave many walks: the walk's position, direction, throughput and
// step count.
struct WalkState {
  vec3 pw, dw;
  Rad thr;
  int n;
};
SD_FN void sss_walk_begin(const Ctx& c, const vec3& pW, const Frame& f, Rng& g, WalkState& w) {
  w.pw = pW - 3.0f * c.P.minLengthScale * f.n;
  float pdf;
  vec3 dl = sample_cosine(g, pdf);
  w.dw = -to_world(dl, f);
  w.thr = Rad(1.0f);
  w.n = 0;
}
enum { WALK_ON = 0, WALK_EXIT = 1, WALK_END = 2 };
// One step of the walk: WALK_EXIT with the exit point, WALK_END when the walk stops inside
// (roulette or the step limit), else WALK_ON.
SD_FN int sss_walk_step(const Ctx& c, Rng& g, const Rad& ssAlb, WalkState& w, vec3& pExit) {
  const SnellyParams& P = c.P;
  if (w.n >= 2048 || w.n > P.maxSSSSteps) return WALK_END;
  float step = -logf(rand01(g)) * P.subsurfaceMFP * P.lengthScale;
  Hit h = march_ray(c.job, w.pw, w.dw, step);
  if (h.hit) {
    pExit = h.p;
    return WALK_EXIT;
  }
  if (w.n > 4) {
    float cont = glsl::clamp(10.0f * maxc(w.thr), 0.0f, 1.0f);
    if (rand01(g) < 1.0f - cont) return WALK_END;
    w.thr /= cont;
  }
  w.dw = sample_hg(w.dw, P.subsurfaceAnisotropy, g);
  w.pw += step * w.dw;
  w.thr *= ssAlb;
  ++w.n;
  return WALK_ON;
}
// The whole walk: true at an exit point.
SD_FN bool sss_walk(const Ctx& c, const vec3& pW, const Frame& f, Rng& g, const Rad& ssAlb, Rad& walkThr, vec3& pExit) {
  WalkState w;
  sss_walk_begin(c, pW, f, g, w);
  int r;
  while ((r = sss_walk_step(c, g, ssAlb, w, pExit)) == WALK_ON) {
  }
  walkThr = w.thr;
  return r == WALK_EXIT;
}

// Direct light at a subsurface exit point through a Lambertian lobe (PT:1521-1593).
SD_FN Rad sss_exit_radiance(const Ctx& c, const vec3& pW, const Frame& f, Rng& g, const Rad& dAlbExit,
                            float& skyPdf, float& sunPdf, float& sphPdf) {
  const SnellyParams& P = c.P;
  vec3 off = 3.0f * P.minLengthScale * f.n;
  Rad Ld = Rad(0.0f);
  Rad lobe = glsl::mix(Rad(1.0f), dAlbExit, P.subsurfaceDiffuseWeight) / kPi;
  if (P.skyPower > kRadianceEps) {
    vec3 woL = sample_cosine(g, skyPdf);
    vec3 woW = to_world(woL, f);
    Rad Li = sky_radiance(c, woW);
    if (avg(Li) > kRadianceEps) {
      Li = shadow_scale(c, Li, transmittance(c, pW + off, woW, P.maxLengthScale));
      if (avg(Li) > kRadianceEps) {
        float w = balance(skyPdf, pdf_cosine(woL));
        Ld += lobe * Li / fmaxf(kPdfEps, skyPdf) * fabsf(glsl::dot(woW, f.n)) * w;
      }
    }
  }
  if (P.sunPower > kRadianceEps) {
    vec3 woW = sample_sun_dir(c, g, sunPdf);
    vec3 woL = to_local(woW, f);
    Rad Li = woL.z < 0.0f ? Rad(0.0f) : sun_radiance(c, woW);
    if (avg(Li) > kRadianceEps) {
      Li = shadow_scale(c, Li, transmittance(c, pW + off, woW, P.maxLengthScale));
      if (avg(Li) > kRadianceEps) {
        float w = balance(sunPdf, pdf_cosine(woL));
        Ld += lobe * Li / fmaxf(kPdfEps, sunPdf) * fabsf(glsl::dot(woW, f.n)) * w;
      }
    }
  }
#ifdef HAS_SPHERE_LIGHT
  if (P.sphereLightPower > kRadianceEps &&
      glsl::dot(pW - v3(P.sphereLightPosition), f.n) <= P.sphereLightRadius) {
    vec3 pHit;
    Rad Li = sample_sphere_light(c, g, pW, pHit, sphPdf);
    if (avg(Li) > kRadianceEps) {
      float dist = fmaxf(0.0f, glsl::length(pHit - pW) - 3.0f * P.minLengthScale);
      vec3 woW = glsl::normalize(pHit - pW);
      vec3 woL = to_local(woW, f);
      Li = shadow_scale(c, Li, transmittance(c, pW + off, woW, dist));
      if (avg(Li) > kRadianceEps) {
        float w = balance(sphPdf, pdf_cosine(woL));
        Ld += lobe * Li / fmaxf(kPdfEps, sphPdf) * fabsf(glsl::dot(woW, f.n)) * w;
      }
    }
  }
#endif
  return glsl::min(Rad(P.radianceClamp), Ld);
}
#endif  // HAS_SURFACE

// Primary ray through the (jittered) pixel, pinhole or thin lens (PT:1602-1622).
SD_FN void primary_ray(const SnellyParams& P, const vec2& pixel, Rng& g, vec3& start, vec3& dir) {
  vec2 ndc = -1.0f + 2.0f * (pixel / vec2(P.resolution[0], P.resolution[1]));
  float fh = tanf(0.5f * glsl::radians(P.camFovy));
  float fw = P.camAspect * fh;
  vec3 s = -fw * ndc.x * v3(P.camX) + fh * ndc.y * v3(P.camY);
  dir = safe_normalize(v3(P.camDir) + s);
  if (P.camAperture <= 0.0f) {
    start = v3(P.camPos);
    return;
  }
  vec3 focal = v3(P.camPos) + P.camFocalDistance * dir / glsl::dot(dir, v3(P.camDir));
  float rad = P.camAperture * sqrtf(rand01(g));
  float th = 2.0f * kPi * rand01(g);
  vec3 lens = v3(P.camPos) + rad * (-v3(P.camX) * cosf(th) + v3(P.camY) * sinf(th));
  start = lens;
  dir = safe_normalize(focal - lens);
}

// Triangle-filter importance sample in [-1, 1] (PT:1928-1932).
SD_FN float tent(float xi) { return xi < 0.5f ? sqrtf(2.0f * xi) - 1.0f : 1.0f - sqrtf(2.0f - 2.0f * xi); }

// ---- the camera path, one vertex at a time (PT:1625-1926) -----------------------------------------
// Everything a path carries from one vertex to the next.
struct PathState {
  vec3 pW, rayDir;
  Rad thr, L;
  float misSky, misSun, misSph;
  int atmScatters;
  bool inDiele;
};

// Next-event estimation whose sky and sun shadow rays are traced later (wavefront stages): the
// unoccluded contribution of each light, to be scaled by the shadow term once the ray is traced.
struct DeferredNee {
  vec3 org;            // shadow-ray origin (the offset vertex)
  Rad thr;             // path throughput at the vertex
  Rad extra;           // sphere-light term, already shadowed
  vec3 dir[2];         // sky, sun
  float dist[2];
  Rad c[2];            // f * Li0 / pdf * |cos| * mis
  Rad li[2];           // Li0 (unshadowed radiance, for the gate)
  bool pending[2];
  bool any;
};

SD_FN void start_path(const Ctx& c, PathState& s, const vec3& start, const vec3& dir) {
  s.pW = start;
  s.rayDir = dir;
  s.thr = Rad(1.0f);
  s.L = Rad(0.0f);
  s.misSky = s.misSun = s.misSph = 1.0f;
  s.atmScatters = 0;
#ifdef HAS_DIELECTRIC
  s.inDiele = c.sc.SDF_DIELECTRIC(start) < 0.0f;
#else
  (void)c;
  s.inDiele = false;
#endif
}

// Next-event estimation at a surface vertex with the sky and sun shadow rays deferred
// (same random numbers in the same order as direct_surface).
SD_FN void direct_surface_deferred(const Ctx& c, const vec3& pW, const Frame& f, const vec3& wiW, int mat, Rng& g,
                                   float& skyPdf, float& sunPdf, float& sphPdf, const Rad& thr, DeferredNee& nd) {
  const SnellyParams& P = c.P;
  vec3 wiL = to_local(wiW, f);
  nd.org = pW;
  nd.thr = thr;
  nd.extra = Rad(0.0f);
  nd.pending[0] = nd.pending[1] = false;
  if (P.skyPower > kRadianceEps) {
    vec3 woL = sample_cosine(g, skyPdf);
    vec3 woW = to_world(woL, f);
    Rad Li = sky_radiance(c, woW);
    if (avg(Li) > kRadianceEps) {
      float bp = fmaxf(kPdfEps, bsdf_pdf(c, pW, f, wiL, woL, mat));
      Rad fv = bsdf_eval(c, pW, f, wiL, woL, mat);
      float w = balance(skyPdf, bp);
      nd.c[0] = fv * Li / fmaxf(kPdfEps, skyPdf) * fabsf(glsl::dot(woW, f.n)) * w;
      nd.li[0] = Li;
      nd.dir[0] = woW;
      nd.dist[0] = P.maxLengthScale;
      nd.pending[0] = true;
    }
  }
  if (P.sunPower > kRadianceEps) {
    vec3 woW = sample_sun_dir(c, g, sunPdf);
    vec3 woL = to_local(woW, f);
    Rad Li = woL.z < 0.0f ? Rad(0.0f) : sun_radiance(c, woW);
    if (avg(Li) > kRadianceEps) {
      float bp = fmaxf(kPdfEps, bsdf_pdf(c, pW, f, wiL, woL, mat));
      Rad fv = bsdf_eval(c, pW, f, wiL, woL, mat);
      float w = balance(sunPdf, bp);
      nd.c[1] = fv * Li / fmaxf(kPdfEps, sunPdf) * fabsf(glsl::dot(woW, f.n)) * w;
      nd.li[1] = Li;
      nd.dir[1] = woW;
      nd.dist[1] = P.maxLengthScale;
      nd.pending[1] = true;
    }
  }
#ifdef HAS_SPHERE_LIGHT
  if (P.sphereLightPower > kRadianceEps &&
      glsl::dot(pW - v3(P.sphereLightPosition), f.n) <= P.sphereLightRadius) {
    vec3 pHit;
    Rad Li = sample_sphere_light(c, g, pW, pHit, sphPdf);
    if (avg(Li) > kRadianceEps) {
      float dist = fmaxf(0.0f, glsl::length(pHit - pW) - 3.0f * P.minLengthScale);
      vec3 woW = glsl::normalize(pHit - pW);
      vec3 woL = to_local(woW, f);
      Li = shadow_scale(c, Li, transmittance(c, pW, woW, dist));
      if (avg(Li) > kRadianceEps) {
        float bp = fmaxf(kPdfEps, bsdf_pdf(c, pW, f, wiL, woL, mat));
        Rad fv = bsdf_eval(c, pW, f, wiL, woL, mat);
        float w = balance(sphPdf, bp);
        nd.extra = fv * Li / fmaxf(kPdfEps, sphPdf) * fabsf(glsl::dot(woW, f.n)) * w;
      }
    }
  }
#else
  (void)sphPdf;
#endif
  nd.any = true;
}

// The deferred estimate once the shadow rays are traced: occluded[l] for each pending light.
SD_FN Rad resolve_deferred(const Ctx& c, const DeferredNee& nd, const bool occluded[2]) {
  Rad Ld = Rad(0.0f);
  for (int l = 0; l < 2; ++l) {
    if (!nd.pending[l]) continue;
    Rad Tr = occluded[l] ? Rad(0.0f) : transmittance_free(c, nd.org, nd.dir[l], nd.dist[l]);
    Rad sc = glsl::abs(Rad(1.0f) - c.P.shadowStrength * (Rad(1.0f) - Tr));
    if (avg(nd.li[l] * sc) > kRadianceEps) Ld += nd.c[l] * sc;
  }
  Ld += nd.extra;
  return nd.thr * glsl::min(Rad(c.P.radianceClamp), Ld);
}

enum { VERTEX_CONTINUE = 0, VERTEX_DONE = 1, VERTEX_SSS = 2, VERTEX_VOLUME = 3 };

// A surface vertex that chose the subsurface walk: what the rest of the vertex needs.
struct SssEntry {
  Frame fr;     // shading frame at the entry point
  vec3 ngW;     // geometric normal there
  Rad ssAlb;    // subsurface albedo
  float probSSS;
};

#ifdef HAS_SURFACE
// The rest of a vertex that chose the subsurface walk (PT:1866-1918): the walk to an exit point,
// the exit's direct light and the Lambertian continuation direction.
// The vertex after a walk that reached an exit point (PT:1884-1918).
SD_FN int sss_exit(const Ctx& c, PathState& s, float probSSS, const Rad& walkThr, const vec3& pExit, Rng& g) {
  const SnellyParams& P = c.P;
  s.pW = pExit;
  vec3 nW = sdf_normal(c.job, pExit, MAT_SURFA);
  Frame fe = make_frame(nW);
  float bsdfPdf = 0.0f;
  vec3 dExit = sample_cosine(g, bsdfPdf);
  vec3 woW = to_world(dExit, fe);
  s.rayDir = woW;
  s.thr *= walkThr;
  float skyPdf = 0.0f, sunPdf = 0.0f, sphPdf = 0.0f;
  Rad dAlbExit = surf_diffuse(c, s.pW, nW, -s.rayDir);
  if (!s.inDiele) s.L += s.thr * sss_exit_radiance(c, pExit, fe, g, dAlbExit, skyPdf, sunPdf, sphPdf);
  s.misSky = balance(bsdfPdf, skyPdf);
  s.misSun = balance(bsdfPdf, sunPdf);
#ifdef HAS_SPHERE_LIGHT
  s.misSph = balance(bsdfPdf, sphPdf);
#endif
  Rad lobe = glsl::mix(Rad(1.0f), dAlbExit, P.subsurfaceDiffuseWeight) / kPi;
  Rad fop = glsl::min(Rad(P.radianceClamp), lobe / fmaxf(kPdfEps, bsdfPdf));
  s.thr *= fop * fabsf(glsl::dot(woW, nW)) / fmaxf(kPdfEps, probSSS);
  s.pW += nW * glsl::sign(glsl::dot(s.rayDir, nW)) * 3.0f * P.minLengthScale;
  if (maxc(s.thr) < kThroughputEps) return VERTEX_DONE;
  return VERTEX_CONTINUE;
}

// The entry's frame for the walk: the geometric normal, with the shading frame's tangents.
SD_FN Frame sss_walk_frame(const SssEntry& e) {
  Frame fw = e.fr;
  fw.n = e.ngW;
  return fw;
}

// The rest of a vertex that chose the subsurface walk (PT:1866-1918): the walk, then the exit.
SD_FN int sss_step(const Ctx& c, PathState& s, const SssEntry& e, Rng& g) {
  Rad walkThr = Rad(0.0f);
  vec3 pExit(0.0f);
  if (!sss_walk(c, s.pW, sss_walk_frame(e), g, e.ssAlb, walkThr, pExit)) return VERTEX_DONE;
  return sss_exit(c, s, e.probSSS, walkThr, pExit, g);
}
#endif

#ifdef HAS_HETERO_VOLUME
// A scattering event of the heterogeneous medium at ps (an extension of this build, see
// pt_device.cuh): the single-scattering albedo, next-event estimation of sky (uniform sphere), sun
// and sphere light through the phase function with the balance heuristic against the phase
// function's pdf, and a continuation direction drawn from the phase function (whose weight is one).
SD_FN int hv_scatter(const Ctx& c, PathState& s, const vec3& ps, Rng& g) {
  const SnellyParams& P = c.P;
  const vec3 sca = c.sc.VOLUME_SCATTERING_COLOR(v3(P.atmosphereScatteringCoeffRGB), ps);
  const vec3 ab = c.sc.VOLUME_ABSORPTION_COLOR(v3(P.atmosphereExtinctionCoeffRGB) - v3(P.atmosphereScatteringCoeffRGB), ps);
  const vec3 ext = sca + ab;
  const vec3 a(ext.x > 0.0f ? sca.x / ext.x : 0.0f, ext.y > 0.0f ? sca.y / ext.y : 0.0f, ext.z > 0.0f ? sca.z / ext.z : 0.0f);
  s.thr *= albedo(a, c.cmf);
  const float gph = c.sc.VOLUME_ANISOTROPY(P.atmosphereAnisotropy, ps);
  const vec3 d = s.rayDir;
  Rad Ld = Rad(0.0f);
  const float skyPdf = 1.0f / (4.0f * kPi);
  float sunPdf = 0.0f, sphPdf = 0.0f;
  if (P.skyPower > kRadianceEps) {
    const vec3 wo = hv_sample_sphere(g);
    Rad Li = sky_radiance(c, wo);
    if (avg(Li) > kRadianceEps) {
      Li = shadow_scale(c, Li, transmittance(c, ps, wo, P.maxLengthScale));
      if (avg(Li) > kRadianceEps) {
        const float ph = hg_phase(glsl::dot(d, wo), gph);
        Ld += ph * Li / skyPdf * balance(skyPdf, ph);
      }
    }
  }
  if (P.sunPower > kRadianceEps) {
    const vec3 wo = sample_sun_dir(c, g, sunPdf);
    Rad Li = sun_radiance(c, wo);
    if (avg(Li) > kRadianceEps) {
      Li = shadow_scale(c, Li, transmittance(c, ps, wo, P.maxLengthScale));
      if (avg(Li) > kRadianceEps) {
        const float ph = hg_phase(glsl::dot(d, wo), gph);
        Ld += ph * Li / fmaxf(kPdfEps, sunPdf) * balance(sunPdf, ph);
      }
    }
  }
#ifdef HAS_SPHERE_LIGHT
  if (P.sphereLightPower > kRadianceEps) {
    vec3 pHit;
    Rad Li = sample_sphere_light(c, g, ps, pHit, sphPdf);
    if (avg(Li) > kRadianceEps) {
      const float dist = fmaxf(0.0f, glsl::length(pHit - ps) - 3.0f * P.minLengthScale);
      const vec3 wo = glsl::normalize(pHit - ps);
      Li = shadow_scale(c, Li, transmittance(c, ps, wo, dist));
      if (avg(Li) > kRadianceEps) {
        const float ph = hg_phase(glsl::dot(d, wo), gph);
        Ld += ph * Li / fmaxf(kPdfEps, sphPdf) * balance(sphPdf, ph);
      }
    }
  }
#endif
  s.L += s.thr * glsl::min(Rad(P.radianceClamp), Ld);
  const vec3 wo = hv_sample_hg(d, gph, g);
  const float php = hg_phase(glsl::dot(d, wo), gph);
  s.misSky = P.skyPower > kRadianceEps ? balance(php, skyPdf) : 1.0f;
  s.misSun = balance(php, sunPdf);
  s.misSph = balance(php, sphPdf);
  s.pW = ps;
  s.rayDir = wo;
  return maxc(s.thr) < kThroughputEps ? VERTEX_DONE : VERTEX_CONTINUE;
}
#endif

// Everything of one loop iteration of the camera path after the ray has been traced (`h`).
// With `nd` non-null the surface vertex's sky/sun next-event estimate is deferred into it; with
// `sss` non-null a vertex that chooses the subsurface walk stops before it, fills `sss` and
// returns VERTEX_SSS (the walk stage finishes it with sss_step); with `vol_ps` non-null a vertex
// that collides in the heterogeneous medium stops there, stores the collision point in `vol_ps`
// and returns VERTEX_VOLUME (the volume stage finishes it with hv_scatter).
SD_FN int vertex_step(const Ctx& c, PathState& s, const Hit& h, int vertex, Rng& g, DeferredNee* nd,
                      SssEntry* sss = nullptr, vec3* vol_ps = nullptr) {
  const SnellyParams& P = c.P;
  (void)vertex;
  (void)vol_ps;
#ifdef HAS_HETERO_VOLUME
  {  // the medium before the hit (or the escape): a collision makes this a scattering vertex
    vec3 ps(0.0f);
    const float seg = h.hit ? glsl::length(h.p - s.pW) : P.maxLengthScale;
    if (hv_collision(c, s.pW, s.rayDir, seg, g, ps)) {
      if (vol_ps) {
        *vol_ps = ps;
        return VERTEX_VOLUME;
      }
      return hv_scatter(c, s, ps, g);
    }
  }
#endif
  float rayLength = P.maxLengthScale;
  if (h.hit) {
    rayLength = glsl::length(h.p - s.pW);
  } else {
    // escaped: environment, sun and sphere light (PT:1657-1712)
    float segLen;
    Rad Tr;
#ifdef HAS_SPHERE_LIGHT
    vec3 pLight;
    Rad LiSph = (P.sphereLightPower < kRadianceEps) ? Rad(0.0f) : sphere_light_hit(c, s.pW, s.rayDir, pLight);
    if (avg(LiSph) > kRadianceEps) {
      segLen = glsl::length(pLight - s.pW);
      Tr = transmittance_free(c, s.pW, s.rayDir, segLen, false);
      float sp = scatter_prob(c, Tr);
      s.L += s.thr * Tr * s.misSph * LiSph / (1.0f - sp);
    } else
#endif
    {
      segLen = P.maxLengthScale;
      Tr = transmittance_free(c, s.pW, s.rayDir, segLen, false);
      float sp = scatter_prob(c, Tr);
      if (avg(Tr) > kRadianceEps) {
        if (!(vertex == 0 && !P.envMapVisible) && s.misSky > 0.0f)
          s.L += s.thr * Tr * s.misSky * sky_radiance(c, s.rayDir) / (1.0f - sp);
        if (!(vertex == 0 && !P.sunVisibleDirectly) && s.misSun > 0.0f)
          s.L += s.thr * Tr * s.misSun * sun_radiance(c, s.rayDir) / (1.0f - sp);
      }
    }
#ifdef HAS_ATMOSPHERE
    if (vertex < 2) s.L += s.thr * atm_inscatter(c, s.pW, s.rayDir, segLen, g);
    if (s.atmScatters + 1 < MAX_ATMOSPHERE_SCATTERS) {
      float sp = scatter_prob(c, Tr);
      if (sp > rand01(g)) {
        vec3 ps(0.0f), wo(0.0f);
        s.thr *= atm_scatter_sample(c, s.pW, s.rayDir, segLen, g, ps, wo) / fmaxf(kDenomTol, sp);
        s.pW = ps;
        s.rayDir = wo;
        s.atmScatters++;
        return VERTEX_CONTINUE;
      }
    }
#endif
    (void)segLen;
    return VERTEX_DONE;
  }

  Rad Tr = Rad(1.0f);
  bool hitSphereLight = false;
  (void)hitSphereLight;
  (void)Tr;
#ifdef HAS_SPHERE_LIGHT
  {
    vec3 pLight;
    Rad LiSph = (P.sphereLightPower < kRadianceEps) ? Rad(0.0f) : sphere_light_hit(c, s.pW, s.rayDir, pLight);
    if (avg(LiSph) > kRadianceEps) {
      float segLen = glsl::length(pLight - s.pW);
      if (segLen < rayLength) {
        hitSphereLight = true;
        Tr = transmittance_free(c, s.pW, s.rayDir, segLen, false);
        s.L += s.thr * Tr * s.misSph * LiSph;
#ifdef HAS_ATMOSPHERE
        if (vertex < 2) s.L += s.thr * atm_inscatter(c, s.pW, s.rayDir, segLen, g);
#endif
      }
    }
  }
#endif
#ifdef HAS_DIELECTRIC
  if (s.inDiele) s.thr *= glsl::exp(-rayLength * diele_absorption(c, s.pW));  // Beer's law (PT:1740-1744)
#endif
#ifdef HAS_ATMOSPHERE
  if (vertex < 2) s.L += s.thr * atm_inscatter(c, s.pW, s.rayDir, rayLength, g);
  if (!hitSphereLight) Tr = transmittance_free(c, s.pW, s.rayDir, rayLength, false);
  if (s.atmScatters + 1 < MAX_ATMOSPHERE_SCATTERS) {
    float sp = scatter_prob(c, Tr);
    if (sp > rand01(g)) {
      vec3 ps(0.0f), wo(0.0f);
      s.thr *= atm_scatter_sample(c, s.pW, s.rayDir, rayLength, g, ps, wo) / fmaxf(kDenomTol, sp);
      s.pW = ps;
      s.rayDir = wo;
      s.atmScatters++;
      return VERTEX_CONTINUE;
    }
    s.thr /= fmaxf(kDenomTol, 1.0f - sp);
  }
  if (hitSphereLight) return VERTEX_DONE;
  s.thr *= transmittance_free(c, s.pW, s.rayDir, rayLength, false);
#endif

  // surface interaction (PT:1782-1794)
  s.pW = h.p;
  vec3 nW = sdf_normal(c.job, s.pW, h.mat);
  vec3 ngW = nW;
  Frame fr = make_frame(nW);
#ifdef HAS_NORMALMAP
  nW = perturb_normal(c, s.pW, fr, h.mat);
  if (glsl::dot(nW, s.rayDir) > 0.0f && h.mat != MAT_DIELE) nW = 2.0f * ngW * glsl::dot(ngW, nW) - nW;
  fr = make_frame(nW);
#endif

  // surface scatter or subsurface walk (PT:1796-1811)
  bool doSSS = false;
  float probSSS = 0.0f;
  Rad ssAlb = Rad(0.0f);
  (void)ssAlb;
#ifdef HAS_SURFACE
  if (P.subsurfaceMFP > 0.0f) {
    ssAlb = subsurf_albedo(c, s.pW, fr.n);
    float wd = (1.0f - P.subsurface) * avg(surf_diffuse(c, s.pW, fr.n, -s.rayDir));
    float ws = avg(surf_specular(c, s.pW, fr.n, -s.rayDir));
    float wss = P.subsurface * avg(ssAlb) * 3.0f;
    float tot = wd + ws + wss;
    probSSS = wss / (tot + kDenomTol);
    probSSS = glsl::clamp(probSSS, 0.0f, 1.0f - kPdfEps);
    doSSS = rand01(g) < probSSS;
  }
#endif
  if (!doSSS) {
    vec3 wiW = -s.rayDir;
    vec3 wiL = to_local(wiW, fr);
    vec3 woL(0.0f);  // an uninitialised local in the reference (PT:1820), zero under WebGL
    float bsdfPdf = 0.0f;
    Rad f = bsdf_sample(c, s.pW, fr, wiL, h.mat, woL, bsdfPdf, g);
    vec3 woW = to_world(woL, fr);
#ifdef HAS_DIELECTRIC
    if (h.mat == MAT_DIELE && glsl::dot(wiW, ngW) * glsl::dot(woW, ngW) < 0.0f) s.inDiele = !s.inDiele;
#endif
#ifdef HAS_VOLUME_EMISSION
    s.L += s.thr * vol_emission(c, s.pW);
#endif
    s.rayDir = woW;
    s.pW += ngW * glsl::sign(glsl::dot(s.rayDir, ngW)) * 3.0f * P.minLengthScale;
    float skyPdf = 0.0f, sunPdf = 0.0f, sphPdf = 0.0f;
    if (!s.inDiele) {
      if (nd) direct_surface_deferred(c, s.pW, fr, wiW, h.mat, g, skyPdf, sunPdf, sphPdf, s.thr, *nd);
      else s.L += s.thr * direct_surface(c, s.pW, fr, wiW, h.mat, g, skyPdf, sunPdf, sphPdf);
    }
    Rad fop = glsl::min(Rad(P.radianceClamp), f / fmaxf(kPdfEps, bsdfPdf));
    s.thr *= fop * fabsf(glsl::dot(woW, nW)) / fmaxf(kPdfEps, 1.0f - probSSS);
    s.misSky = balance(bsdfPdf, skyPdf);
    s.misSun = balance(bsdfPdf, sunPdf);
#ifdef HAS_SPHERE_LIGHT
    s.misSph = balance(bsdfPdf, sphPdf);
#endif
  }
#ifdef HAS_SURFACE
  else {  // subsurface random walk to a new vertex (PT:1866-1918)
    SssEntry e{fr, ngW, ssAlb, probSSS};
    if (sss) {
      *sss = e;
      return VERTEX_SSS;
    }
    return sss_step(c, s, e, g);
  }
#else
  (void)sss;
#endif
  if (maxc(s.thr) < kThroughputEps) return VERTEX_DONE;
  return VERTEX_CONTINUE;
}

// The loop bound on vertices: the module's MAX_BOUNCES, or a smaller per-job value.
SD_FN int max_bounces(const SnellyParams& P) {
  return (P.maxBounces > 0 && P.maxBounces < MAX_BOUNCES) ? P.maxBounces : MAX_BOUNCES;
}

// One camera path, path-per-thread (PT:1625-1926).
SD_FN Rad camera_path(const Ctx& c, vec3 pW, vec3 rayDir, Rng& g) {
  PathState s;
  start_path(c, s, pW, rayDir);
  const int maxb = max_bounces(c.P);
  for (int vertex = 0; vertex <= maxb; ++vertex) {
    if (maxc(s.thr) < kThroughputEps) break;
    Hit h = march_ray(c.job, s.pW, s.rayDir, c.P.maxLengthScale);
    if (vertex_step(c, s, h, vertex, g, nullptr) == VERTEX_DONE) break;
  }
  return s.L;
}

// The wavelength at parameter w in [0, 1] of 390..750 nm: sets c.lambda and the normalised rgb
// colour-matching weights c.cmf, returns the CIE XYZ weights (PT:1940-1947). The wavefront
// stores w per path and rebuilds these from it in each stage.
SD_FN vec3 wavelength_at(Ctx& c, float w) {
#ifdef DISPERSION_ENABLED
  c.lambda = 390.0f + (750.0f - 390.0f) * w;
  vec3 xyz = table_xyz(c.Pg->xyzTable, w);
  c.cmf = xyz_to_rgb_normalized(xyz);
  return xyz;
#else
  (void)w;
  c.lambda = 390.0f + (750.0f - 390.0f) * 0.5f;
  c.cmf = vec3(0.0f);
  return vec3(0.0f);
#endif
}

// Wavelength for this pixel and frame (PT:1936-1947): the inverse CDF of the emission spectrum
// at a stratum centre in [0.1, 0.9]; returns the CIE XYZ weights at that wavelength, and its
// parameter w in `w_out`.
SD_FN vec3 pick_wavelength(Ctx& c, Rng& g, float* w_out = nullptr) {
#ifdef DISPERSION_ENABLED
  const SnellyParams& P = c.P;
  float ns = float(P.wavelengthSamples);
  float xi = 0.1f + 0.8f * (0.5f + glsl::s_floor(ns * rand01(g))) / ns;
  float w = table1(c.Pg->icdfTable, SNELLY_ICDF_SAMPLES, xi);
#else
  (void)g;
  float w = 0.5f;
#endif
  if (w_out) *w_out = w;
  return wavelength_at(c, w);
}

// A scene's CONSTRUCT_PRIMARY_RAY hook works on the reference's float RNG state; the integer
// state converts to and from it exactly (all lanes are integers below 2^23).
SD_FN void primary_ray_hook(const Ctx& c, const vec2& pixel, Rng& g, vec3& start, vec3& dir) {
#ifdef HAS_CUSTOM_CAMERA
  vec4 r(float(g.s[0]), float(g.s[1]), float(g.s[2]), float(g.s[3]));
  c.sc.CONSTRUCT_PRIMARY_RAY(pixel, r, start, dir);
  g.s[0] = unsigned(r.x);
  g.s[1] = unsigned(r.y);
  g.s[2] = unsigned(r.z);
  g.s[3] = unsigned(r.w);
#else
  primary_ray(c.P, pixel, g, start, dir);
#endif
}

// All samples of one pixel for one frame (PT:1934-1989); returns the XYZ contribution.
SD_FN vec3 pixel_samples(Ctx& c, const vec2& pixel, Rng& g) {
  vec3 xyz = pick_wavelength(c, g);
  c.sun = make_frame(v3(c.P.sunDir));
  Rad L = Rad(0.0f);
  for (int n = 0; n < MAX_SAMPLES_PER_FRAME; ++n) {
    float jx = 0.5f * c.P.filterRadius * tent(rand01(g));
    float jy = 0.5f * c.P.filterRadius * tent(rand01(g));
    vec3 start, dir;
    primary_ray_hook(c, pixel + vec2(jx, jy), g, start, dir);
    L += camera_path(c, start, dir, g);
  }
  L /= float(MAX_SAMPLES_PER_FRAME);
#ifdef DISPERSION_ENABLED
  return xyz * L;
#else
  (void)xyz;
  return rgb_to_xyz(L);
#endif
}

}  // namespace sdev
