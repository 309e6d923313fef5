// pt_wavefront.cuh - wavefront integrator: the camera path of pt_integrator.cuh split into stages
// over queues of rays and paths in HBM (one job per launch, one sample per pixel per frame).
//
//   generate: camera rays (wavelength, jitter, primary ray) for every pixel -> active queue.
//   extend  : persistent warps trace the continuation rays of the active paths, the pending
//             shadow rays of the previous vertex and the rays parked by the previous iteration.
//             A lane that finishes a ray takes the next one from a global work head
//             (warp-aggregated atomics), so warps stay full however uneven the sphere-tracing
//             step counts are; when the work runs out, the longest rays are parked for the next
//             iteration instead of holding the launch. A path whose last ray finished is appended
//             to the per-material segment of the shade queue (misses and finishing paths first).
//   shade   : per path: resolve the previous vertex's deferred next-event estimate with the
//             shadow results, then run the vertex (vertex_step) with the sky/sun shadow rays
//             deferred; continuing paths and new shadow rays go to the next iteration's queues,
//             finished paths add their XYZ to the pixel's Kahan sums.
// The host launches generate once and (extend, shade) until every path of the frame has finished
// (a count the shade stage decrements); the queue counters ping-pong by iteration parity.
#pragma once
#include "pt_integrator.cuh"
#include "pt_launch.h"

#ifndef WF_REFILL
#define WF_REFILL 4  // idle lanes of a warp that trigger a refill
#endif
#ifndef WF_GRAB
#define WF_GRAB 32  // work items a warp claims from the global head at a time
#endif
#ifndef WF_CHUNK
#define WF_CHUNK 8  // sphere-tracing steps between refills
#endif
#define WF_FULL 0xffffffffu

namespace sdev {

enum { WF_INDIELE = 1, WF_FINISHING = 2, WF_NEE = 4, WF_NEE_SKY = 8, WF_NEE_SUN = 16 };

#ifdef DISPERSION_ENABLED
SD_FN Rad ld_rad(const float4& v) { return v.x; }
SD_FN float4 st_rad(const Rad& r) { return make_float4(r, 0.0f, 0.0f, 0.0f); }
#else
SD_FN Rad ld_rad(const float4& v) { return vec3(v.x, v.y, v.z); }
SD_FN float4 st_rad(const Rad& r) { return make_float4(r.x, r.y, r.z, 0.0f); }
#endif
SD_FN vec3 ld3(const float4& v) { return vec3(v.x, v.y, v.z); }
SD_FN float4 st3(const vec3& v, float w = 0.0f) { return make_float4(v.x, v.y, v.z, w); }
SD_FN unsigned lanemask_lt() { return (1u << (threadIdx.x & 31)) - 1u; }

// Warp-aggregated append: every lane calls it; lanes with `on` get consecutive slots.
SD_FN int warp_append(int* counter, bool on) {
  unsigned m = __ballot_sync(WF_FULL, on);
  if (!m) return -1;
  int leader = __ffs(m) - 1;
  int base = 0;
  if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(counter, __popc(m));
  base = __shfl_sync(WF_FULL, base, leader);
  return on ? base + __popc(m & lanemask_lt()) : -1;
}

SD_FN float enc_hit(bool hit, int mat) { return __int_as_float((hit ? 1 : 0) | ((mat + 1) << 1)); }
SD_FN void dec_hit(float w, bool& hit, int& mat) {
  int v = __float_as_int(w);
  hit = v & 1;
  mat = (v >> 1) - 1;
}

// Final contribution of a path: XYZ added to the pixel's Kahan sums, RNG written back.
SD_FN void finish_path(const JobRec& J, const WfBuffers& B, int path, const Rad& L, const vec3& xyzw, const Rng& g) {
  long long i = (long long)B.pixel_begin + path;
#ifdef DISPERSION_ENABLED
  vec3 c = xyzw * (L / float(MAX_SAMPLES_PER_FRAME));
#else
  (void)xyzw;
  vec3 c = rgb_to_xyz(L / float(MAX_SAMPLES_PER_FRAME));
#endif
  float4 s = J.acc[i], cp = J.comp[i];
  float y, t;
  y = c.x - cp.x; t = s.x + y; cp.x = (t - s.x) - y; s.x = t;
  y = c.y - cp.y; t = s.y + y; cp.y = (t - s.y) - y; s.y = t;
  y = c.z - cp.z; t = s.z + y; cp.z = (t - s.z) - y; s.z = t;
  s.w += 1.0f;
  J.acc[i] = s;
  J.comp[i] = cp;
  if (J.acc64) {
    J.acc64[4 * i + 0] += double(c.x);
    J.acc64[4 * i + 1] += double(c.y);
    J.acc64[4 * i + 2] += double(c.z);
    J.acc64[4 * i + 3] += 1.0;
  }
  J.rng[i] = make_uint4(g.s[0], g.s[1], g.s[2], g.s[3]);
}

}  // namespace sdev

extern "C" __global__ void __launch_bounds__(SNELLY_BLOCK) snelly_wf_generate(const JobRec* __restrict__ jobs,
                                                                           const SnellyParams* __restrict__ gparams,
                                                                           WfBuffers B) {
  using namespace sdev;
  const JobRec& J = jobs[0];
  int path = blockIdx.x * blockDim.x + threadIdx.x;
  if (path == 0) {
    for (int k = 0; k < WF_COUNTERS; ++k) B.cnt[k] = 0;
    B.cnt[WF_A + 0] = B.paths;
    B.cnt[WF_LEFT] = B.paths;
  }
  if (path >= B.paths) return;
  long long i = (long long)B.pixel_begin + path;
  const SnellyParams& P = c_params[0];
  uint4 r4 = J.rng[i];
  Rng g;
  g.s[0] = r4.x; g.s[1] = r4.y; g.s[2] = r4.z; g.s[3] = r4.w;
  Scene sc(uniforms_of(0));
  sc.INIT();
  Ctx c{P, gparams, sc, 0, 0.0f, vec3(0.0f), Frame()};
  const int W = J.width;
  const int x = int(i % W), y = int(i / W);
  vec3 xyzw = pick_wavelength(c, g);
  c.sun = make_frame(v3(P.sunDir));
  float jx = 0.5f * P.filterRadius * tent(rand01(g));
  float jy = 0.5f * P.filterRadius * tent(rand01(g));
  vec3 start, dir;
  primary_ray_hook(c, vec2(float(x) + 0.5f, float(y) + 0.5f) + vec2(jx, jy), g, start, dir);
  PathState s;
  start_path(c, s, start, dir);
  B.pos[path] = st3(s.pW);
  B.dir[path] = st3(s.rayDir);
  B.thr[path] = st_rad(s.thr);
  B.rad[path] = st_rad(s.L);
  B.cmf[path] = st3(c.cmf, c.lambda);
  B.mis[path] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
  B.xyzw[path] = st3(xyzw);
  B.info[path] = make_int4(0, 0, s.inDiele ? WF_INDIELE : 0, 0);
  B.rng[path] = make_uint4(g.s[0], g.s[1], g.s[2], g.s[3]);
  B.pend[path] = 1;  // the camera ray
  B.qa[0][path] = path;
}

// Trace the rays of iteration `it`: the continuation rays of the active paths, the pending shadow
// rays of their previous vertex, and rays an earlier iteration set aside unfinished.
//
// Every pass of the loop runs up to WF_CHUNK sphere-tracing steps, each evaluating the scene SDFs
// once for every lane that holds a ray; a ray's first evaluation (at its origin, which fixes the
// marching sign, PT:888-900) is such a step too, so refilled lanes march in step with the rest of
// the warp. Idle lanes are refilled when at least WF_REFILL of them are idle, or when none of the
// warp is busy, from a range of WF_GRAB items the warp claims from the global work head with one
// atomic. Once the work of the iteration is exhausted, a warp marches at most `drain` more steps
// (0: no limit) and then parks its unfinished rays (distance, sign, step count) for the next
// iteration, so no launch waits for the few longest rays. The march of a ray is the same sequence
// of operations however it is split, so results do not depend on where it was interrupted.
//
// A path is shaded once all its rays (continuation and shadows) are done: each finished ray
// decrements the path's pending count, and the last one queues the path for shading in the
// shade-queue segment of its continuation hit's material (misses and finishing paths: segment 0).
extern "C" __global__ void __launch_bounds__(SNELLY_BLOCK) snelly_wf_extend(WfBuffers B, int it, int drain) {
  using namespace sdev;
  const SnellyParams& P = c_params[0];
  Scene sc(uniforms_of(0));
  sc.INIT();
  int* cnt = B.cnt;
  const int cur = it & 1, nxt = cur ^ 1;
  if (blockIdx.x == 0 && threadIdx.x == 0) {  // queues the next shade stage and iteration fill
    cnt[WF_A + nxt] = 0;
    cnt[WF_S + nxt] = 0;
    for (int k = 0; k < 4; ++k) cnt[WF_Q + 4 * nxt + k] = 0;
  }
  const int nA = cnt[WF_A + cur], nS = cnt[WF_S + cur], nC = cnt[WF_C + cur];
  const int total = nA + nS + nC;
  const int* qa = B.qa[cur];
  const int* qs = B.qs[cur];
  const int* qc = B.qc[cur];
  int* qcnt = cnt + WF_Q + 4 * cur;
  const float minMarch = P.minLengthScale;
  const float maxLen = P.maxLengthScale;
  const int P2 = 2 * B.paths;

  bool has = false, first = false;
  int path = 0, sidx = -1;  // sidx >= 0: a shadow ray
  vec3 o(0.0f), d(0.0f);
  float t = 0.0f, sgn = 1.0f, maxd = 0.0f;
  int n = 0;
  // The warp's claimed range [wbase, wlim) of work items (warp-uniform).
  int wbase = 0, wlim = 0;
  bool wdone = false;
  int drained = 0;  // steps marched since the iteration's work ran out (warp-uniform)
  for (;;) {
    bool done = false, res_hit = false;
    int res_mat = MAT_INVAL;
    // ---- refill idle lanes ----------------------------------------------------------------
    const bool want = !has;
    const unsigned need = __ballot_sync(WF_FULL, want);
    const unsigned busy = __ballot_sync(WF_FULL, has);
    if (!wdone && need && (__popc(need) >= WF_REFILL || !busy)) {
      if (wbase >= wlim) {
        int nb = 0;
        if ((threadIdx.x & 31) == 0) nb = atomicAdd(cnt + WF_HEAD + it, WF_GRAB);
        nb = __shfl_sync(WF_FULL, nb, 0);
        wbase = nb;
        wlim = min(nb + WF_GRAB, total);
        wdone = nb >= total;
      }
      const int w = wbase + __popc(need & lanemask_lt());
      wbase = min(wbase + __popc(need), wlim);
      if (want && w < wlim) {
        int r;  // ray id: 2 * path + light for a shadow ray, 2 * paths + path for a continuation
        bool resume = false;
        if (w < nA) {
          r = P2 + qa[w];
        } else if (w < nA + nS) {
          r = qs[w - nA];
        } else {
          r = qc[w - nA - nS];
          resume = true;
        }
        if (r >= P2) {
          path = r - P2;
          sidx = -1;
          o = ld3(B.pos[path]);
          d = ld3(B.dir[path]);
          maxd = maxLen;
        } else {
          sidx = r;
          path = sidx >> 1;
          o = ld3(B.nee_org[path]);
          float4 dd = B.nee_dir[sidx & 1][path];
          d = ld3(dd);
          maxd = dd.w;
        }
        has = true;
        first = !resume;
        if (resume) {
          float4 m = B.mt[r];
          t = m.x;
          sgn = m.y;
          n = __float_as_int(m.z);
        }
      }
    }
    // ---- up to WF_CHUNK sphere-tracing steps (PT:888-919); a lane stops when its ray is done ----
    for (int k = 0; k < WF_CHUNK && has && !done; ++k) {
      const vec3 p = first ? o : o + t * d;
      float sdf = 1.0e20f;
      int m = MAT_INVAL;
#ifdef HAS_SURFACE
      {
        float dd = fabsf(sc.SDF_SURFACE(p));
        if (!first && dd < minMarch) m = MAT_SURFA;
        sdf = fminf(sdf, dd);
      }
#endif
#ifdef HAS_METAL
      if (m == MAT_INVAL) {
        float dd = fabsf(sc.SDF_METAL(p));
        if (!first && dd < minMarch) m = MAT_METAL;
        sdf = fminf(sdf, dd);
      }
#endif
#ifdef HAS_DIELECTRIC
      if (m == MAT_INVAL) {
        float dd = fabsf(sc.SDF_DIELECTRIC(p));
        if (!first && dd < minMarch) m = MAT_DIELE;
        sdf = fminf(sdf, dd);
      }
#endif
      if (first) {  // the distance at the origin fixes the marching sign and the first step
        first = false;
        sgn = glsl::sign(sdf);
        t = sgn * sdf;
        n = 0;
        if (fabsf(t) >= maxd) {
          done = true;
          res_hit = false;
        }
      } else if (m != MAT_INVAL) {
        done = true;
        res_hit = true;
        res_mat = m;
      } else {
        t += sgn * sdf;
        if (fabsf(t) >= maxd) {
          done = true;
          res_hit = false;
        } else if (++n >= MAX_MARCH_STEPS) {  // out of steps: a hit at the zero position unless maxStepsIsMiss
          done = true;
          res_hit = !P.maxStepsIsMiss;
          res_mat = MAT_INVAL;
          t = 0.0f;
          o = vec3(0.0f);
          d = vec3(0.0f);
        }
      }
    }
    if (wdone) drained += WF_CHUNK;
    const bool park = drain > 0 && drained >= drain && has && !done;  // set aside for the next iteration
    // ---- results ---------------------------------------------------------------------------
    if (__any_sync(WF_FULL, done || park)) {
      int seg = -1;
      if (done) {
        if (sidx < 0) B.hit[path] = st3(o + t * d, enc_hit(res_hit, res_mat));
        else B.shadow[sidx] = res_hit ? 1 : 0;
        __threadfence();
        if (atomicSub(B.pend + path, 1) == 1) {  // the path's last ray: queue it for shading
          bool h;
          int hm;
          if (sidx < 0) {
            h = res_hit;
            hm = res_mat;
          } else {
            dec_hit(__ldcg(&B.hit[path].w), h, hm);
          }
          seg = !h ? 0 : (hm == MAT_SURFA ? 1 : (hm == MAT_METAL ? 2 : (hm == MAT_DIELE ? 3 : 0)));
        }
      }
      for (int sgi = 0; sgi < 4; ++sgi) {
        int slot = warp_append(qcnt + sgi, seg == sgi);
        if (slot >= 0) B.qshade[cur][sgi * B.paths + slot] = path;
      }
      const int r = sidx >= 0 ? sidx : P2 + path;
      if (park) B.mt[r] = make_float4(t, sgn, __int_as_float(n), 0.0f);
      int slot = warp_append(cnt + WF_C + nxt, park);
      if (slot >= 0) B.qc[nxt][slot] = r;
      if (done || park) has = false;
    }
    if (wdone && !__any_sync(WF_FULL, has)) break;
  }
}

// Shade every path the extend stage of iteration `it` queued, and count the frame's paths down.
extern "C" __global__ void __launch_bounds__(SNELLY_BLOCK, SNELLY_SHADE_MIN_BLOCKS) snelly_wf_shade(const JobRec* __restrict__ jobs,
                                                                        const SnellyParams* __restrict__ gparams,
                                                                        WfBuffers B, int it) {
  using namespace sdev;
  const JobRec& J = jobs[0];
  const SnellyParams& P = c_params[0];
  int* cnt = B.cnt;
  const int cur = it & 1, nxt = cur ^ 1;
  const int* qc = cnt + WF_Q + 4 * cur;
  const int n0 = qc[0], n1 = qc[1], n2 = qc[2], n3 = qc[3];
  const int total = n0 + n1 + n2 + n3;
  if (blockIdx.x == 0 && threadIdx.x == 0) cnt[WF_C + cur] = 0;  // filled again by the next extend stage
  Scene sc(uniforms_of(0));
  sc.INIT();
  const int stride = gridDim.x * blockDim.x;
  for (int base = blockIdx.x * blockDim.x; base < total; base += stride) {
    int w = base + threadIdx.x;
    bool valid = w < total;
    int path = 0;
    bool push_active = false, push_direct = false, finished = false;
    int push_shadow = 0;  // bit 0: sky, bit 1: sun
    if (valid) {
      int seg = w < n0 ? 0 : (w < n0 + n1 ? 1 : (w < n0 + n1 + n2 ? 2 : 3));
      int off = w - (seg == 0 ? 0 : (seg == 1 ? n0 : (seg == 2 ? n0 + n1 : n0 + n1 + n2)));
      path = B.qshade[cur][seg * B.paths + off];
      int4 info = B.info[path];
      float4 cm = B.cmf[path];
      Ctx c{P, gparams, sc, 0, cm.w, ld3(cm), make_frame(v3(P.sunDir))};
      PathState s;
      s.pW = ld3(B.pos[path]);
      s.rayDir = ld3(B.dir[path]);
      s.thr = ld_rad(B.thr[path]);
      s.L = ld_rad(B.rad[path]);
      float4 mw = B.mis[path];
      s.misSky = mw.x;
      s.misSun = mw.y;
      s.misSph = mw.z;
      s.atmScatters = info.y;
      s.inDiele = info.z & WF_INDIELE;
      uint4 r4 = B.rng[path];
      Rng g;
      g.s[0] = r4.x; g.s[1] = r4.y; g.s[2] = r4.z; g.s[3] = r4.w;
      int flags = info.z;
      if (flags & WF_NEE) {  // the previous vertex's next-event estimate, now that its shadows are traced
        DeferredNee nd;
        nd.org = ld3(B.nee_org[path]);
        nd.thr = ld_rad(B.nee_thr[path]);
        nd.extra = ld_rad(B.nee_extra[path]);
        bool occ[2] = {false, false};
        for (int l = 0; l < 2; ++l) {
          nd.pending[l] = flags & (l == 0 ? WF_NEE_SKY : WF_NEE_SUN);
          if (nd.pending[l]) {
            float4 dd = B.nee_dir[l][path];
            nd.dir[l] = ld3(dd);
            nd.dist[l] = dd.w;
            nd.c[l] = ld_rad(B.nee_c[l][path]);
            nd.li[l] = ld_rad(B.nee_li[l][path]);
            occ[l] = B.shadow[2 * path + l];
          }
        }
        s.L += resolve_deferred(c, nd, occ);
        flags &= ~(WF_NEE | WF_NEE_SKY | WF_NEE_SUN);
      }
      bool continues = false;
      if (flags & WF_FINISHING) {
        finished = true;
      } else {
        float4 hw = B.hit[path];
        Hit h;
        h.p = ld3(hw);
        dec_hit(hw.w, h.hit, h.mat);
        int vertex = info.x;
        DeferredNee nd;
        nd.any = false;
        int r = vertex_step(c, s, h, vertex, g, &nd);
        ++vertex;
        finished = r == VERTEX_DONE || vertex > max_bounces(P) || maxc(s.thr) < kThroughputEps;
        continues = !finished;
        if (nd.any) {
          flags |= WF_NEE;
          B.nee_org[path] = st3(nd.org);
          B.nee_thr[path] = st_rad(nd.thr);
          B.nee_extra[path] = st_rad(nd.extra);
          for (int l = 0; l < 2; ++l)
            if (nd.pending[l]) {
              flags |= (l == 0 ? WF_NEE_SKY : WF_NEE_SUN);
              B.nee_dir[l][path] = st3(nd.dir[l], nd.dist[l]);
              B.nee_c[l][path] = st_rad(nd.c[l]);
              B.nee_li[l][path] = st_rad(nd.li[l]);
              push_shadow |= 1 << l;
            }
          if (finished) flags |= WF_FINISHING;  // one more pass to resolve the shadows
          finished = false;
        }
        info.x = vertex;
      }
      s.inDiele ? (flags |= WF_INDIELE) : (flags &= ~WF_INDIELE);
      if (finished) {
        finish_path(J, B, path, s.L, ld3(B.xyzw[path]), g);
      } else {
        B.pos[path] = st3(s.pW);
        B.dir[path] = st3(s.rayDir);
        B.thr[path] = st_rad(s.thr);
        B.rad[path] = st_rad(s.L);
        B.mis[path] = make_float4(s.misSky, s.misSun, s.misSph, 0.0f);
        B.info[path] = make_int4(info.x, s.atmScatters, flags, 0);
        B.rng[path] = make_uint4(g.s[0], g.s[1], g.s[2], g.s[3]);
        // rays the path waits for: its continuation (unless it only resolves its shadows) and
        // its shadow rays; a path with none goes straight to the next shade stage
        const int nrays = (continues ? 1 : 0) + __popc(push_shadow);
        if (!continues) B.hit[path] = make_float4(0.0f, 0.0f, 0.0f, enc_hit(false, MAT_INVAL));
        B.pend[path] = nrays;
        push_active = continues;
        push_direct = nrays == 0;
      }
    }
    int slot = warp_append(cnt + WF_A + nxt, push_active);
    if (slot >= 0) B.qa[nxt][slot] = path;
    for (int l = 0; l < 2; ++l) {
      int ss = warp_append(cnt + WF_S + nxt, (push_shadow >> l) & 1);
      if (ss >= 0) B.qs[nxt][ss] = 2 * path + l;
    }
    // a path with no ray to wait for goes straight to the next shade stage's queue (the other
    // buffer: this launch is still reading its own)
    int ds = warp_append(cnt + WF_Q + 4 * nxt, push_direct);
    if (ds >= 0) B.qshade[nxt][ds] = path;
    unsigned fin = __ballot_sync(WF_FULL, finished);
    if (fin && (int)(threadIdx.x & 31) == __ffs(fin) - 1) atomicSub(cnt + WF_LEFT, __popc(fin));
  }
}
