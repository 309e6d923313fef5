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
// The host launches generate once and (extend, shade) until every path has finished (a count the
// shade stage decrements); the queue counters ping-pong by iteration parity. One generate launch
// may start several samples per pixel (B.samples): a path that finishes one sample of its pixel
// starts the next in place, with the RNG state the finished one left, so the frames of a launch
// sequence overlap (no stage waits for the last paths of a frame) and every pixel still draws
// its random numbers and adds its samples in the same order as frame by frame.
#pragma once
#include "pt_integrator.cuh"
#include "pt_launch.h"

#define WF_FULL 0xffffffffu

namespace sdev {

enum { WF_INDIELE = 1, WF_FINISHING = 2, WF_NEE = 4, WF_NEE_SKY = 8, WF_NEE_SUN = 16 };
// flags bits from here up: the index of the path's sample among those of its launch sequence
#define WF_SAMPLE_SHIFT 8

// ---- the path record ----------------------------------------------------------------------------
// One path's state: WF_REC float4 slots, contiguous. Slots a stage reads together sit in the same
// 32-byte sectors: extend reads R_POS + R_DIR (one sector) for a continuation ray, R_NORG and one
// shadow direction for a shadow ray; shade reads R_POS..R_INFO (96 bytes) and, when the previous
// vertex deferred its light estimate, R_NORG..R_NC. The colour-matching weights are rebuilt from
// the wavelength parameter w (in R_INFO.w) instead of being stored. With a surface material the
// record ends with the subsurface-walk hand-over (R_S0..), written only by paths that take it.
#ifdef DISPERSION_ENABLED
enum {
  R_POS = 0,    // vertex pW (xyz), throughput (w)
  R_DIR = 1,    // ray direction (xyz), radiance L (w)
  R_HIT = 2,    // continuation hit position (xyz), encoded hit flag and material (w)
  R_MIS = 3,    // MIS weights sky, sun, sphere (xyz), deferred estimate's sphere-light term (w)
  R_RNG = 4,    // RNG lanes
  R_INFO = 5,   // vertex, atmosphere scatters, flags, wavelength parameter w (float bits)
  R_NORG = 6,   // shadow-ray origin (xyz), throughput at the deferred estimate's vertex (w)
  R_NDIR = 7,   // [2] sky, sun shadow directions (xyz) and lengths (w)
  R_NC = 9,     // unoccluded contributions c0, c1 and unshadowed radiance li0, li1
  R_S0 = 10,    // subsurface entry: shading normal (xyz), probSSS (w)
  R_S1 = 11,    // tangent (xyz), subsurface albedo (w)
  R_S2 = 12,    // bitangent (xyz)
  R_S3 = 13,    // geometric normal (xyz)
  R_BASE = 10
};
#else
enum {
  R_POS = 0,    // pW (xyz), misSky (w)
  R_DIR = 1,    // ray direction (xyz), misSun (w)
  R_HIT = 2,    // hit position (xyz), encoded hit (w)
  R_THR = 3,    // throughput (xyz), misSph (w)
  R_L = 4,      // radiance (xyz)
  R_RNG = 5,
  R_INFO = 6,   // vertex, atmosphere scatters, flags, unused
  R_NORG = 7,   // shadow-ray origin (xyz)
  R_NDIR = 8,   // [2] shadow directions and lengths
  R_NTHR = 10,  // throughput at the deferred estimate's vertex
  R_NEXTRA = 11,  // sphere-light term
  R_NC = 12,    // [2] unoccluded contributions
  R_NLI = 14,   // [2] unshadowed radiance
  R_S0 = 16,    // shading normal (xyz), probSSS (w)
  R_S1 = 17,    // tangent
  R_S2 = 18,    // bitangent
  R_S3 = 19,    // geometric normal
  R_S4 = 20,    // subsurface albedo (xyz)
  R_BASE = 16
};
#endif
#ifdef HAS_SURFACE
#ifdef DISPERSION_ENABLED
#define WF_REC 14
#else
#define WF_REC 21
#endif
#else
#define WF_REC R_BASE
#endif

SD_FN vec3 ld3(const float4& v) { return vec3(v.x, v.y, v.z); }
SD_FN float4 st3(const vec3& v, float w = 0.0f) { return make_float4(v.x, v.y, v.z, w); }
SD_FN unsigned lanemask_lt() { return (1u << (threadIdx.x & 31)) - 1u; }
SD_FN float4* rec_of(float4* rec, int path) { return rec + (size_t)path * WF_REC; }
// One of a ping-pong pair of queues. A select, not an index: a kernel parameter block indexed with
// a run-time value is copied to local memory.
SD_FN int* pp(int* const (&q)[2], int k) { return k ? q[1] : q[0]; }

// The part of PathState a path carries between stages, and its bookkeeping.
struct WfState {
  PathState s;
  Rng g;
  int vertex, flags;
  float w;  // wavelength parameter
};

SD_FN void load_state(const float4* r, WfState& st) {
  float4 a = r[R_POS], b = r[R_DIR];
  uint4 q = *reinterpret_cast<const uint4*>(r + R_RNG);
  int4 in = *reinterpret_cast<const int4*>(r + R_INFO);
  st.s.pW = ld3(a);
  st.s.rayDir = ld3(b);
#ifdef DISPERSION_ENABLED
  float4 m = r[R_MIS];
  st.s.thr = a.w;
  st.s.L = b.w;
  st.s.misSky = m.x;
  st.s.misSun = m.y;
  st.s.misSph = m.z;
#else
  float4 t = r[R_THR], l = r[R_L];
  st.s.thr = ld3(t);
  st.s.L = ld3(l);
  st.s.misSky = a.w;
  st.s.misSun = b.w;
  st.s.misSph = t.w;
#endif
  st.g.s[0] = q.x; st.g.s[1] = q.y; st.g.s[2] = q.z; st.g.s[3] = q.w;
  st.vertex = in.x;
  st.s.atmScatters = in.y;
  st.flags = in.z;
  st.w = __int_as_float(in.w);
  st.s.inDiele = in.z & WF_INDIELE;
}

SD_FN void store_state(float4* r, const WfState& st, float nee_extra_w = 0.0f) {
  (void)nee_extra_w;
#ifdef DISPERSION_ENABLED
  r[R_POS] = st3(st.s.pW, st.s.thr);
  r[R_DIR] = st3(st.s.rayDir, st.s.L);
  r[R_MIS] = make_float4(st.s.misSky, st.s.misSun, st.s.misSph, nee_extra_w);
#else
  r[R_POS] = st3(st.s.pW, st.s.misSky);
  r[R_DIR] = st3(st.s.rayDir, st.s.misSun);
  r[R_THR] = st3(st.s.thr, st.s.misSph);
  r[R_L] = st3(st.s.L);
#endif
  *reinterpret_cast<uint4*>(r + R_RNG) = make_uint4(st.g.s[0], st.g.s[1], st.g.s[2], st.g.s[3]);
  *reinterpret_cast<int4*>(r + R_INFO) = make_int4(st.vertex, st.s.atmScatters, st.flags, __float_as_int(st.w));
}

// The deferred next-event estimate of a path's previous vertex.
SD_FN void store_nee(float4* r, const DeferredNee& nd) {
#ifdef DISPERSION_ENABLED
  r[R_NORG] = st3(nd.org, nd.thr);
  r[R_NC] = make_float4(nd.c[0], nd.c[1], nd.li[0], nd.li[1]);
#else
  r[R_NORG] = st3(nd.org);
  r[R_NTHR] = st3(nd.thr);
  r[R_NEXTRA] = st3(nd.extra);
  for (int l = 0; l < 2; ++l) {
    r[R_NC + l] = st3(nd.c[l]);
    r[R_NLI + l] = st3(nd.li[l]);
  }
#endif
  for (int l = 0; l < 2; ++l)
    if (nd.pending[l]) r[R_NDIR + l] = st3(nd.dir[l], nd.dist[l]);
}
SD_FN void load_nee(const float4* r, DeferredNee& nd, int flags) {
  float4 o = r[R_NORG];
  nd.org = ld3(o);
#ifdef DISPERSION_ENABLED
  float4 cc = r[R_NC];
  nd.thr = o.w;
  nd.extra = r[R_MIS].w;
  nd.c[0] = cc.x;
  nd.c[1] = cc.y;
  nd.li[0] = cc.z;
  nd.li[1] = cc.w;
#else
  nd.thr = ld3(r[R_NTHR]);
  nd.extra = ld3(r[R_NEXTRA]);
  for (int l = 0; l < 2; ++l) {
    nd.c[l] = ld3(r[R_NC + l]);
    nd.li[l] = ld3(r[R_NLI + l]);
  }
#endif
  for (int l = 0; l < 2; ++l) {
    nd.pending[l] = flags & (l == 0 ? WF_NEE_SKY : WF_NEE_SUN);
    if (nd.pending[l]) {
      float4 dd = r[R_NDIR + l];
      nd.dir[l] = ld3(dd);
      nd.dist[l] = dd.w;
    }
  }
}

#ifdef HAS_SURFACE
SD_FN void store_sss(float4* r, const SssEntry& e) {
#ifdef DISPERSION_ENABLED
  r[R_S0] = st3(e.fr.n, e.probSSS);
  r[R_S1] = st3(e.fr.t, e.ssAlb);
  r[R_S2] = st3(e.fr.b);
  r[R_S3] = st3(e.ngW);
#else
  r[R_S0] = st3(e.fr.n, e.probSSS);
  r[R_S1] = st3(e.fr.t);
  r[R_S2] = st3(e.fr.b);
  r[R_S3] = st3(e.ngW);
  r[R_S4] = st3(e.ssAlb);
#endif
}
SD_FN SssEntry load_sss(const float4* r) {
  SssEntry e;
  float4 a = r[R_S0], b = r[R_S1];
  e.fr.n = ld3(a);
  e.probSSS = a.w;
  e.fr.t = ld3(b);
  e.fr.b = ld3(r[R_S2]);
  e.ngW = ld3(r[R_S3]);
#ifdef DISPERSION_ENABLED
  e.ssAlb = b.w;
#else
  e.ssAlb = ld3(r[R_S4]);
#endif
  return e;
}
#endif

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

// Entry of every wavefront kernel. With programmatic dependent launch (the host's launch attribute)
// the kernel may start while the previous kernel of its stream is still running: it first waits
// for that grid to complete and its writes to be visible (griddepcontrol.wait, a no-op without
// the attribute), then lets the next kernel of the stream begin launching, so its launch and block
// set-up overlap this one's work.
SD_FN void wf_kernel_entry() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// The pixel a path of this range traces: the range's contiguous pixels from pixel_begin, or,
// with interleaved ranges, the path's group among those dealt to range pixel_begin in turn
// (group b of the image goes to range b mod pixel_parts).
SD_FN long long pixel_of(const WfBuffers& B, int path) {
  if (B.pixel_group <= 0) return (long long)B.pixel_begin + path;
  const int g = path / B.pixel_group;
  return ((long long)g * B.pixel_parts + B.pixel_begin) * B.pixel_group + (path - g * B.pixel_group);
}

// Final contribution of a path: XYZ added to the pixel's Kahan sums, and the RNG state written back
// when it is the pixel's last sample of the launch sequence (save_rng).
SD_FN void finish_path(const JobRec& J, const WfBuffers& B, int path, const Rad& L, const vec3& xyzw, const Rng& g,
                       bool save_rng) {
  long long i = pixel_of(B, path);
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
  if (save_rng) J.rng[i] = make_uint4(g.s[0], g.s[1], g.s[2], g.s[3]);
}

// A camera sample of pixel i (PT:1934-1955): the wavelength, the filter jitter and the primary
// ray, drawn from st.g in that order; the path starts over at vertex 0 as sample `sample`.
SD_FN void start_sample(Ctx& c, const JobRec& J, long long i, WfState& st, int sample) {
  const SnellyParams& P = c.P;
  const int W = J.width;
  const int x = int(i % W), y = int(i / W);
  pick_wavelength(c, st.g, &st.w);
  float jx = 0.5f * P.filterRadius * tent(rand01(st.g));
  float jy = 0.5f * P.filterRadius * tent(rand01(st.g));
  vec3 start, dir;
  primary_ray_hook(c, vec2(float(x) + 0.5f, float(y) + 0.5f) + vec2(jx, jy), st.g, start, dir);
  start_path(c, st.s, start, dir);
  st.vertex = 0;
  st.flags = (st.s.inDiele ? WF_INDIELE : 0) | (sample << WF_SAMPLE_SHIFT);
}

// A path whose sample just finished: the pixel's sample is added, and unless it was the pixel's
// last of the launch sequence the next one starts in the same record, waiting for its camera ray
// (returns true: the caller queues the path as active).
SD_FN bool finish_sample(Ctx& c, const JobRec& J, const WfBuffers& B, int path, WfState& st, const vec3& xyzw) {
  const int sample = (st.flags >> WF_SAMPLE_SHIFT) + 1;
  const bool more = sample < B.samples;
  finish_path(J, B, path, st.s.L, xyzw, st.g, !more);
  if (!more) return false;
  start_sample(c, J, pixel_of(B, path), st, sample);
  store_state(rec_of(B.rec, path), st);
  B.pend[path] = 1;
  return true;
}

}  // namespace sdev

// Record layout the host allocates for (float4 slots per path).
extern "C" __constant__ int snelly_wf_rec_f4 = WF_REC;

extern "C" __global__ void __launch_bounds__(SNELLY_BLOCK) snelly_wf_generate(const JobRec* __restrict__ jobs,
                                                                           const SnellyParams* __restrict__ gparams,
                                                                           WfBuffers B) {
  using namespace sdev;
  wf_kernel_entry();
  const JobRec& J = jobs[0];
  int path = blockIdx.x * blockDim.x + threadIdx.x;
  if (B.rec_f4 != snelly_wf_rec_f4) {  // buffers laid out for another record size: trace nothing
    if (path == 0)
      for (int k = 0; k < WF_COUNTERS; ++k) B.cnt[k] = 0;
    return;
  }
  if (path == 0) {
    for (int k = 0; k < WF_COUNTERS; ++k) B.cnt[k] = 0;
    B.cnt[WF_A + 0] = B.paths;
    B.cnt[WF_LEFT] = B.paths;
  }
  if (path >= B.paths) return;
  long long i = pixel_of(B, path);
  const SnellyParams& P = c_params[B.slot];
  uint4 r4 = J.rng[i];
  WfState st;
  st.g.s[0] = r4.x; st.g.s[1] = r4.y; st.g.s[2] = r4.z; st.g.s[3] = r4.w;
  Scene sc(uniforms_of(B.slot));
  sc.INIT();
  Ctx c{P, gparams, sc, B.slot, 0.0f, vec3(0.0f), make_frame(v3(P.sunDir))};
  start_sample(c, J, i, st, 0);
  store_state(rec_of(B.rec, path), st);
  B.pend[path] = 1;  // the camera ray
  B.qa[0][path] = path;
}

// Trace the rays of iteration `it`: the continuation rays of the active paths, the pending shadow
// rays of their previous vertex, and rays an earlier iteration set aside unfinished.
//
// Every pass of the loop runs up to `chunk` sphere-tracing steps, each evaluating the scene SDFs
// once for every lane that holds a ray; a ray's first evaluation (at its origin, which fixes the
// marching sign, PT:888-900) is such a step too, so refilled lanes march in step with the rest of
// the warp. Idle lanes are refilled when at least `refill` of them are idle, or when none of the
// warp is busy, from a range of `grab` items the warp claims from the global work head with one
// atomic (all three chosen by the host's autotuner; 8, 32 and 8 by default). Once the work of the
// iteration is exhausted, a warp marches at most `drain` more steps
// (0: no limit) and then parks its unfinished rays (distance, sign, step count) for the next
// iteration, so no launch waits for the few longest rays. The march of a ray is the same sequence
// of operations however it is split, so results do not depend on where it was interrupted.
//
// A path is shaded once all its rays (continuation and shadows) are done: each finished ray
// decrements the path's pending count, and the last one queues the path for shading in the
// shade-queue segment of its continuation hit's material (misses and finishing paths: segment 0).
extern "C" __global__ void __launch_bounds__(SNELLY_BLOCK) snelly_wf_extend(WfBuffers B, int it, int drain, int chunk,
                                                                                  int grab, int refill) {
  using namespace sdev;
  wf_kernel_entry();
  const SnellyParams& P = c_params[B.slot];
  Scene sc(uniforms_of(B.slot));
  sc.INIT();
  int* cnt = B.cnt;
  const int cur = it & 1, nxt = cur ^ 1;
  if (blockIdx.x == 0 && threadIdx.x == 0) {  // queues the next shade stage and iteration fill
    cnt[WF_A + nxt] = 0;
    cnt[WF_S + nxt] = 0;
    cnt[WF_SSS] = 0;
    cnt[WF_WHEAD] = 0;
    cnt[WF_XQ] = 0;
    cnt[WF_VOL] = 0;
    cnt[WF_HEAD + nxt] = 0;
    for (int k = 0; k < 4; ++k) cnt[WF_Q + 4 * nxt + k] = 0;
  }
  const int nA = cnt[WF_A + cur], nS = cnt[WF_S + cur], nC = cnt[WF_C + cur];
  const int total = nA + nS + nC;
  const int* qa = pp(B.qa, cur);
  const int* qs = pp(B.qs, cur);
  const int* qc = pp(B.qc, cur);
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
    if (!wdone && need && (__popc(need) >= refill || !busy)) {
      if (wbase >= wlim) {
        int nb = 0;
        if ((threadIdx.x & 31) == 0) nb = atomicAdd(cnt + WF_HEAD + cur, grab);
        nb = __shfl_sync(WF_FULL, nb, 0);
        wbase = nb;
        wlim = min(nb + grab, total);
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
          const float4* rp = rec_of(B.rec, path);
          o = ld3(rp[R_POS]);
          d = ld3(rp[R_DIR]);
          maxd = maxLen;
        } else {
          sidx = r;
          path = sidx >> 1;
          const float4* rp = rec_of(B.rec, path);
          o = ld3(rp[R_NORG]);
          float4 dd = rp[R_NDIR + (sidx & 1)];
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
    // ---- up to `chunk` sphere-tracing steps (PT:888-919); a lane stops when its ray is done ----
    for (int k = 0; k < chunk && has && !done; ++k) {
      const vec3 p = first ? o : o + t * d;
      float sdf = 1.0e20f;
      int m = MAT_INVAL;
      // Every SDF, unconditionally, and the hit named by selects: the first of surface, metal,
      // dielectric below the threshold, as the reference's early returns decide (PT:906-912). No
      // branch around an SDF, so the warp does not split where one lane's ray hits; the extra
      // evaluations on a hit step change nothing (the march ends there).
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
      if (first) m = MAT_INVAL;  // the origin is never a hit (its distance only fixes the sign)
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
    if (wdone) drained += chunk;
    const bool park = drain > 0 && drained >= drain && has && !done;  // set aside for the next iteration
    // ---- results ---------------------------------------------------------------------------
    if (__any_sync(WF_FULL, done || park)) {
      int seg = -1;
      if (done) {
        if (sidx < 0) rec_of(B.rec, path)[R_HIT] = st3(o + t * d, enc_hit(res_hit, res_mat));
        else B.shadow[sidx] = res_hit ? 1 : 0;
        __threadfence();
        if (atomicSub(B.pend + path, 1) == 1) {  // the path's last ray: queue it for shading
          bool h;
          int hm;
          if (sidx < 0) {
            h = res_hit;
            hm = res_mat;
          } else {
            dec_hit(__ldcg(&rec_of(B.rec, path)[R_HIT].w), h, hm);
          }
          seg = !h ? 0 : (hm == MAT_SURFA ? 1 : (hm == MAT_METAL ? 2 : (hm == MAT_DIELE ? 3 : 0)));
        }
      }
      for (int sgi = 0; sgi < 4; ++sgi) {
        int slot = warp_append(qcnt + sgi, seg == sgi);
        if (slot >= 0) pp(B.qshade, cur)[sgi * B.paths + slot] = path;
      }
      const int r = sidx >= 0 ? sidx : P2 + path;
      if (park) B.mt[r] = make_float4(t, sgn, __int_as_float(n), 0.0f);
      int slot = warp_append(cnt + WF_C + nxt, park);
      if (slot >= 0) pp(B.qc, nxt)[slot] = r;
      if (done || park) has = false;
    }
    if (wdone && !__any_sync(WF_FULL, has)) break;
  }
}

// ---- shading -------------------------------------------------------------------------------------
namespace sdev {

// Shade one queued path of iteration `it`: resolve the previous vertex's deferred next-event
// estimate with its shadow results, run the vertex (vertex_step) with the sky/sun shadow rays
// deferred, and queue what the path waits for next. MAT is the material every path of the calling
// kernel hit (MAT_INVAL: read it from the record). Returns true when the path finished. With
// B.vol_stage, a vertex that collides in the heterogeneous medium stops at the collision point
// (kept in the R_HIT slot) and joins the volume stage's queue (push_vol).
template <int MAT>
SD_FN void shade_path(const JobRec& J, const SnellyParams* gparams, const WfBuffers& B, Scene& sc, int path, int nxt,
                      bool& push_active, int& push_shadow, bool& push_direct, bool& push_sss, bool& push_vol,
                      bool& finished) {
  const SnellyParams& P = c_params[B.slot];
  float4* r = rec_of(B.rec, path);
  WfState st;
  load_state(r, st);
  Ctx c{P, gparams, sc, B.slot, 0.0f, vec3(0.0f), make_frame(v3(P.sunDir))};
  const vec3 xyzw = wavelength_at(c, st.w);
  int flags = st.flags;
  if (flags & WF_NEE) {  // the previous vertex's next-event estimate, now that its shadows are traced
    DeferredNee nd;
    load_nee(r, nd, flags);
    bool occ[2] = {false, false};
    for (int l = 0; l < 2; ++l)
      if (nd.pending[l]) occ[l] = B.shadow[2 * path + l];
    st.s.L += resolve_deferred(c, nd, occ);
    flags &= ~(WF_NEE | WF_NEE_SKY | WF_NEE_SUN);
  }
  bool continues = false;
  float extra_w = 0.0f;
  if (flags & WF_FINISHING) {
    finished = true;
  } else {
    float4 hw = r[R_HIT];
    Hit h;
    h.p = ld3(hw);
    dec_hit(hw.w, h.hit, h.mat);
    if (MAT != MAT_INVAL) {  // every path of this kernel hit material MAT
      h.hit = true;
      h.mat = MAT;
    }
    DeferredNee nd;
    nd.any = false;
    vec3 vps(0.0f);  // a collision in the heterogeneous medium, handed to the volume stage
    vec3* volp = nullptr;
#ifdef HAS_HETERO_VOLUME
    if (B.vol_stage) volp = &vps;
#endif
#ifdef HAS_SURFACE
    SssEntry se;
    int rv = vertex_step(c, st.s, h, st.vertex, st.g, &nd, &se, volp);
    if (rv == VERTEX_SSS) {  // the walk stage finishes this vertex
      store_sss(r, se);
      st.flags = (flags & ~WF_INDIELE) | (st.s.inDiele ? WF_INDIELE : 0);
      store_state(r, st);
      push_sss = true;
      return;
    }
#else
    int rv = vertex_step(c, st.s, h, st.vertex, st.g, &nd, nullptr, volp);
#endif
    if (rv == VERTEX_VOLUME) {  // the volume stage finishes this vertex
      r[R_HIT] = st3(vps, enc_hit(false, MAT_INVAL));
      st.flags = (flags & ~WF_INDIELE) | (st.s.inDiele ? WF_INDIELE : 0);
      store_state(r, st);
      push_vol = true;
      return;
    }
    ++st.vertex;
    finished = rv == VERTEX_DONE || st.vertex > max_bounces(P) || maxc(st.s.thr) < kThroughputEps;
    continues = !finished;
    if (nd.any) {
      flags |= WF_NEE;
      for (int l = 0; l < 2; ++l)
        if (nd.pending[l]) {
          flags |= (l == 0 ? WF_NEE_SKY : WF_NEE_SUN);
          push_shadow |= 1 << l;
        }
      store_nee(r, nd);
#ifdef DISPERSION_ENABLED
      extra_w = nd.extra;
#endif
      if (finished) flags |= WF_FINISHING;  // one more pass to resolve the shadows
      finished = false;
    }
  }
  st.s.inDiele ? (flags |= WF_INDIELE) : (flags &= ~WF_INDIELE);
  if (finished) {
    st.flags = flags;
    if (finish_sample(c, J, B, path, st, xyzw)) {  // the pixel's next sample: its camera ray
      finished = false;
      push_active = true;
    }
    return;
  }
  st.flags = flags;
  store_state(r, st, extra_w);
  // rays the path waits for: its continuation (unless it only resolves its shadows) and its
  // shadow rays; a path with none goes straight to the next shade stage
  const int nrays = (continues ? 1 : 0) + __popc(push_shadow);
  if (!continues) r[R_HIT] = make_float4(0.0f, 0.0f, 0.0f, enc_hit(false, MAT_INVAL));
  B.pend[path] = nrays;
  push_active = continues;
  push_direct = nrays == 0;
  (void)nxt;
}

// Queue the outcome of a warp's shaded paths for the next iteration, and count finished paths.
SD_FN void shade_push(const WfBuffers& B, int* cnt, int nxt, int path, bool push_active, int push_shadow,
                      bool push_direct, bool push_sss, bool finished, bool push_vol = false) {
  int slot = warp_append(cnt + WF_A + nxt, push_active);
  if (slot >= 0) pp(B.qa, nxt)[slot] = path;
  for (int l = 0; l < 2; ++l) {
    int ss = warp_append(cnt + WF_S + nxt, (push_shadow >> l) & 1);
    if (ss >= 0) pp(B.qs, nxt)[ss] = 2 * path + l;
  }
  // a path with no ray to wait for goes straight to the next shade stage's queue (the other
  // buffer: this iteration's shade launches are still reading their own)
  int ds = warp_append(cnt + WF_Q + 4 * nxt, push_direct);
  if (ds >= 0) pp(B.qshade, nxt)[ds] = path;
  int ws = warp_append(cnt + WF_SSS, push_sss);
  if (ws >= 0) B.qsss[ws] = path;
#ifdef HAS_HETERO_VOLUME
  int vs = warp_append(cnt + WF_VOL, push_vol);
  if (vs >= 0) B.qvol[vs] = path;
#else
  (void)push_vol;
#endif
  unsigned fin = __ballot_sync(WF_FULL, finished);
  if (fin && (int)(threadIdx.x & 31) == __ffs(fin) - 1) atomicSub(cnt + WF_LEFT, __popc(fin));
}

// The shade stage over segments [seg_lo, seg_hi] of iteration `it`'s shade queue.
template <int MAT>
SD_FN void shade_segments(const JobRec* jobs, const SnellyParams* gparams, const WfBuffers& B, int it, int seg_lo,
                          int seg_hi) {
  wf_kernel_entry();
  const JobRec& J = jobs[0];
  int* cnt = B.cnt;
  const int cur = it & 1, nxt = cur ^ 1;
  const int* qn = cnt + WF_Q + 4 * cur;
  const int n0 = seg_lo <= 0 ? qn[0] : 0;
  const int n1 = seg_lo <= 1 && seg_hi >= 1 ? qn[1] : 0;
  const int n2 = seg_lo <= 2 && seg_hi >= 2 ? qn[2] : 0;
  const int n3 = seg_hi >= 3 ? qn[3] : 0;
  const int total = n0 + n1 + n2 + n3;
  if (blockIdx.x == 0 && threadIdx.x == 0) cnt[WF_C + cur] = 0;  // filled again by the next extend stage
  Scene sc(uniforms_of(B.slot));
  sc.INIT();
  const int stride = gridDim.x * blockDim.x;
  for (int base = blockIdx.x * blockDim.x; base < total; base += stride) {
    const int w = base + threadIdx.x;
    int path = 0;
    bool push_active = false, push_direct = false, push_sss = false, push_vol = false, finished = false;
    int push_shadow = 0;  // bit 0: sky, bit 1: sun
    if (w < total) {
      const int seg = w < n0 ? 0 : (w < n0 + n1 ? 1 : (w < n0 + n1 + n2 ? 2 : 3));
      const int off = w - (seg == 0 ? 0 : (seg == 1 ? n0 : (seg == 2 ? n0 + n1 : n0 + n1 + n2)));
      path = pp(B.qshade, cur)[seg * B.paths + off];
      shade_path<MAT>(J, gparams, B, sc, path, nxt, push_active, push_shadow, push_direct, push_sss, push_vol,
                      finished);
    }
    shade_push(B, cnt, nxt, path, push_active, push_shadow, push_direct, push_sss, finished, push_vol);
  }
}

}  // namespace sdev

// Shade every path the extend stage of iteration `it` queued (all four segments in one launch).
extern "C" __global__ void __launch_bounds__(SNELLY_BLOCK, SNELLY_SHADE_MIN_BLOCKS) snelly_wf_shade(
    const JobRec* __restrict__ jobs, const SnellyParams* __restrict__ gparams, WfBuffers B, int it) {
  sdev::shade_segments<sdev::MAT_INVAL>(jobs, gparams, B, it, 0, 3);
}

// The same stage as one launch per queue segment, each compiled for its material only (fewer
// registers and no material dispatch): misses and finishing paths, surface, metal, dielectric.
// The host runs them back to back in place of snelly_wf_shade when the autotuner prefers it.
#ifndef SNELLY_SHADE_SEG_MIN_BLOCKS
#define SNELLY_SHADE_SEG_MIN_BLOCKS 5
#endif
extern "C" __global__ void __launch_bounds__(SNELLY_BLOCK, SNELLY_SHADE_SEG_MIN_BLOCKS) snelly_wf_shade_miss(
    const JobRec* __restrict__ jobs, const SnellyParams* __restrict__ gparams, WfBuffers B, int it) {
  sdev::shade_segments<sdev::MAT_INVAL>(jobs, gparams, B, it, 0, 0);
}
#ifdef HAS_SURFACE
extern "C" __global__ void __launch_bounds__(SNELLY_BLOCK, SNELLY_SHADE_SEG_MIN_BLOCKS) snelly_wf_shade_surface(
    const JobRec* __restrict__ jobs, const SnellyParams* __restrict__ gparams, WfBuffers B, int it) {
  sdev::shade_segments<sdev::MAT_SURFA>(jobs, gparams, B, it, 1, 1);
}
#endif
#ifdef HAS_METAL
extern "C" __global__ void __launch_bounds__(SNELLY_BLOCK, SNELLY_SHADE_SEG_MIN_BLOCKS) snelly_wf_shade_metal(
    const JobRec* __restrict__ jobs, const SnellyParams* __restrict__ gparams, WfBuffers B, int it) {
  sdev::shade_segments<sdev::MAT_METAL>(jobs, gparams, B, it, 2, 2);
}
#endif
#ifdef HAS_DIELECTRIC
extern "C" __global__ void __launch_bounds__(SNELLY_BLOCK, SNELLY_SHADE_SEG_MIN_BLOCKS) snelly_wf_shade_dielectric(
    const JobRec* __restrict__ jobs, const SnellyParams* __restrict__ gparams, WfBuffers B, int it) {
  sdev::shade_segments<sdev::MAT_DIELE>(jobs, gparams, B, it, 3, 3);
}
#endif

#ifdef HAS_SURFACE
// The subsurface-walk stage of iteration `it` (PT:1464-1593, 1866-1918): the surface vertices the
// shade stage handed over walk inside SDF_SURFACE to an exit point, take its direct light and
// continue from there. One thread per path over the walk queue, so a warp holds only walking
// paths; the walk's own marches and the exit's shadow rays are traced inline.
extern "C" __global__ void __launch_bounds__(SNELLY_BLOCK, SNELLY_SHADE_MIN_BLOCKS) snelly_wf_sss(
    const JobRec* __restrict__ jobs, const SnellyParams* __restrict__ gparams, WfBuffers B, int it) {
  using namespace sdev;
  wf_kernel_entry();
  const JobRec& J = jobs[0];
  const SnellyParams& P = c_params[B.slot];
  int* cnt = B.cnt;
  const int nxt = (it & 1) ^ 1;
  const int total = cnt[WF_SSS];
  Scene sc(uniforms_of(B.slot));
  sc.INIT();
  const int stride = gridDim.x * blockDim.x;
  for (int base = blockIdx.x * blockDim.x; base < total; base += stride) {
    const int w = base + threadIdx.x;
    int path = 0;
    bool push_active = false, finished = false;
    if (w < total) {
      path = B.qsss[w];
      float4* r = rec_of(B.rec, path);
      WfState st;
      load_state(r, st);
      Ctx c{P, gparams, sc, B.slot, 0.0f, vec3(0.0f), make_frame(v3(P.sunDir))};
      const vec3 xyzw = wavelength_at(c, st.w);
      const SssEntry e = load_sss(r);
      int rv = sss_step(c, st.s, e, st.g);
      ++st.vertex;
      finished = rv == VERTEX_DONE || st.vertex > max_bounces(P) || maxc(st.s.thr) < kThroughputEps;
      if (finished) {
        if (finish_sample(c, J, B, path, st, xyzw)) {
          finished = false;
          push_active = true;
        }
      } else {
        st.s.inDiele ? (st.flags |= WF_INDIELE) : (st.flags &= ~WF_INDIELE);
        store_state(r, st);
        B.pend[path] = 1;
        push_active = true;
      }
    }
    shade_push(B, cnt, nxt, path, push_active, 0, false, false, finished);
  }
}
#endif

#ifdef HAS_HETERO_VOLUME
// The volume stage of iteration `it`: the vertices the shade stage stopped at a collision in the
// heterogeneous medium scatter there (hv_scatter: the single-scattering albedo, next-event
// estimates of sky, sun and sphere light through the phase function, with their shadow rays
// traced inline through the SDFs and ratio-tracked through the medium, then a new direction from
// the phase function). One thread per path over the volume queue, so a warp holds only medium
// vertices and their shadow marches; the rest of the vertex (the bounce count, the throughput
// cut, the pixel's next sample) is the shade stage's, in the same order.
extern "C" __global__ void __launch_bounds__(SNELLY_BLOCK, SNELLY_SHADE_MIN_BLOCKS) snelly_wf_volume(
    const JobRec* __restrict__ jobs, const SnellyParams* __restrict__ gparams, WfBuffers B, int it) {
  using namespace sdev;
  wf_kernel_entry();
  const JobRec& J = jobs[0];
  const SnellyParams& P = c_params[B.slot];
  int* cnt = B.cnt;
  const int nxt = (it & 1) ^ 1;
  const int total = cnt[WF_VOL];
  Scene sc(uniforms_of(B.slot));
  sc.INIT();
  const int stride = gridDim.x * blockDim.x;
  for (int base = blockIdx.x * blockDim.x; base < total; base += stride) {
    const int w = base + threadIdx.x;
    int path = 0;
    bool push_active = false, finished = false;
    if (w < total) {
      path = B.qvol[w];
      float4* r = rec_of(B.rec, path);
      WfState st;
      load_state(r, st);
      Ctx c{P, gparams, sc, B.slot, 0.0f, vec3(0.0f), make_frame(v3(P.sunDir))};
      const vec3 xyzw = wavelength_at(c, st.w);
      const vec3 ps = ld3(r[R_HIT]);
      int rv = hv_scatter(c, st.s, ps, st.g);
      ++st.vertex;
      finished = rv == VERTEX_DONE || st.vertex > max_bounces(P) || maxc(st.s.thr) < kThroughputEps;
      st.s.inDiele ? (st.flags |= WF_INDIELE) : (st.flags &= ~WF_INDIELE);
      if (finished) {
        if (finish_sample(c, J, B, path, st, xyzw)) {
          finished = false;
          push_active = true;
        }
      } else {
        store_state(r, st);
        B.pend[path] = 1;
        push_active = true;
      }
    }
    shade_push(B, cnt, nxt, path, push_active, 0, false, false, finished);
  }
}
#endif

#ifdef HAS_SURFACE
// ---- persistent subsurface walker (the alternative to snelly_wf_sss) ------------------------------
// After a walk the record holds, in place of the entry's bitangent, the exit point and the walk's
// outcome (R_S2: xyz, w = WALK_EXIT or WALK_END as int bits), and the walk's throughput in place of
// the subsurface albedo (R_S1.w in dispersive mode, R_S4 in RGB mode).
//
// Each lane runs one walk a step at a time (sss_walk_step: one march, the roulette, one phase
// sample) and, when it ends, takes the next walk of the iteration's walk queue: a warp claims
// `grab` queue entries per atomic and refills once `refill` lanes are idle, so it stays full
// however uneven the walks' lengths are. Every path draws its random numbers in the same order as
// sss_step, so images are the same as with snelly_wf_sss. A finished walk goes to the exit queue.
extern "C" __global__ void __launch_bounds__(SNELLY_BLOCK) snelly_wf_walk(const JobRec* __restrict__ jobs,
                                                                       const SnellyParams* __restrict__ gparams,
                                                                       WfBuffers B, int it, int grab, int refill) {
  using namespace sdev;
  wf_kernel_entry();
  (void)jobs;
  (void)it;
  const SnellyParams& P = c_params[B.slot];
  Scene sc(uniforms_of(B.slot));
  sc.INIT();
  const Ctx c{P, gparams, sc, B.slot, 0.0f, vec3(0.0f), Frame()};
  int* cnt = B.cnt;
  const int total = cnt[WF_SSS];
  bool has = false;
  int path = 0;
  WalkState w;
  w.pw = vec3(0.0f);
  w.dw = vec3(0.0f);
  w.thr = Rad(0.0f);
  w.n = 0;
  Rng g;
  g.s[0] = g.s[1] = g.s[2] = g.s[3] = 1u;
  Rad ssAlb = Rad(0.0f);
  int wbase = 0, wlim = 0;  // the warp's claimed range of queue entries (warp-uniform)
  bool wdone = false;
  for (;;) {
    const bool want = !has;
    const unsigned need = __ballot_sync(WF_FULL, want);
    const unsigned busy = __ballot_sync(WF_FULL, has);
    if (!wdone && need && (__popc(need) >= refill || !busy)) {
      if (wbase >= wlim) {
        int nb = 0;
        if ((threadIdx.x & 31) == 0) nb = atomicAdd(cnt + WF_WHEAD, grab);
        nb = __shfl_sync(WF_FULL, nb, 0);
        wbase = nb;
        wlim = min(nb + grab, total);
        wdone = nb >= total;
      }
      const int q = wbase + __popc(need & lanemask_lt());
      wbase = min(wbase + __popc(need), wlim);
      if (want && q < wlim) {  // start this lane's next walk (PT:1466-1470)
        path = B.qsss[q];
        const float4* r = rec_of(B.rec, path);
        const uint4 rq = *reinterpret_cast<const uint4*>(r + R_RNG);
        g.s[0] = rq.x; g.s[1] = rq.y; g.s[2] = rq.z; g.s[3] = rq.w;
        const SssEntry e = load_sss(r);
        ssAlb = e.ssAlb;
        sss_walk_begin(c, ld3(r[R_POS]), sss_walk_frame(e), g, w);
        has = true;
      }
    }
    int res = WALK_ON;
    vec3 pExit(0.0f);
    if (has) res = sss_walk_step(c, g, ssAlb, w, pExit);
    const bool ended = has && res != WALK_ON;
    if (ended) {
      float4* r = rec_of(B.rec, path);
      *reinterpret_cast<uint4*>(r + R_RNG) = make_uint4(g.s[0], g.s[1], g.s[2], g.s[3]);
      r[R_S2] = st3(pExit, __int_as_float(res));
#ifdef DISPERSION_ENABLED
      r[R_S1].w = w.thr;
#else
      r[R_S4] = st3(w.thr);
#endif
    }
    const int slot = warp_append(cnt + WF_XQ, ended);
    if (slot >= 0) B.qexit[slot] = path;
    if (ended) has = false;
    if (wdone && !__any_sync(WF_FULL, has)) break;
  }
}

// The vertices whose walk the persistent walker finished: the exit's normal, direct light and
// continuation (sss_exit), or the end of the path when the walk stopped inside.
extern "C" __global__ void __launch_bounds__(SNELLY_BLOCK, SNELLY_SHADE_MIN_BLOCKS) snelly_wf_walk_exit(
    const JobRec* __restrict__ jobs, const SnellyParams* __restrict__ gparams, WfBuffers B, int it) {
  using namespace sdev;
  wf_kernel_entry();
  const JobRec& J = jobs[0];
  const SnellyParams& P = c_params[B.slot];
  int* cnt = B.cnt;
  const int nxt = (it & 1) ^ 1;
  const int total = cnt[WF_XQ];
  Scene sc(uniforms_of(B.slot));
  sc.INIT();
  const int stride = gridDim.x * blockDim.x;
  for (int base = blockIdx.x * blockDim.x; base < total; base += stride) {
    const int q = base + threadIdx.x;
    int path = 0;
    bool push_active = false, finished = false;
    if (q < total) {
      path = B.qexit[q];
      float4* r = rec_of(B.rec, path);
      WfState st;
      load_state(r, st);
      Ctx c{P, gparams, sc, B.slot, 0.0f, vec3(0.0f), make_frame(v3(P.sunDir))};
      const vec3 xyzw = wavelength_at(c, st.w);
      const float4 ex = r[R_S2];
      const float probSSS = r[R_S0].w;
#ifdef DISPERSION_ENABLED
      const Rad wthr = r[R_S1].w;
#else
      const Rad wthr = ld3(r[R_S4]);
#endif
      const int rv = __float_as_int(ex.w) == WALK_EXIT ? sss_exit(c, st.s, probSSS, wthr, ld3(ex), st.g) : VERTEX_DONE;
      ++st.vertex;
      finished = rv == VERTEX_DONE || st.vertex > max_bounces(P) || maxc(st.s.thr) < kThroughputEps;
      if (finished) {
        if (finish_sample(c, J, B, path, st, xyzw)) {
          finished = false;
          push_active = true;
        }
      } else {
        st.s.inDiele ? (st.flags |= WF_INDIELE) : (st.flags &= ~WF_INDIELE);
        store_state(r, st);
        B.pend[path] = 1;
        push_active = true;
      }
    }
    shade_push(B, cnt, nxt, path, push_active, 0, false, false, finished);
  }
}
#endif
