// oracle_main.cpp - C entry points of the CPU oracle library, built once per scene by
// oracle/build.py with the scene's translated GLSL included as SCENE_INC.
//
// TEST INFRASTRUCTURE: loaded by tests/ and by the benchmark's CPU-baseline leg only.
#include <cstdint>
#include <cstring>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef ORACLE_COUNT_OPS
#include "counted.h"  // must precede glslcompat.h: it supplies gfloat
#endif
#include "glslcompat.h"
namespace glsl {
#include SCENE_INC
}
#include "pt_oracle.h"
#include "tm_oracle.h"

namespace {

// Per-pixel seeding used by the CUDA path tracer, restated: lane k of pixel i is
// 1 + (z_k mod (m_k - 1)) for successive SplitMix64 outputs z_k of the stream keyed by
// splitmix64(seed) ^ i (the reference seeds with Math.random(), js/renderer.js:696-702).
uint64_t splitmix_next(uint64_t& s) {
  s += 0x9E3779B97F4A7C15ull;
  uint64_t z = s;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Threads of one render call: `threads` if positive, else every processor. Given as the
// parallel region's num_threads clause, so that no call changes the process-wide OpenMP setting
// that other libraries in the process (the reference build, torch) read.
int team_size(int threads) {
#ifdef _OPENMP
  return threads > 0 ? threads : omp_get_num_procs();
#else
  (void)threads;
  return 1;
#endif
}

int g_last_team = 0;  // threads the last render call ran on

}  // namespace

extern "C" {

// Threads the last oracle_render / oracle_firsthit call ran on.
int oracle_last_team(void) { return g_last_team; }

void oracle_seed(uint64_t seed, uint64_t pixel, uint32_t* out4) {
  static const uint32_t m[4] = {4194287u, 4194277u, 4194191u, 4194167u};
  uint64_t s = seed;
  uint64_t key = splitmix_next(s) ^ pixel;
  for (int k = 0; k < 4; ++k) out4[k] = 1u + (uint32_t)(splitmix_next(key) % (uint64_t)(m[k] - 1u));
}

// One rand() of PT:119-130 on a 4-lane state (float arithmetic), for RNG checks.
float oracle_rand(uint32_t* st) {
  glsl::SceneUniforms U;
  std::memset((void*)&U, 0, sizeof U);
  glsl::Scene sc(U);
  SnellyParams P;
  std::memset(&P, 0, sizeof P);
  oracle::Invocation inv(P, sc);
  glsl::vec4 rnd((float)st[0], (float)st[1], (float)st[2], (float)st[3]);
  float r = glsl::s_tofloat(inv.rand(rnd));
  st[0] = (uint32_t)glsl::s_tofloat(rnd.x);
  st[1] = (uint32_t)glsl::s_tofloat(rnd.y);
  st[2] = (uint32_t)glsl::s_tofloat(rnd.z);
  st[3] = (uint32_t)glsl::s_tofloat(rnd.w);
  return r;
}

size_t oracle_uniform_block_size(void) { return sizeof(glsl::SceneUniforms); }

// Operation tallies of the calling thread (counting builds; zero otherwise).
void oracle_counts(uint64_t* flops, uint64_t* special) {
#ifdef ORACLE_COUNT_OPS
  *flops = glsl::op_counts().flops;
  *special = glsl::op_counts().special;
  glsl::op_counts() = glsl::OpCounts{0, 0};
#else
  *flops = 0;
  *special = 0;
#endif
}

// Render `frames` frames for the n pixels listed in `pixels` (indices y*width + x, row 0 at the
// bottom). rng: 4 lanes per listed pixel, in/out. xyz_sum: 3 doubles per listed pixel, the sum of
// the per-frame XYZ contributions (added to). mean: 4 floats per listed pixel (X, Y, Z, N), the
// running mean updated exactly as PT:1975-1987 (in/out; N = 0 for a fresh pixel).
int oracle_render(const SnellyParams* P, const void* uniforms, int width, int height, const int* pixels, int n,
                  int frames, uint32_t* rng, double* xyz_sum, float* mean, int threads) {
  (void)height;
  const glsl::SceneUniforms& U = *reinterpret_cast<const glsl::SceneUniforms*>(uniforms);
  const int nt = team_size(threads);
  g_last_team = 1;
#pragma omp parallel num_threads(nt)
  {
#ifdef _OPENMP
#pragma omp single nowait
    g_last_team = omp_get_num_threads();
#endif
#pragma omp for schedule(dynamic, 1)
  for (int k = 0; k < n; ++k) {
    int idx = pixels[k];
    int x = idx % width, y = idx / width;
    glsl::vec4 rnd((float)rng[4 * k + 0], (float)rng[4 * k + 1], (float)rng[4 * k + 2], (float)rng[4 * k + 3]);
    for (int f = 0; f < frames; ++f) {
      glsl::Scene sc(U);
      sc.INIT();
      oracle::Invocation inv(*P, sc);
      glsl::vec3 c = inv.pathtrace(glsl::vec2(float(x) + 0.5f, float(y) + 0.5f), rnd);
      float cx = glsl::s_tofloat(c.x), cy = glsl::s_tofloat(c.y), cz = glsl::s_tofloat(c.z);
      xyz_sum[3 * k + 0] += (double)cx;
      xyz_sum[3 * k + 1] += (double)cy;
      xyz_sum[3 * k + 2] += (double)cz;
      float oldN = mean[4 * k + 3], newN = oldN + 1.0f;
      mean[4 * k + 0] = (oldN * mean[4 * k + 0] + cx) / newN;
      mean[4 * k + 1] = (oldN * mean[4 * k + 1] + cy) / newN;
      mean[4 * k + 2] = (oldN * mean[4 * k + 2] + cz) / newN;
      mean[4 * k + 3] = newN;
    }
    rng[4 * k + 0] = (uint32_t)glsl::s_tofloat(rnd.x);
    rng[4 * k + 1] = (uint32_t)glsl::s_tofloat(rnd.y);
    rng[4 * k + 2] = (uint32_t)glsl::s_tofloat(rnd.z);
    rng[4 * k + 3] = (uint32_t)glsl::s_tofloat(rnd.w);
  }
  }  // omp parallel
  return 0;
}

// `frames` frames of the other programs for the listed pixels: mode 1 normals (NM:293-345),
// 2 ambient occlusion (AO:395-488), 4 the simplified path tracer (SP:1083-1130), all updating rng,
// xyz_sum and the running mean as oracle_render does; mode 3 pick (PK:133-152) at each pixel
// centre, writing (distance, material, 0, 0) to mean (rng and xyz_sum untouched).
int oracle_firsthit(const SnellyParams* P, const void* uniforms, int mode, int width, int height, const int* pixels,
                    int n, int frames, uint32_t* rng, double* xyz_sum, float* mean, int threads) {
  (void)height;
  if (mode < 1 || mode > 4) return -1;
  const glsl::SceneUniforms& U = *reinterpret_cast<const glsl::SceneUniforms*>(uniforms);
  const int nt = team_size(threads);
  g_last_team = 1;
#pragma omp parallel num_threads(nt)
  {
#ifdef _OPENMP
#pragma omp single nowait
    g_last_team = omp_get_num_threads();
#endif
#pragma omp for schedule(dynamic, 1)
  for (int k = 0; k < n; ++k) {
    int idx = pixels[k];
    int x = idx % width, y = idx / width;
    glsl::vec2 pixel(float(x) + 0.5f, float(y) + 0.5f);
    if (mode == 3) {
      glsl::Scene sc(U);
      sc.INIT();
      oracle::Invocation inv(*P, sc);
      glsl::vec2 r = inv.pick(pixel);
      mean[4 * k + 0] = glsl::s_tofloat(r.x);
      mean[4 * k + 1] = glsl::s_tofloat(r.y);
      mean[4 * k + 2] = 0.0f;
      mean[4 * k + 3] = 0.0f;
      continue;
    }
    glsl::vec4 rnd((float)rng[4 * k + 0], (float)rng[4 * k + 1], (float)rng[4 * k + 2], (float)rng[4 * k + 3]);
    for (int f = 0; f < frames; ++f) {
      glsl::Scene sc(U);
      oracle::Invocation inv(*P, sc);
      glsl::vec3 c;
      bool skipped = false;
      if (mode == 1) {
        sc.INIT();
        c = inv.normals(pixel, rnd);
      } else if (mode == 4) {
        sc.INIT();
        c = inv.ptsimple(pixel, rnd);
      } else {
        // AO:397-414: the interactive-mode skip comes before INIT()
        c = inv.ao_frame(pixel, rnd, skipped);
      }
      if (skipped) continue;
      float cx = glsl::s_tofloat(c.x), cy = glsl::s_tofloat(c.y), cz = glsl::s_tofloat(c.z);
      xyz_sum[3 * k + 0] += (double)cx;
      xyz_sum[3 * k + 1] += (double)cy;
      xyz_sum[3 * k + 2] += (double)cz;
      float oldN = mean[4 * k + 3], newN = oldN + 1.0f;
      mean[4 * k + 0] = (oldN * mean[4 * k + 0] + cx) / newN;
      mean[4 * k + 1] = (oldN * mean[4 * k + 1] + cy) / newN;
      mean[4 * k + 2] = (oldN * mean[4 * k + 2] + cz) / newN;
      mean[4 * k + 3] = newN;
    }
    rng[4 * k + 0] = (uint32_t)glsl::s_tofloat(rnd.x);
    rng[4 * k + 1] = (uint32_t)glsl::s_tofloat(rnd.y);
    rng[4 * k + 2] = (uint32_t)glsl::s_tofloat(rnd.z);
    rng[4 * k + 3] = (uint32_t)glsl::s_tofloat(rnd.w);
  }
  }  // omp parallel
  return 0;
}

// The display transform (TM:36-97) of n mean XYZ pixels (4 floats each, N ignored) with the
// shader's uniforms p = {exposure, invGamma, contrast, saturation, hueShift}; out: RGBA floats.
int oracle_tonemap(const float* in4, int n, const float* p, float* out4) {
  oracle::ToneMapper tm{p[0], p[1], p[2], p[3], p[4]};
  for (int k = 0; k < n; ++k) {
    glsl::vec4 c = tm.apply(glsl::vec3(in4[4 * k + 0], in4[4 * k + 1], in4[4 * k + 2]));
    for (int i = 0; i < 4; ++i) out4[4 * k + i] = glsl::s_tofloat(c[i]);
  }
  return 0;
}

}  // extern "C"
