// ref_harness.cpp - runs one of the reference's own fragment shaders (translated to C++ by
// oracle/build_ref.py into ref_shader.inc) once per pixel and frame on the CPU: the path tracer,
// normals and ambient-occlusion programs through ref_render, the pick program through ref_pick.
//
// TEST INFRASTRUCTURE: part of the oracle/_ref build recipe.
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "glslcompat.h"
namespace glsl {
#include "ref_shader.inc"
}

extern "C" size_t ref_block_size(void) { return sizeof(glsl::RefShaderUniforms); }

namespace {
// Threads of one call: `threads` if positive, else every processor, given as the parallel
// region's num_threads clause so that no call changes the process-wide OpenMP setting.
int team_size(int threads) {
#ifdef _OPENMP
  return threads > 0 ? threads : omp_get_num_procs();
#else
  (void)threads;
  return 1;
#endif
}
int g_last_team = 0;
}  // namespace

// Threads the last ref_render / ref_pick call ran on.
extern "C" int ref_last_team(void) { return g_last_team; }

#ifdef REF_TONEMAP
// The tonemapper program (built with -DREF_TONEMAP): the Radiance texture bound to each input
// texel in turn (1x1 NEAREST); out: g_outputColor per texel.
extern "C" int ref_tonemap(const void* block, size_t block_bytes, size_t off_radiance, const float* in4, int n,
                           float* out4) {
  if (block_bytes != sizeof(glsl::RefShaderUniforms)) return -1;
  std::vector<unsigned char> local(block_bytes + 16);
  unsigned char* lb = local.data();
  float rad[4];
  glsl::sampler2D radS{rad, 1, 1, 4, 0, 0, 0};
  std::memcpy(lb, block, block_bytes);
  std::memcpy(lb + off_radiance, &radS, sizeof radS);
  for (int k = 0; k < n; ++k) {
    for (int c = 0; c < 4; ++c) rad[c] = in4[4 * k + c];
    glsl::RefShader sh(*reinterpret_cast<const glsl::RefShaderUniforms*>(lb));
    sh.vTexCoord = glsl::vec2(0.5f, 0.5f);
    sh.main();
    for (int c = 0; c < 4; ++c) out4[4 * k + c] = sh.g_outputColor[c];
  }
  return 0;
}
#elif defined(REF_PICK)
// The pick program (built with -DREF_PICK): one invocation per listed pixel with mousePick at the
// pixel centre; out: gbuf_pick (distance, material, 0, 0) per pixel.
extern "C" int ref_pick(const void* block, size_t block_bytes, size_t off_mouse, int width, const int* pixels, int n,
                        float* out, int threads) {
  if (block_bytes != sizeof(glsl::RefShaderUniforms)) return -1;
  const int nt = team_size(threads);
  g_last_team = 1;
#pragma omp parallel num_threads(nt)
  {
#ifdef _OPENMP
#pragma omp single nowait
    g_last_team = omp_get_num_threads();
#endif
    std::vector<unsigned char> local(block_bytes + 16);
    unsigned char* lb = local.data();
#pragma omp for schedule(dynamic, 1)
    for (int k = 0; k < n; ++k) {
      std::memcpy(lb, block, block_bytes);
      int idx = pixels[k], x = idx % width, y = idx / width;
      float mp[2] = {float(x) + 0.5f, float(y) + 0.5f};
      std::memcpy(lb + off_mouse, mp, sizeof mp);
      glsl::RefShader sh(*reinterpret_cast<const glsl::RefShaderUniforms*>(lb));
      sh.gl_FragCoord = glsl::vec4(0.5f, 0.5f, 0.5f, 1.0f);
      sh.main();
      for (int c = 0; c < 4; ++c) out[4 * k + c] = sh.gbuf_pick[c];
    }
  }
  return 0;
}
#else

// block: the uniform block (samplers included); off_radiance / off_rng: offsets of the Radiance
// and RngData sampler records, re-pointed for each pixel at a 1x1 NEAREST texture holding that
// pixel's state. rng: 4 lanes per listed pixel (in/out); mean: (X, Y, Z, N) per pixel, the
// shader's own running mean (in/out, N = 0 for a fresh pixel).
extern "C" int ref_render(const void* block, size_t block_bytes, size_t off_radiance, size_t off_rng, int width,
                          int height, const int* pixels, int n, int frames, uint32_t* rng, float* mean, int threads) {
  (void)height;
  if (block_bytes != sizeof(glsl::RefShaderUniforms)) return -1;
  const int nt = team_size(threads);
  g_last_team = 1;
#pragma omp parallel num_threads(nt)
  {
#ifdef _OPENMP
#pragma omp single nowait
    g_last_team = omp_get_num_threads();
#endif
    std::vector<unsigned char> local(block_bytes + 16);
    unsigned char* lb = local.data();
    float rad[4], st[4];
    glsl::sampler2D radS{rad, 1, 1, 4, 0, 0, 0}, rngS{st, 1, 1, 4, 0, 0, 0};
#pragma omp for schedule(dynamic, 1)
    for (int k = 0; k < n; ++k) {
      std::memcpy(lb, block, block_bytes);
      std::memcpy(lb + off_radiance, &radS, sizeof radS);
      std::memcpy(lb + off_rng, &rngS, sizeof rngS);
      int idx = pixels[k], x = idx % width, y = idx / width;
      for (int c = 0; c < 4; ++c) {
        rad[c] = mean[4 * k + c];
        st[c] = (float)rng[4 * k + c];
      }
      for (int f = 0; f < frames; ++f) {
        glsl::RefShader sh(*reinterpret_cast<const glsl::RefShaderUniforms*>(lb));
        sh.gl_FragCoord = glsl::vec4(float(x) + 0.5f, float(y) + 0.5f, 0.5f, 1.0f);
        sh.vTexCoord = glsl::vec2(0.5f, 0.5f);
        sh.main();
        for (int c = 0; c < 4; ++c) {
          rad[c] = sh.gbuf_rad[c];
          st[c] = sh.gbuf_rng[c];
        }
      }
      for (int c = 0; c < 4; ++c) {
        mean[4 * k + c] = rad[c];
        rng[4 * k + c] = (uint32_t)st[c];
      }
    }
  }
  return 0;
}
#endif  // REF_PICK
