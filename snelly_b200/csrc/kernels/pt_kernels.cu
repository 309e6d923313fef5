// pt_kernels.cu - kernel entry points of the spectral path tracer, compiled per scene by NVRTC.
//
// Per-pixel state lives in HBM as structure-of-arrays buffers owned by the runtime:
//   rng   uint4  per pixel: the four LCG lanes (PT:119-130), persistent across frames;
//   acc   float4 per pixel: Kahan running sum of XYZ, and the frame count in .w;
//   comp  float4 per pixel: Kahan compensation terms;
//   acc64 double4 per pixel (optional): the same sums in FP64, for the accumulation study.
// Pixel index i = y * width + x with y = 0 the bottom row (gl_FragCoord convention).
//
// A launch serves a batch of jobs that share this scene module; `JobRec` describes each job's
// buffers and the range of its pixels the launch covers, and jobs start on block boundaries so
// that every warp works on one job.
#pragma once
#include "pt_integrator.cuh"
#include "pt_launch.h"

namespace sdev {

// ---- per-pixel RNG seeding ---------------------------------------------------------------------
// The reference seeds each lane with Math.random()*4194167 (js/renderer.js:696-702), which is
// neither reproducible nor integer. Here lane k of pixel i gets 1 + (z_k mod (m_k - 1)), where
// z_0.. are successive SplitMix64 outputs of a stream keyed by splitmix64(seed) ^ i. The oracle
// implements the same function.
SD_FN unsigned long long splitmix64_next(unsigned long long& s) {
  s += 0x9E3779B97F4A7C15ull;
  unsigned long long z = s;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
SD_FN uint4 seed_pixel(unsigned long long seed, unsigned long long pixel) {
  unsigned long long s = seed;
  unsigned long long key = splitmix64_next(s) ^ pixel;
  const unsigned m[4] = {4194287u, 4194277u, 4194191u, 4194167u};
  unsigned v[4];
  for (int k = 0; k < 4; ++k) v[k] = 1u + unsigned(splitmix64_next(key) % (unsigned long long)(m[k] - 1u));
  return make_uint4(v[0], v[1], v[2], v[3]);
}

SD_FN int job_of_block(const int* __restrict__ block_start, int njobs, int b) {
  int j = 0;
  while (j + 1 < njobs && __ldg(block_start + j + 1) <= b) ++j;
  return j;
}

SD_FN void kahan_add(float4& s, float4& c, const vec3& v) {
  float y, t;
  y = v.x - c.x; t = s.x + y; c.x = (t - s.x) - y; s.x = t;
  y = v.y - c.y; t = s.y + y; c.y = (t - s.y) - y; s.y = t;
  y = v.z - c.z; t = s.z + y; c.z = (t - s.z) - y; s.z = t;
  s.w += 1.0f;
}

}  // namespace sdev

extern "C" __global__ void __launch_bounds__(SNELLY_BLOCK) snelly_seed(const JobRec* __restrict__ jobs, const int* __restrict__ block_start,
                                                                    int njobs) {
  int j = sdev::job_of_block(block_start, njobs, blockIdx.x);
  const JobRec& J = jobs[j];
  long long i = (long long)(blockIdx.x - block_start[j]) * blockDim.x + threadIdx.x + J.pixel_begin;
  if (i >= (long long)J.pixel_begin + J.pixel_count) return;
  J.rng[i] = sdev::seed_pixel(J.seed, (unsigned long long)i);
  J.acc[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  J.comp[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (J.acc64) {
    J.acc64[4 * i + 0] = 0.0;
    J.acc64[4 * i + 1] = 0.0;
    J.acc64[4 * i + 2] = 0.0;
    J.acc64[4 * i + 3] = 0.0;
  }
}

// One frame (MAX_SAMPLES_PER_FRAME samples) for every pixel of every job in the batch: the
// path-per-thread kernel. Each thread runs the whole camera path of its pixel.
extern "C" __global__ void __launch_bounds__(SNELLY_BLOCK, SNELLY_MEGA_MIN_BLOCKS) snelly_frame_mega(const JobRec* __restrict__ jobs,
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
#ifdef INTERACTIVE_MODE
  if (rand01(g) < P.skipProbability) {
    J.rng[i] = make_uint4(g.s[0], g.s[1], g.s[2], g.s[3]);
    return;
  }
#endif
  Scene sc(uniforms_of(slot));
  sc.INIT();
  Ctx c{P, gparams + slot, sc, slot, 0.0f, vec3(0.0f), Frame()};
  const int W = J.width;
  const int x = int(i % W), y = int(i / W);
  vec3 xyz = pixel_samples(c, vec2(float(x) + 0.5f, float(y) + 0.5f), g);
  J.rng[i] = make_uint4(g.s[0], g.s[1], g.s[2], g.s[3]);
  float4 s = J.acc[i], cp = J.comp[i];
  kahan_add(s, cp, xyz);
  J.acc[i] = s;
  J.comp[i] = cp;
  if (J.acc64) {
    J.acc64[4 * i + 0] += double(xyz.x);
    J.acc64[4 * i + 1] += double(xyz.y);
    J.acc64[4 * i + 2] += double(xyz.z);
    J.acc64[4 * i + 3] += 1.0;
  }
}

#include "pt_wavefront.cuh"
#include "pt_firsthit.cuh"
#include "pt_simple.cuh"

// Mean XYZ and sample count per pixel into `out` (float4), for readback.
extern "C" __global__ void __launch_bounds__(SNELLY_BLOCK) snelly_resolve(const JobRec* __restrict__ jobs, const int* __restrict__ block_start,
                                                                       int njobs) {
  int j = sdev::job_of_block(block_start, njobs, blockIdx.x);
  const JobRec& J = jobs[j];
  long long i = (long long)(blockIdx.x - block_start[j]) * blockDim.x + threadIdx.x + J.pixel_begin;
  if (i >= (long long)J.pixel_begin + J.pixel_count) return;
  float4 s = J.acc[i];
  float n = s.w;
  float inv = n > 0.0f ? 1.0f / n : 0.0f;
  J.out[i] = make_float4(s.x * inv, s.y * inv, s.z * inv, n);
}
