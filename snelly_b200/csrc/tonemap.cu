// tonemap.cu - the reference's display transform, shaders/tonemapper-fragment-shader.glsl (cited
// TM:line), as a scene-independent kernel over a job's resolved mean image: XYZ -> linear RGB,
// gamut shift, gamma, exposure, L/(1+L) per channel, saturation, contrast, optional hue shift.
// Compiled ahead of time without fast-math or contraction, so every operation is the IEEE
// float operation the shader names, in the shader's order.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "glslcompat.h"
#include "runtime_internal.h"
#include "snelly.h"

namespace {

using glsl::vec3;
using glsl::vec4;

__device__ float tone_curve(float L) { return L / (1.0f + L); }  // TM:14-17

// TM:19-27
__device__ vec3 rgb2hsv(vec3 c) {
  vec4 K = vec4(0.0f, -1.0f / 3.0f, 2.0f / 3.0f, -1.0f);
  vec4 p = glsl::mix(vec4(c.b, c.g, K.w, K.z), vec4(c.g, c.b, K.x, K.y), glsl::step(c.b, c.g));
  vec4 q = glsl::mix(vec4(p.x, p.y, p.w, c.r), vec4(c.r, p.y, p.z, p.x), glsl::step(p.x, c.r));
  float d = q.x - fminf(q.w, q.y);
  float e = 1.0e-10f;
  return vec3(fabsf(q.z + (q.w - q.y) / (6.0f * d + e)), d / (q.x + e), q.x);
}

// TM:29-34
__device__ vec3 hsv2rgb(vec3 c) {
  vec4 K = vec4(1.0f, 2.0f / 3.0f, 1.0f / 3.0f, 3.0f);
  vec3 p = glsl::abs(glsl::fract(vec3(c.x) + vec3(K.x, K.y, K.z)) * 6.0f - vec3(K.w));
  return c.z * glsl::mix(vec3(K.x), glsl::clamp(p - vec3(K.x), 0.0f, 1.0f), c.y);
}

// sign(d) * pow(|d|, e) of TM:74-84
__device__ float signed_pow(float d, float e) { return glsl::sign(d) * powf(fabsf(d), e); }

// TM:36-97 for one pixel's mean XYZ.
__device__ vec4 tonemap_pixel(float X, float Y, float Z, const snelly_tonemap_params& t) {
  vec3 RGB;
  RGB.r = 3.2406f * X - 1.5372f * Y - 0.4986f * Z;
  RGB.g = -0.9689f * X + 1.8758f * Y + 0.0415f * Z;
  RGB.b = 0.0557f * X - 0.2040f * Y + 1.0570f * Z;
  float delta = -fminf(0.0f, fminf(fminf(RGB.r, RGB.g), RGB.b));
  RGB.r += delta;
  RGB.g += delta;
  RGB.b += delta;
  RGB = vec3(powf(RGB.r, t.invGamma), powf(RGB.g, t.invGamma), powf(RGB.b, t.invGamma));
  RGB *= powf(2.0f, t.exposure);
  float R = tone_curve(RGB.r), G = tone_curve(RGB.g), B = tone_curve(RGB.b);
  float mean = (R + G + B) / 3.0f;
  float dR = R - mean, dG = G - mean, dB = B - mean;
  R = mean + signed_pow(dR, 1.0f / t.saturation);
  G = mean + signed_pow(dG, 1.0f / t.saturation);
  B = mean + signed_pow(dB, 1.0f / t.saturation);
  dR = R - 0.5f;
  dG = G - 0.5f;
  dB = B - 0.5f;
  R = 0.5f + signed_pow(dR, 1.0f / t.contrast);
  G = 0.5f + signed_pow(dG, 1.0f / t.contrast);
  B = 0.5f + signed_pow(dB, 1.0f / t.contrast);
  vec3 C = vec3(R, G, B);
  if (t.hueShift > 0.0f) {
    vec3 hsv = rgb2hsv(C);
    hsv.r = glsl::mod(hsv.r + t.hueShift, 1.0f);
    C = hsv2rgb(hsv);
  }
  return vec4(C.r, C.g, C.b, 1.0f);
}

// One thread per pixel of the mean image `in` (X, Y, Z, N). RGBA8 output follows the GL ES
// conversion of a colour-buffer write to an 8-bit unsigned normalised channel: clamp to [0, 1],
// scale by 255, round to nearest.
__global__ void __launch_bounds__(256) tonemap_kernel(const float4* __restrict__ in, long long n,
                                                      snelly_tonemap_params t, int fmt, void* __restrict__ out) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 m = in[i];
  vec4 c = tonemap_pixel(m.x, m.y, m.z, t);
  if (fmt == SNELLY_TONEMAP_RGBA32F) {
    reinterpret_cast<float4*>(out)[i] = make_float4(c.x, c.y, c.z, c.w);
  } else {
    auto q = [](float v) { return (unsigned)(fminf(fmaxf(v, 0.0f), 1.0f) * 255.0f + 0.5f); };
    reinterpret_cast<uchar4*>(out)[i] = make_uchar4(q(c.x), q(c.y), q(c.z), q(c.w));
  }
}

}  // namespace

extern "C" int snelly_tonemap(snelly_ctx* ctx, uint64_t job_id, const snelly_tonemap_params* params, void* out,
                              size_t bytes, int format) {
  if (!ctx || !params || !out) return snelly::fail(SNELLY_EINVAL, "null argument to snelly_tonemap");
  if (format != SNELLY_TONEMAP_RGBA8 && format != SNELLY_TONEMAP_RGBA32F)
    return snelly::fail(SNELLY_EINVAL, "bad tonemap format");
  if (!(params->saturation != 0.0f && params->contrast != 0.0f))
    return snelly::fail(SNELLY_EINVAL, "saturation and contrast must be non-zero");
  snelly::Context& c = *ctx->c;
  std::lock_guard<std::mutex> lk(c.mu);
  auto it = c.jobs.find(job_id);
  if (it == c.jobs.end()) return snelly::fail(SNELLY_ENOTFOUND, "unknown job id");
  snelly::Job& j = it->second;
  if (j.cancelled) return snelly::fail(SNELLY_ECANCELLED, "job was cancelled");
  int rc = snelly::wait_job(c, j, SNELLY_READ_WAIT);
  if (rc) return rc;
  const long long npix = (long long)j.desc.width * j.desc.height;
  const size_t need = (size_t)npix * (format == SNELLY_TONEMAP_RGBA8 ? 4 : 16);
  if (bytes < need) return snelly::fail(SNELLY_EINVAL, "output buffer too small: need " + std::to_string(need) + " bytes");
  if (j.display.bytes < need) {
    c.release(j.display);
    rc = c.alloc(j.display, need);
    if (rc) return rc;
  }
  // the job's stream order puts this after its enqueued frames and their resolve
  const int blocks = (int)((npix + 255) / 256);
  tonemap_kernel<<<blocks, 256, 0, c.stream>>>((const float4*)j.out.ptr, npix, *params, format, j.display.ptr);
  c.launches += 1;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, j.display.ptr, need, cudaMemcpyDeviceToHost, c.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
  if (e != cudaSuccess) return snelly::fail(SNELLY_EDEVICE, std::string("tonemap: ") + cudaGetErrorString(e));
  return SNELLY_OK;
}
