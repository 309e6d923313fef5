// aot_kernels.cu - scene-independent kernels compiled ahead of time for sm_100a into libsnelly:
// the FP32 peak microbenchmark used as the roofline denominator, and an L2 flush for timing.
#include <cuda_runtime.h>

#include <string>

#include "runtime_internal.h"
#include "snelly.h"

namespace {

// Independent FMA chains per thread: 8 accumulators x `iters` x 2 flops.
__global__ void __launch_bounds__(256) ffma_peak_kernel(float* out, int iters, float a, float b) {
  float x0 = threadIdx.x * 1e-7f, x1 = x0 + 1.0f, x2 = x0 + 2.0f, x3 = x0 + 3.0f;
  float x4 = x0 + 4.0f, x5 = x0 + 5.0f, x6 = x0 + 6.0f, x7 = x0 + 7.0f;
#pragma unroll 1
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
      x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
    }
  }
  float s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (s == 1234.5f) out[blockIdx.x] = s;  // keeps the chains live
}

__global__ void l2_flush_kernel(float4* buf, size_t n, float v) {
  size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) buf[i] = make_float4(v, v, v, v);
}

}  // namespace

extern "C" {

int snelly_measure_fp32_peak(snelly_ctx* ctx, double* tflops, double* ms_out) {
  if (!ctx || !tflops) return snelly::fail(SNELLY_EINVAL, "null argument");
  snelly::Context& c = *ctx->c;
  float* out = nullptr;
  if (cudaMalloc(&out, 4 << 20) != cudaSuccess) return snelly::fail(SNELLY_EDEVICE, "cudaMalloc failed");
  const int blocks = c.sm_count * 8, threads = 256, iters = 4096;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int w = 0; w < 3; ++w) ffma_peak_kernel<<<blocks, threads, 0, c.stream>>>(out, iters, 0.9999f, 1e-4f);
  float best = 1e30f;
  for (int r = 0; r < 5; ++r) {
    cudaEventRecord(e0, c.stream);
    ffma_peak_kernel<<<blocks, threads, 0, c.stream>>>(out, iters, 0.9999f, 1e-4f);
    cudaEventRecord(e1, c.stream);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess) return snelly::fail(SNELLY_EDEVICE, cudaGetErrorString(err));
  double flops = 2.0 * 8.0 * 16.0 * iters * (double)blocks * threads;
  *tflops = flops / (best * 1e-3) / 1e12;
  if (ms_out) *ms_out = best;
  c.launches += 8;
  return SNELLY_OK;
}

int snelly_flush_l2(snelly_ctx* ctx, size_t bytes) {
  if (!ctx) return snelly::fail(SNELLY_EINVAL, "null argument");
  snelly::Context& c = *ctx->c;
  static thread_local void* buf = nullptr;
  static thread_local size_t have = 0;
  if (have < bytes) {
    if (buf) cudaFree(buf);
    buf = nullptr;
    if (cudaMalloc(&buf, bytes) != cudaSuccess) return snelly::fail(SNELLY_EDEVICE, "cudaMalloc failed");
    have = bytes;
  }
  l2_flush_kernel<<<c.sm_count * 4, 256, 0, c.stream>>>((float4*)buf, bytes / 16, 0.0f);
  c.launches += 1;
  if (cudaGetLastError() != cudaSuccess) return snelly::fail(SNELLY_EDEVICE, "flush launch failed");
  return SNELLY_OK;
}

}  // extern "C"
