// aot_kernels.cu - scene-independent kernels compiled ahead of time for sm_100a into libsnelly:
// the FP32 peak microbenchmark used as the roofline denominator, an L2 flush for timing, the image
// statistics reduction, and exhaustive self-tests of the arithmetic replacements the scene
// kernels use (this file is compiled without fast-math, so floorf and __fdiv_rn are IEEE).
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "kernels/pt_rng.cuh"
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

// Image statistics of a job's accumulators, pass 1: per-block partial sums (in double, fixed
// order) of the per-pixel mean X, Y, Z, of Y^2 and of the sample counts -> partial[block].
// The per-pixel mean is the Kahan sum minus its compensation, over the count.
constexpr int kStatsThreads = 256;
__global__ void __launch_bounds__(kStatsThreads) image_stats_partial(const float4* __restrict__ acc,
                                                                      const float4* __restrict__ comp, long long npix,
                                                                      double* __restrict__ partial) {
  __shared__ double sh[5][kStatsThreads];
  double a[5] = {0, 0, 0, 0, 0};
  for (long long i = (long long)blockIdx.x * kStatsThreads + threadIdx.x; i < npix; i += (long long)gridDim.x * kStatsThreads) {
    float4 s = acc[i], c = comp[i];
    double n = s.w;
    if (n > 0) {
      double x = ((double)s.x - c.x) / n, y = ((double)s.y - c.y) / n, z = ((double)s.z - c.z) / n;
      a[0] += x;
      a[1] += y;
      a[2] += z;
      a[3] += y * y;
    }
    a[4] += n;
  }
  for (int k = 0; k < 5; ++k) sh[k][threadIdx.x] = a[k];
  __syncthreads();
  for (int w = kStatsThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int k = 0; k < 5; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 5) partial[5 * blockIdx.x + threadIdx.x] = sh[threadIdx.x][0];
}

// Pass 2: one block folds the partials (in block order) into out[5].
__global__ void __launch_bounds__(32) image_stats_final(const double* __restrict__ partial, int nblocks,
                                                        double* __restrict__ out) {
  if (threadIdx.x < 5) {
    double t = 0;
    for (int b = 0; b < nblocks; ++b) t += partial[5 * b + threadIdx.x];
    out[threadIdx.x] = t;
  }
}

// Self-test 0: the RNG's conversion and quotient for every state x in [0, m) of each modulus,
// against float(x) and __fdiv_rn.
__global__ void selftest_rng_quotients(unsigned long long* bad) {
  const unsigned m[4] = {4194287u, 4194277u, 4194191u, 4194167u};
  const float inv[4] = {SNELLY_RNG_INV_M0, SNELLY_RNG_INV_M1, SNELLY_RNG_INV_M2, SNELLY_RNG_INV_M3};
  unsigned long long n = 0;
  const unsigned stride = gridDim.x * blockDim.x;
  for (int k = 0; k < 4; ++k) {
    const float mf = (float)m[k];
    for (unsigned x = blockIdx.x * blockDim.x + threadIdx.x; x < m[k]; x += stride) {
      float xf = sdev::small_uint_to_float(x);
      float q = sdev::quotient_small(xf, mf, inv[k]);
      n += (xf == (float)x && __float_as_uint(q) == __float_as_uint(__fdiv_rn((float)x, mf))) ? 0 : 1;
    }
  }
  if (n) atomicAdd(bad, n);
}

// ---- image statistics without allocation ------------------------------------------------------
// Scratch of snelly_image_stats_static, in file-scope device memory so that entry point allocates
// nothing: one partial record (5 doubles) per block for up to kStaticStatsMaxBlocks blocks of
// kStaticStatsPixelsPerBlock pixels, the folded result, and the completion counter of the
// last-block fold (which must start at zero). 160 KiB per device.
constexpr int kStaticStatsMaxBlocks = 4096;
constexpr int kStaticStatsPixelsPerThread = 8;
constexpr int kStaticStatsPixelsPerBlock = kStatsThreads * kStaticStatsPixelsPerThread;
constexpr long long kStaticStatsMaxPixels = (long long)kStaticStatsMaxBlocks * kStaticStatsPixelsPerBlock;
struct StaticStatsScratch {
  double partial[5 * kStaticStatsMaxBlocks];
  double result[8];
  unsigned int done_blocks;
};
static __device__ __align__(256) StaticStatsScratch g_static_stats_scratch;

// One launch: block b reduces pixels [b * 2048, (b + 1) * 2048) into partial[b] (same per-pixel
// terms as image_stats_partial), and the last block to finish folds the partials in block order
// into result and resets the counter.
__global__ void __launch_bounds__(kStatsThreads) image_stats_static(const float4* __restrict__ acc,
                                                                     const float4* __restrict__ comp, long long npix,
                                                                     StaticStatsScratch* __restrict__ scratch) {
  __shared__ double sh[5][kStatsThreads];
  __shared__ bool last;
  double a[5] = {0, 0, 0, 0, 0};
  const long long base = (long long)blockIdx.x * kStaticStatsPixelsPerBlock;
  for (int k = 0; k < kStaticStatsPixelsPerThread; ++k) {
    long long i = base + (long long)k * kStatsThreads + threadIdx.x;
    if (i >= npix) break;
    float4 s = acc[i], c = comp[i];
    double n = s.w;
    if (n > 0) {
      double x = ((double)s.x - c.x) / n, y = ((double)s.y - c.y) / n, z = ((double)s.z - c.z) / n;
      a[0] += x;
      a[1] += y;
      a[2] += z;
      a[3] += y * y;
    }
    a[4] += n;
  }
  for (int k = 0; k < 5; ++k) sh[k][threadIdx.x] = a[k];
  __syncthreads();
  for (int w = kStatsThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int k = 0; k < 5; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 5) scratch->partial[5 * blockIdx.x + threadIdx.x] = sh[threadIdx.x][0];
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&scratch->done_blocks, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x < 5) {
    double t = 0;
    for (unsigned b = 0; b < gridDim.x; ++b) t += __ldcg(&scratch->partial[5 * b + threadIdx.x]);
    scratch->result[threadIdx.x] = t;
  }
  if (threadIdx.x == 0) scratch->done_blocks = 0;
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

// Blocks of the statistics reduction: enough to fill the GPU, at most kStatsMaxBlocks.
constexpr int kStatsMaxBlocks = 1184;  // 8 blocks per SM on 148 SMs

int snelly_image_stats(snelly_ctx* ctx, uint64_t job_id, double* out5) {
  if (!ctx || !out5) return snelly::fail(SNELLY_EINVAL, "null argument to snelly_image_stats");
  snelly::Context& c = *ctx->c;
  std::lock_guard<std::mutex> lk(c.mu);
  auto it = c.jobs.find(job_id);
  if (it == c.jobs.end()) return snelly::fail(SNELLY_ENOTFOUND, "unknown job id");
  snelly::Job& j = it->second;
  long long npix = (long long)j.desc.width * j.desc.height;
  int blocks = (int)std::min<long long>(kStatsMaxBlocks, (npix + kStatsThreads - 1) / kStatsThreads);
  if (blocks < 1) blocks = 1;
  // scratch: per-block partials + the result, owned by the context
  size_t need = sizeof(double) * (5 * (size_t)kStatsMaxBlocks + 8);
  if (c.stats_scratch.bytes < need) {
    c.release(c.stats_scratch);
    int rc = c.alloc(c.stats_scratch, need);
    if (rc) return rc;
  }
  double* partial = (double*)c.stats_scratch.ptr;
  double* result = partial + 5 * kStatsMaxBlocks;
  image_stats_partial<<<blocks, kStatsThreads, 0, c.stream>>>((const float4*)j.acc.ptr, (const float4*)j.comp.ptr,
                                                               npix, partial);
  image_stats_final<<<1, 32, 0, c.stream>>>(partial, blocks, result);
  c.launches += 2;
  if (cudaMemcpyAsync(out5, result, 5 * sizeof(double), cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
      cudaStreamSynchronize(c.stream) != cudaSuccess)
    return snelly::fail(SNELLY_EDEVICE, "image statistics failed");
  return SNELLY_OK;
}

int snelly_selftest(snelly_ctx* ctx, int which, uint64_t* mismatches) {
  if (!ctx || !mismatches) return snelly::fail(SNELLY_EINVAL, "null argument to snelly_selftest");
  if (which != 0) return snelly::fail(SNELLY_EINVAL, "unknown self-test");
  snelly::Context& c = *ctx->c;
  std::lock_guard<std::mutex> lk(c.mu);
  snelly::DevBuf cnt;
  int rc = c.alloc(cnt, sizeof(unsigned long long));
  if (rc) return rc;
  unsigned long long* d = (unsigned long long*)cnt.ptr;
  unsigned long long h = 0;
  cudaError_t e = cudaMemsetAsync(d, 0, sizeof h, c.stream);
  if (e == cudaSuccess) {
    selftest_rng_quotients<<<c.sm_count * 16, 256, 0, c.stream>>>(d);
    c.launches += 1;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d, sizeof h, cudaMemcpyDeviceToHost, c.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
  c.release(cnt);
  if (e != cudaSuccess) return snelly::fail(SNELLY_EDEVICE, std::string("self-test: ") + cudaGetErrorString(e));
  *mismatches = h;
  return SNELLY_OK;
}

int snelly_image_stats_static(snelly_ctx* ctx, uint64_t job_id, double* out5) {
  if (!ctx || !out5) return snelly::fail(SNELLY_EINVAL, "null argument to snelly_image_stats_static");
  snelly::Context& c = *ctx->c;
  std::lock_guard<std::mutex> lk(c.mu);
  auto it = c.jobs.find(job_id);
  if (it == c.jobs.end()) return snelly::fail(SNELLY_ENOTFOUND, "unknown job id");
  snelly::Job& j = it->second;
  const long long npix = (long long)j.desc.width * j.desc.height;
  if (npix > kStaticStatsMaxPixels)
    return snelly::fail(SNELLY_EINVAL, "snelly_image_stats_static handles at most " + std::to_string(kStaticStatsMaxPixels) +
                                           " pixels (its fixed scratch has " + std::to_string(kStaticStatsMaxBlocks) +
                                           " partial records); this job has " + std::to_string(npix));
  // The device address of the file-scope scratch, looked up at the context's first call (with the
  // context's device current) and kept with the context: a context created after a device reset
  // looks it up again.
  if (!c.static_stats_scratch) {
    int prev = -1;
    cudaError_t e = cudaGetDevice(&prev);
    if (e == cudaSuccess && prev != c.device) e = cudaSetDevice(c.device);
    void* p = nullptr;
    if (e == cudaSuccess) e = cudaGetSymbolAddress(&p, g_static_stats_scratch);
    if (prev >= 0 && prev != c.device) cudaSetDevice(prev);
    if (e != cudaSuccess || !p)
      return snelly::fail(SNELLY_EDEVICE, std::string("cudaGetSymbolAddress of the statistics scratch: ") +
                                              cudaGetErrorString(e));
    c.static_stats_scratch = p;
  }
  StaticStatsScratch* scratch = (StaticStatsScratch*)c.static_stats_scratch;
  const int blocks = (int)std::max<long long>(1, (npix + kStaticStatsPixelsPerBlock - 1) / kStaticStatsPixelsPerBlock);
  cudaError_t e = cudaMemsetAsync(&scratch->done_blocks, 0, sizeof(unsigned int), c.stream);
  if (e == cudaSuccess) {
    image_stats_static<<<blocks, kStatsThreads, 0, c.stream>>>((const float4*)j.acc.ptr, (const float4*)j.comp.ptr,
                                                               npix, scratch);
    c.launches += 1;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(out5, scratch->result, 5 * sizeof(double), cudaMemcpyDeviceToHost, c.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
  if (e != cudaSuccess) return snelly::fail(SNELLY_EDEVICE, std::string("image statistics failed: ") + cudaGetErrorString(e));
  return SNELLY_OK;
}

int snelly_flush_l2(snelly_ctx* ctx, size_t bytes) {
  if (!ctx) return snelly::fail(SNELLY_EINVAL, "null argument");
  snelly::Context& c = *ctx->c;
  std::lock_guard<std::mutex> lk(c.mu);
  if (c.flush_bytes < bytes) {  // the context's buffer, grown on demand and freed with the context
    if (c.flush_buf) {
      cudaStreamSynchronize(c.stream);
      cudaFree(c.flush_buf);
    }
    c.flush_buf = nullptr;
    c.flush_bytes = 0;
    if (cudaMalloc(&c.flush_buf, bytes) != cudaSuccess) {
      c.flush_buf = nullptr;
      return snelly::fail(SNELLY_EDEVICE, "cudaMalloc failed");
    }
    c.flush_bytes = bytes;
  }
  l2_flush_kernel<<<c.sm_count * 4, 256, 0, c.stream>>>((float4*)c.flush_buf, bytes / 16, 0.0f);
  c.launches += 1;
  if (cudaGetLastError() != cudaSuccess) return snelly::fail(SNELLY_EDEVICE, "flush launch failed");
  return SNELLY_OK;
}

}  // extern "C"
