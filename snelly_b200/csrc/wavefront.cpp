// wavefront.cpp - host side of the wavefront integrator (kernels in kernels/pt_wavefront.cuh):
// the per-path state and queues in HBM, and the stage launches of one frame.
#include "runtime_internal.h"

namespace snelly {

int Context::alloc_wavefront(Job& j) {
  if (j.scene->opts.max_samples_per_frame != 1) return SNELLY_OK;  // served by the per-pixel kernel
  const size_t P = (size_t)j.desc.width * j.desc.height;
  const size_t f4 = 16 * P;
  // 17 float4 arrays + info + rng, shadow flags, 2+2+1(x4) int queues, counters
  size_t bytes = 19 * f4 + 2 * P + (2 + 2 * 2 + 4) * 4 * P + 4 * WF_COUNTERS + 27 * 256;
  int rc = alloc(j.wf, bytes);
  if (rc) return rc;
  char* p = (char*)j.wf.ptr;
  auto take = [&](size_t n) {  // 256-byte aligned sub-buffers
    char* q = p;
    p += (n + 255) / 256 * 256;
    return q;
  };
  WfBuffers& B = j.wfb;
  float4** f4s[] = {&B.pos, &B.dir, &B.thr, &B.rad, &B.cmf, &B.mis, &B.xyzw, &B.hit, &B.nee_org, &B.nee_thr,
                    &B.nee_extra, &B.nee_dir[0], &B.nee_dir[1], &B.nee_c[0], &B.nee_c[1], &B.nee_li[0],
                    &B.nee_li[1]};
  for (float4** q : f4s) *q = (float4*)take(f4);
  B.info = (int4*)take(f4);
  B.rng = (uint4*)take(f4);
  B.qa[0] = (int*)take(4 * P);
  B.qa[1] = (int*)take(4 * P);
  B.qs[0] = (int*)take(8 * P);
  B.qs[1] = (int*)take(8 * P);
  B.qshade = (int*)take(16 * P);
  B.cnt = (int*)take(4 * WF_COUNTERS);
  B.shadow = (unsigned char*)take(2 * P);
  B.paths = (int)P;
  B.pixel_begin = 0;
  if ((size_t)(p - (char*)j.wf.ptr) > bytes) return fail(SNELLY_EDEVICE, "wavefront buffer layout overflow");
  return SNELLY_OK;
}

void Context::release_wavefront(Job& j) {
  release(j.wf);
  j.wfb = WfBuffers{};
}

int Context::enqueue_wavefront_frame(Job& j) {
  Module& m = *j.module;
  if (!j.wf.ptr || !m.f_wf_generate || !m.f_wf_extend || !m.f_wf_shade)
    return fail(SNELLY_EINVAL, "wavefront integrator not available for this job");
  void* jobs = j.tables.ptr;
  void* gparams = j.gparams.ptr;
  WfBuffers B = j.wfb;
  int gen_blocks = (B.paths + SNELLY_BLOCK - 1) / SNELLY_BLOCK;
  void* gargs[] = {&jobs, &gparams, &B};
  int rc = launch(m.f_wf_generate, gen_blocks, SNELLY_BLOCK, gargs);
  if (rc) return rc;
  const int iters = j.scene->opts.max_bounces + 2;
  const int extend_blocks = sm_count * m.extend_blocks_per_sm, shade_blocks = sm_count * 4;
  for (int it = 0; it < iters; ++it) {
    void* eargs[] = {&B, &it};
    if ((rc = launch(m.f_wf_extend, extend_blocks, SNELLY_BLOCK, eargs))) return rc;
    void* sargs[] = {&jobs, &gparams, &B, &it};
    if ((rc = launch(m.f_wf_shade, shade_blocks, SNELLY_BLOCK, sargs))) return rc;
  }
  return SNELLY_OK;
}

// The integrator choice of SNELLY_KERNEL_AUTO: per (scene module, image-size class) the first job
// times one warm-up and two frames of each integrator on its own buffers, keeps the faster and
// caches the decision; the job's state is seeded again afterwards by the caller. The size class is
// the power of two nearest the pixel count (tail effects make the choice size-dependent).
int Context::autotune(Job& j) {
  const long long npix = (long long)j.desc.width * j.desc.height;
  int cls = 0;
  while ((1ll << (cls + 1)) <= npix) ++cls;
  if (npix - (1ll << cls) > (1ll << (cls + 1)) - npix) ++cls;
  const std::string key = j.module->key + "/" + std::to_string(cls);
  auto it = tuned.find(key);
  int best;
  if (it != tuned.end()) {
    best = it->second;
  } else {
    int rc = upload_slot(j, 0);
    if (rc) return rc;
    void* tables = j.tables.ptr;
    void* bstart = (char*)j.tables.ptr + 128;
    int njobs = 1;
    void* gparams = j.gparams.ptr;
    void* sargs[] = {&tables, &bstart, &njobs};
    void* margs[] = {&tables, &bstart, &njobs, &gparams};
    if ((rc = launch(j.module->f_seed, j.blocks, SNELLY_BLOCK, sargs))) return rc;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
      if (e0) cudaEventDestroy(e0);
      return fail(SNELLY_EDEVICE, "autotune event creation failed");
    }
    float ms[2] = {0.0f, 0.0f};
    for (int k = 0; k < 2 && !rc; ++k) {
      for (int f = 0; f < 3 && !rc; ++f) {
        if (f == 1) cudaEventRecord(e0, stream);
        rc = k == 0 ? launch(j.module->f_frame_mega, j.blocks, SNELLY_BLOCK, margs) : enqueue_wavefront_frame(j);
      }
      cudaEventRecord(e1, stream);
      if (!rc && cudaEventSynchronize(e1) != cudaSuccess) rc = fail(SNELLY_EDEVICE, "autotune timing failed");
      if (!rc) cudaEventElapsedTime(&ms[k], e0, e1);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    best = ms[1] < ms[0] ? SNELLY_KERNEL_WAVEFRONT : SNELLY_KERNEL_MEGA;
    tuned[key] = best;
  }
  j.kernel_mode = best;
  if (best == SNELLY_KERNEL_MEGA) release_wavefront(j);
  return SNELLY_OK;
}

}  // namespace snelly
