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

}  // namespace snelly
