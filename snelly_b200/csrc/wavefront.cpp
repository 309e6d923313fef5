// wavefront.cpp - host side of the wavefront integrator (kernels in kernels/pt_wavefront.cuh):
// the per-path state and queues in HBM, and the stage launches of one frame on one or more
// concurrent streams.
#include <algorithm>
#include <thread>

#include "runtime_internal.h"

namespace snelly {

// The job's pixels are split into up to wf_split contiguous ranges ("parts"), each with its own
// path state, queues and counters, whose stages run on their own streams: while one part's
// extend launch drains (its last, longest rays on few lanes) or its shade stage runs, the other
// parts' launches fill the SMs it leaves idle. A path's computation does not depend on its part.
int Context::alloc_wavefront(Job& j) {
  if (j.scene->opts.max_samples_per_frame != 1) return SNELLY_OK;  // served by the per-pixel kernel
  const size_t P = (size_t)j.desc.width * j.desc.height;
  int parts = std::max(1, std::min(wf_split, SNELLY_WF_MAX_PARTS));
  if (P < (size_t)parts * 65536) parts = 1;  // small images: one part keeps each launch full
  // per path: 17 float4 arrays + info + rng + parked-ray state (3 per path), shadow flags, pending
  // count, int queues (2 active, 2 x 2 shadow, 2 x 3 parked, 2 x 4 shade); per part: counters
  // and the 256-byte alignment of its 31 sub-buffers
  size_t bytes = (19 * 16 + 3 * 16 + 2 + 4 + (2 + 2 * 2 + 2 * 3 + 2 * 4) * 4) * P +
                 (size_t)parts * (4 * WF_COUNTERS + 32 * 256);
  int rc = alloc(j.wf, bytes);
  if (rc) return rc;
  char* p = (char*)j.wf.ptr;
  auto take = [&](size_t n) {  // 256-byte aligned sub-buffers
    char* q = p;
    p += (n + 255) / 256 * 256;
    return q;
  };
  size_t begin = 0;
  for (int k = 0; k < parts; ++k) {
    const size_t Pk = P / parts + ((size_t)k < P % parts ? 1 : 0);
    const size_t f4 = 16 * Pk;
    WfBuffers& B = j.wfb[k];
    float4** f4s[] = {&B.pos, &B.dir, &B.thr, &B.rad, &B.cmf, &B.mis, &B.xyzw, &B.hit, &B.nee_org, &B.nee_thr,
                      &B.nee_extra, &B.nee_dir[0], &B.nee_dir[1], &B.nee_c[0], &B.nee_c[1], &B.nee_li[0],
                      &B.nee_li[1]};
    for (float4** q : f4s) *q = (float4*)take(f4);
    B.info = (int4*)take(f4);
    B.rng = (uint4*)take(f4);
    B.mt = (float4*)take(3 * f4);
    B.pend = (int*)take(4 * Pk);
    B.qc[0] = (int*)take(12 * Pk);
    B.qc[1] = (int*)take(12 * Pk);
    B.qa[0] = (int*)take(4 * Pk);
    B.qa[1] = (int*)take(4 * Pk);
    B.qs[0] = (int*)take(8 * Pk);
    B.qs[1] = (int*)take(8 * Pk);
    B.qshade[0] = (int*)take(16 * Pk);
    B.qshade[1] = (int*)take(16 * Pk);
    B.cnt = (int*)take(4 * WF_COUNTERS);
    B.shadow = (unsigned char*)take(2 * Pk);
    B.paths = (int)Pk;
    B.pixel_begin = (int)begin;
    begin += Pk;
  }
  j.wf_parts = parts;
  if ((size_t)(p - (char*)j.wf.ptr) > bytes) return fail(SNELLY_EDEVICE, "wavefront buffer layout overflow");
  return SNELLY_OK;
}

void Context::release_wavefront(Job& j) {
  release(j.wf);
  for (auto& B : j.wfb) B = WfBuffers{};
  j.wf_parts = 0;
}

int Context::enqueue_wavefront_frames(Job& j, int frames) {
  Module& m = *j.module;
  if (!j.wf.ptr || j.wf_parts < 1 || !m.f_wf_generate || !m.f_wf_extend || !m.f_wf_shade)
    return fail(SNELLY_EINVAL, "wavefront integrator not available for this job");
  if (frames <= 0) return SNELLY_OK;
  const int parts = j.wf_parts;
  // streams and events, created on first use; part 0 runs on the context stream
  wf_streams[0] = stream;
  for (int k = 1; k < parts; ++k)
    if (!wf_streams[k]) RT_TRY(cudaStreamCreateWithFlags(&wf_streams[k], cudaStreamNonBlocking));
  if (!wf_fork) RT_TRY(cudaEventCreateWithFlags(&wf_fork, cudaEventDisableTiming));
  for (int k = 0; k < parts; ++k)
    if (!wf_join[k]) RT_TRY(cudaEventCreateWithFlags(&wf_join[k], cudaEventDisableTiming));
  if (!poll_host) {
    if (cudaMallocHost((void**)&poll_host, 2 * SNELLY_WF_MAX_PARTS * sizeof(int)) != cudaSuccess) {
      poll_host = nullptr;
      return fail(SNELLY_EDEVICE, "pinned host allocation failed");
    }
  }
  for (auto& row : poll_done)
    for (int k = 0; k < parts; ++k)
      if (!row[k]) RT_TRY(cudaEventCreateWithFlags(&row[k], cudaEventDisableTiming));
  // the other parts start after the work already on the context stream (parameter upload)
  RT_TRY(cudaEventRecord(wf_fork, stream));
  for (int k = 1; k < parts; ++k) RT_TRY(cudaStreamWaitEvent(wf_streams[k], wf_fork, 0));
  void* jobs = j.tables.ptr;
  void* gparams = j.gparams.ptr;
  auto launch_on = [&](int k, cudaKernel_t f, int blocks, void** args) -> int {
    RT_TRY(cudaLaunchKernel((const void*)f, dim3((unsigned)blocks), dim3(SNELLY_BLOCK), args, 0, wf_streams[k]));
    launches++;
    return SNELLY_OK;
  };
  // Per frame and part: generate, then iterations of (extend, shade). The first `budgeted`
  // iterations park the slowest rays when their work runs out; after them every iteration
  // advances every path by one vertex, so `nominal` more always finish the frame. Beyond the
  // nominal count, a part's iterations go in pairs, each followed by a read of its paths-left
  // count; a part gets its next pair once the read of the pair before last has landed, so its
  // stream always has a pair queued, and it moves on to its next frame once a read shows zero (an
  // extra pair then finds empty queues and returns at once). The parts are independent pixel
  // ranges on their own streams, so a part that finishes a frame early starts the next one while
  // the others still trace the stragglers of theirs; the host serves whichever part's read has
  // landed and never waits on one part while another could be fed.
  const int nominal = j.scene->opts.max_bounces + 2;
  const int budgeted = wf_park_iters >= 0 ? std::min(wf_park_iters, 8 * nominal) : 3 * nominal;
  const int max_iters = budgeted + nominal;
  if (max_iters + 2 > WF_MAX_ITERS) return fail(SNELLY_EINVAL, "too many wavefront iterations for max_bounces");
  const int extend_blocks = sm_count * m.extend_blocks_per_sm, shade_blocks = sm_count * 4;
  struct PartRun {
    int frame = 0, it = 0, checks = 0;
    int left = 0;  // paths of the frame not finished at the latest read (an upper bound afterwards)
    bool started = false;
  } run[SNELLY_WF_MAX_PARTS];
  auto pair = [&](int k) -> int {
    WfBuffers B = j.wfb[k];
    int it = run[k].it;
    int drain = it < budgeted ? wf_drain_steps : 0;
    // Both stages take their work from device-side counters whatever their grid. Once a read has
    // shown few paths left, smaller grids do the same work without launching blocks that would
    // find nothing to do: at most 3 rays (continuation, sky and sun shadows) per unfinished path.
    const long long left = run[k].left;
    const int eb = (int)std::max<long long>(sm_count, std::min<long long>(extend_blocks, (3 * left + SNELLY_BLOCK - 1) / SNELLY_BLOCK));
    const int sb = (int)std::max<long long>(sm_count, std::min<long long>(shade_blocks, (left + SNELLY_BLOCK - 1) / SNELLY_BLOCK));
    void* eargs[] = {&B, &it, &drain};
    int r = launch_on(k, m.f_wf_extend, eb, eargs);
    if (r) return r;
    void* sargs[] = {&jobs, &gparams, &B, &it};
    r = launch_on(k, m.f_wf_shade, sb, sargs);
    if (r) return r;
    ++run[k].it;
    return SNELLY_OK;
  };
  int rc, active = parts;
  while (active > 0) {
    bool progress = false;
    for (int k = 0; k < parts; ++k) {
      PartRun& R = run[k];
      if (R.frame >= frames) continue;
      if (!R.started) {  // the part's next frame: camera rays, then the unpolled iterations
        WfBuffers B = j.wfb[k];
        void* gargs[] = {&jobs, &gparams, &B};
        if ((rc = launch_on(k, m.f_wf_generate, (B.paths + SNELLY_BLOCK - 1) / SNELLY_BLOCK, gargs))) return rc;
        R.started = true;
        R.it = 0;
        R.checks = 0;
        R.left = B.paths;
        while (R.it < nominal)
          if ((rc = pair(k))) return rc;
        progress = true;
        continue;
      }
      bool frame_done = R.it >= max_iters;
      if (!frame_done && R.checks >= 2) {  // the older of the part's two outstanding reads
        const int prev = R.checks & 1;
        const cudaError_t q = cudaEventQuery(poll_done[prev][k]);
        if (q == cudaErrorNotReady) continue;  // the part still has two pairs queued: serve the others
        if (q != cudaSuccess) return fail(SNELLY_EDEVICE, std::string("wavefront progress wait failed: ") + cudaGetErrorString(q));
        R.left = poll_host[prev * SNELLY_WF_MAX_PARTS + k];
        frame_done = R.left == 0;
      }
      progress = true;
      if (frame_done) {
        R.started = false;
        if (++R.frame >= frames) --active;
        continue;
      }
      if ((rc = pair(k)) || (rc = pair(k))) return rc;
      const int slot = R.checks & 1;
      if (cudaMemcpyAsync(poll_host + slot * SNELLY_WF_MAX_PARTS + k, j.wfb[k].cnt + WF_LEFT, sizeof(int),
                          cudaMemcpyDeviceToHost, wf_streams[k]) != cudaSuccess ||
          cudaEventRecord(poll_done[slot][k], wf_streams[k]) != cudaSuccess)
        return fail(SNELLY_EDEVICE, "wavefront progress read failed");
      ++R.checks;
    }
    if (!progress) std::this_thread::yield();  // every part has work queued
  }
  // later work on the context stream (resolve, readback) waits for every part
  for (int k = 1; k < parts; ++k) {
    RT_TRY(cudaEventRecord(wf_join[k], wf_streams[k]));
    RT_TRY(cudaStreamWaitEvent(stream, wf_join[k], 0));
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
        rc = k == 0 ? launch(j.module->f_frame_mega, j.blocks, SNELLY_BLOCK, margs) : enqueue_wavefront_frames(j, 1);
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
