// wavefront.cpp - host side of the wavefront integrator (kernels in kernels/pt_wavefront.cuh):
// the per-path state and queues in HBM, and the stage launches of one frame on one or more
// concurrent streams.
#include <algorithm>
#include <cmath>
#include <thread>

#include "runtime_internal.h"

namespace snelly {

// The job's pixels are split into up to wfc.parts contiguous ranges ("parts"), each with its own
// path state, queues and counters, whose stages run on their own streams: while one part's
// extend launch drains (its last, longest rays on few lanes) or its shade stage runs, the other
// parts' launches fill the SMs it leaves idle. A path's computation does not depend on its part.
int Context::alloc_wavefront(Job& j) {
  if (j.scene->opts.max_samples_per_frame != 1) return SNELLY_OK;  // served by the per-pixel kernel
  const size_t P = (size_t)j.desc.width * j.desc.height;
  int parts = std::max(1, std::min(j.wfc.parts, SNELLY_WF_MAX_PARTS));
  while (parts > 1 && P < (size_t)parts * 65536) --parts;  // at least 65,536 pixels per range keep each launch full
  const int rec_f4 = j.module->wf_rec_f4;
  if (rec_f4 <= 0) return fail(SNELLY_EDEVICE, "module has no wavefront record layout");
  // per path: the record, parked-ray state (3 rays), shadow flags, pending count, int queues
  // (2 active, 2 x 2 shadow, 2 x 3 parked, 2 x 4 shade, subsurface walk, walk exit, medium
  // scatter); per part: counters and the 256-byte alignment of its 16 sub-buffers
  size_t bytes = ((size_t)rec_f4 * 16 + 3 * 16 + 2 + 4 + (2 + 2 * 2 + 2 * 3 + 2 * 4 + 3) * 4) * P +
                 (size_t)parts * (4 * WF_COUNTERS + 18 * 256);
  int rc = alloc(j.wf, bytes);
  if (rc) return rc;
  char* p = (char*)j.wf.ptr;
  auto take = [&](size_t n) {  // 256-byte aligned sub-buffers
    char* q = p;
    p += (n + 255) / 256 * 256;
    return q;
  };
  // interleaved ranges: the image's rows go to the ranges in turn (range k: rows k, k + parts, ...;
  // only the last row can be short), so that every range holds a like share of the scene and the
  // ranges finish their launch sequences together instead of the emptiest ones first
  const size_t G = (j.wfc.interleave && parts > 1) ? (size_t)j.desc.width : 0;
  const size_t ng = G ? (P + G - 1) / G : 0;
  const bool dealt = G > 0 && ng >= (size_t)parts;
  size_t begin = 0;
  for (int k = 0; k < parts; ++k) {
    size_t Pk = P / parts + ((size_t)k < P % parts ? 1 : 0);
    if (dealt) {
      const size_t groups = (ng - k + parts - 1) / parts;
      Pk = groups * G - ((ng - 1) % parts == (size_t)k ? ng * G - P : 0);
    }
    const size_t f4 = 16 * Pk;
    WfBuffers& B = j.wfb[k];
    B.rec = (float4*)take((size_t)rec_f4 * f4);
    B.rec_f4 = rec_f4;
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
    B.qsss = (int*)take(4 * Pk);
    B.qexit = (int*)take(4 * Pk);
    B.qvol = (int*)take(4 * Pk);
    B.cnt = (int*)take(4 * WF_COUNTERS);
    B.shadow = (unsigned char*)take(2 * Pk);
    B.paths = (int)Pk;
    B.pixel_begin = dealt ? k : (int)begin;
    B.pixel_group = dealt ? (int)G : 0;
    B.pixel_parts = parts;
    begin += Pk;
  }
  if (begin != P) return fail(SNELLY_EDEVICE, "wavefront pixel ranges do not cover the image");
  j.wf_parts = parts;
  j.wfc.parts = parts;
  if ((size_t)(p - (char*)j.wf.ptr) > bytes) return fail(SNELLY_EDEVICE, "wavefront buffer layout overflow");
  return SNELLY_OK;
}

void Context::release_wavefront(Job& j) {
  release(j.wf);
  for (auto& B : j.wfb) B = WfBuffers{};
  j.wf_parts = 0;
}

int Context::enqueue_wavefront_frames(Job& j, int frames) {
  std::vector<Job*> js{&j};
  std::vector<int> fs{frames};
  return enqueue_wavefront(js, fs, {}, true);
}

// The wavefront frames of several jobs at once. Every job's pixel ranges ("parts") get their own
// stream; a job's parameters and scene uniforms go to its own constant-memory slot, uploaded on
// its first part's stream once the work it follows is done (`after`: an event per module, for
// slots that another launch sequence of that module used). Up to SNELLY_MAX_BATCH jobs run
// concurrently; more wait for the next wave. With `slot0_ready` (one job whose
// parameters its caller has already uploaded into slot 0 on the context stream, enqueue_frames),
// the job runs its first part on the context stream in slot 0 and nothing is uploaded.
//
// Per launch sequence and part: generate, then iterations of (extend, shade [, subsurface walk]).
// With overlapping frames (wfc.overlap) one sequence runs all of the advance's frames: generate
// starts every pixel's first sample and each finished sample starts the pixel's next in place
// (B.samples), so no iteration waits for the last paths of a frame; otherwise each frame is a
// sequence of its own. The first `budgeted` iterations park the slowest rays when their work runs
// out; after them every iteration advances every path by one vertex, so `nominal` more per sample
// always finish the sequence. Beyond the first `nominal`, a part's iterations go in pairs, each
// followed by a read of its paths-left count; a part gets its next pair once the read of the pair
// before last has landed, so its stream always has a pair queued, and it moves on to its next
// sequence once a read shows zero (an extra pair then finds empty queues and returns at once).
// The parts are independent pixel ranges, so a part that finishes early starts its next sequence
// while the others still trace the stragglers of theirs; the host serves whichever part's read
// has landed and never waits on one part while another could be fed.
int Context::enqueue_wavefront(const std::vector<Job*>& js, const std::vector<int>& frames,
                               const std::map<Module*, cudaEvent_t>& after, bool slot0_ready) {
  for (size_t q = 0; q < js.size(); ++q) {
    Job& j = *js[q];
    Module& m = *j.module;
    if (!j.wf.ptr || j.wf_parts < 1 || !m.f_wf_generate || !m.f_wf_extend || !m.f_wf_shade ||
        m.wf_rec_f4 != j.wfb[0].rec_f4)
      return fail(SNELLY_EINVAL, "wavefront integrator not available for this job");
  }
  if (slot0_ready && js.size() != 1) return fail(SNELLY_EINVAL, "slot 0 holds one job's parameters");
  const bool single = slot0_ready;
  // waves of at most SNELLY_MAX_BATCH concurrent jobs (so at most that many jobs' ranges and
  // streams at a time, and one constant-memory slot per job of a module)
  std::vector<int> wave(js.size(), 0), slot(js.size(), 0);
  {
    std::map<std::pair<int, Module*>, int> seen;
    for (size_t q = 0; q < js.size(); ++q) {
      wave[q] = (int)(q / SNELLY_MAX_BATCH);
      slot[q] = seen[{wave[q], js[q]->module}]++;
    }
  }
  const int nwaves = js.empty() ? 0 : *std::max_element(wave.begin(), wave.end()) + 1;
  if (!wf_fork) RT_TRY(cudaEventCreateWithFlags(&wf_fork, cudaEventDisableTiming));
  for (int w = 0; w < nwaves; ++w) {
    // the parts of this wave, each with a stream and two progress-read events
    struct PartRun {
      Job* j;
      int k, total = 0, frame = 0, it = 0, checks = 0;  // total, frame: launch sequences
      int samples = 1;  // samples per pixel of each sequence
      long long left = 0;  // paths of the frame not finished at the latest read (an upper bound afterwards)
      bool started = false;
      cudaStream_t st = nullptr;
      int idx = 0;  // index into the stream / event / pinned-word pools
    };
    std::vector<PartRun> runs;
    for (size_t q = 0; q < js.size(); ++q) {
      if (wave[q] != w || frames[q] <= 0) continue;
      for (int k = 0; k < js[q]->wf_parts; ++k) {
        PartRun R;
        R.j = js[q];
        R.k = k;
        R.total = js[q]->wfc.overlap ? 1 : frames[q];
        R.samples = js[q]->wfc.overlap ? frames[q] : 1;
        R.idx = (int)runs.size();
        runs.push_back(R);
      }
    }
    if (runs.empty()) continue;
    const size_t np = runs.size();
    while (wf_pool.size() < np) {  // streams, created on first use
      cudaStream_t st;
      RT_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
      wf_pool.push_back(st);
    }
    while (wf_events.size() < 3 * np) {  // per part: two progress reads and a join
      cudaEvent_t e;
      RT_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      wf_events.push_back(e);
    }
    if (poll_cap < 2 * np) {
      if (poll_host) cudaFreeHost(poll_host);
      poll_host = nullptr;
      poll_cap = 0;
      if (cudaMallocHost((void**)&poll_host, 2 * np * sizeof(int)) != cudaSuccess) {
        poll_host = nullptr;
        return fail(SNELLY_EDEVICE, "pinned host allocation failed");
      }
      poll_cap = 2 * np;
    }
    for (auto& R : runs) R.st = (single && R.k == 0) ? stream : wf_pool[R.idx];
    // every part starts after the work already on the context stream (parameter upload, seeding)
    RT_TRY(cudaEventRecord(wf_fork, stream));
    for (auto& R : runs)
      if (R.st != stream) RT_TRY(cudaStreamWaitEvent(R.st, wf_fork, 0));
    for (size_t q = 0; q < js.size(); ++q) {  // slots, and the uploads into them on each job's first part
      if (wave[q] != w || frames[q] <= 0) continue;
      Job& j = *js[q];
      for (int k = 0; k < j.wf_parts; ++k) j.wfb[k].slot = single ? 0 : slot[q];
      if (single) continue;
      PartRun* first = nullptr;
      for (auto& R : runs)
        if (R.j == &j && R.k == 0) first = &R;
      auto a = after.find(j.module);
      if (a != after.end() && a->second) RT_TRY(cudaStreamWaitEvent(first->st, a->second, 0));
      Module& m = *j.module;
      RT_TRY(cudaMemcpyAsync(m.c_params + slot[q] * sizeof(SnellyParams), &j.params, sizeof(SnellyParams),
                             cudaMemcpyHostToDevice, first->st));
      size_t ub = std::min(j.ublock.size(), m.slot_uniform_bytes);
      if (ub)
        RT_TRY(cudaMemcpyAsync(m.c_uniforms + slot[q] * m.slot_uniform_bytes, j.ublock.data(), ub,
                               cudaMemcpyHostToDevice, first->st));
      if (j.wf_parts > 1) {  // the job's other parts read the slot too
        cudaEvent_t up = wf_events[3 * first->idx + 2];
        RT_TRY(cudaEventRecord(up, first->st));
        for (auto& R : runs)
          if (R.j == &j && R.k > 0) RT_TRY(cudaStreamWaitEvent(R.st, up, 0));
      }
    }
    // Programmatic dependent launch (wf_pdl): a kernel may begin launching while the previous
    // kernel of its stream runs; it waits for that grid on entry (wf_kernel_entry).
    cudaLaunchAttribute pdl_attr[1];
    pdl_attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    pdl_attr[0].val.programmaticStreamSerializationAllowed = 1;
    auto launch_on = [&](PartRun& R, cudaKernel_t f, int blocks, int threads, void** args) -> int {
      cudaLaunchConfig_t lc = {};
      lc.gridDim = dim3((unsigned)blocks);
      lc.blockDim = dim3((unsigned)threads);
      lc.dynamicSmemBytes = 0;
      lc.stream = R.st;
      lc.attrs = pdl_attr;
      lc.numAttrs = wf_pdl ? 1 : 0;
      RT_TRY(cudaLaunchKernelExC(&lc, (const void*)f, args));
      launches++;
      return SNELLY_OK;
    };
    auto pair = [&](PartRun& R) -> int {
      Job& j = *R.j;
      Module& m = *j.module;
      WfBuffers B = j.wfb[R.k];
      B.samples = R.samples;
      void* jobs = j.tables.ptr;
      void* gparams = j.gparams.ptr;
      const int nominal = j.scene->opts.max_bounces + 2;
      const int budgeted = R.samples * (wf_park_iters >= 0 ? std::min(wf_park_iters, 8 * nominal) : 3 * nominal);
      int it = R.it;
      const WfConfig& cf = j.wfc;
      // rays are parked in the first `budgeted` iterations while more than park_left / 1024 of
      // the part's paths are unfinished (per the latest read): a few stragglers are then marched
      // to the end in one launch instead of a few dozen steps per iteration
      int drain = (it < budgeted && R.left * 1024 > (long long)cf.park_left * B.paths) ? cf.drain : 0;
      int chunk = cf.chunk, grab = cf.grab, refill = cf.refill;
      const int bs = cf.block;
      // Both stages take their work from device-side counters whatever their grid. Once a read has
      // shown few paths left, smaller grids do the same work without launching blocks that would
      // find nothing to do: at most 3 rays (continuation, sky and sun shadows) per unfinished path.
      const long long left = R.left;
      const long long extend_blocks = (long long)sm_count * (bs < 128 ? m.extend_blocks_per_sm64 : m.extend_blocks_per_sm);
      const long long shade_blocks =
          std::max<long long>(1, (long long)sm_count * m.shade_blocks_per_sm * cf.shade_share / 8) * (128 / bs);
      const long long lanes = (3 * left + cf.lane_rays - 1) / cf.lane_rays;
      const int eb = (int)std::max<long long>(sm_count, std::min(extend_blocks, (lanes + bs - 1) / bs));
      const int sb = (int)std::max<long long>(sm_count, std::min(shade_blocks, (left + bs - 1) / bs));
      const bool split = cf.shade_split && m.f_wf_shade_seg[0];
      const bool walk = m.f_wf_sss && j.params.subsurfaceMFP > 0.0f;  // vertices may choose the walk
      const bool volume = m.f_wf_volume && cf.vol_stage;  // medium collisions go to the volume stage
      B.vol_stage = volume ? 1 : 0;
      void* eargs[] = {&B, &it, &drain, &chunk, &grab, &refill};
      int r = launch_on(R, m.f_wf_extend, eb, bs, eargs);
      if (r) return r;
      void* sargs[] = {&jobs, &gparams, &B, &it};
      if (split) {  // one launch per material segment, each compiled for its material
        for (int sg = 0; sg < 4; ++sg)
          if (m.f_wf_shade_seg[sg] && (r = launch_on(R, m.f_wf_shade_seg[sg], sb, bs, sargs))) return r;
      } else if ((r = launch_on(R, m.f_wf_shade, sb, bs, sargs))) {
        return r;
      }
      if (walk && cf.walker && m.f_wf_walk && m.f_wf_walk_exit) {  // the walks it handed over: walker, then exits
        const int wb = sm_count * m.walk_blocks_per_sm;
        void* wargs[] = {&jobs, &gparams, &B, &it, &grab, &refill};
        if ((r = launch_on(R, m.f_wf_walk, wb, SNELLY_BLOCK, wargs))) return r;
        if ((r = launch_on(R, m.f_wf_walk_exit, sb, bs, sargs))) return r;
      } else if (walk && (r = launch_on(R, m.f_wf_sss, sb, bs, sargs))) {  // one thread per walk
        return r;
      }
      if (volume && (r = launch_on(R, m.f_wf_volume, sb, bs, sargs))) return r;  // the medium vertices
      ++R.it;
      return SNELLY_OK;
    };
    int rc;
    size_t active = runs.size();
    while (active > 0) {
      bool progress = false;
      for (auto& R : runs) {
        if (R.frame >= R.total) continue;
        Job& j = *R.j;
        const int nominal = j.scene->opts.max_bounces + 2;
        const int budgeted = R.samples * (wf_park_iters >= 0 ? std::min(wf_park_iters, 8 * nominal) : 3 * nominal);
        const int max_iters = budgeted + R.samples * nominal;
        if (!R.started) {  // the part's next sequence: camera rays, then the unpolled iterations
          WfBuffers B = j.wfb[R.k];
          B.samples = R.samples;
          void* jobs = j.tables.ptr;
          void* gparams = j.gparams.ptr;
          void* gargs[] = {&jobs, &gparams, &B};
          if ((rc = launch_on(R, j.module->f_wf_generate, (B.paths + SNELLY_BLOCK - 1) / SNELLY_BLOCK, SNELLY_BLOCK, gargs)))
            return rc;
          R.started = true;
          R.it = 0;
          R.checks = 0;
          R.left = B.paths;
          while (R.it < nominal)
            if ((rc = pair(R))) return rc;
          progress = true;
          continue;
        }
        bool frame_done = R.it >= max_iters;
        if (!frame_done && R.checks >= 2) {  // the older of the part's two outstanding reads
          const int prev = R.checks & 1;
          const cudaError_t q = cudaEventQuery(wf_events[3 * R.idx + prev]);
          if (q == cudaErrorNotReady) continue;  // the part still has two pairs queued: serve the others
          if (q != cudaSuccess)
            return fail(SNELLY_EDEVICE, std::string("wavefront progress wait failed: ") + cudaGetErrorString(q));
          R.left = poll_host[2 * R.idx + prev];
          frame_done = R.left == 0;
        }
        progress = true;
        if (frame_done) {
          R.started = false;
          if (++R.frame >= R.total) --active;
          continue;
        }
        if ((rc = pair(R)) || (rc = pair(R))) return rc;
        const int ps = R.checks & 1;
        if (cudaMemcpyAsync(poll_host + 2 * R.idx + ps, j.wfb[R.k].cnt + WF_LEFT, sizeof(int), cudaMemcpyDeviceToHost,
                            R.st) != cudaSuccess ||
            cudaEventRecord(wf_events[3 * R.idx + ps], R.st) != cudaSuccess)
          return fail(SNELLY_EDEVICE, "wavefront progress read failed");
        ++R.checks;
      }
      if (!progress) std::this_thread::yield();  // every part has work queued
    }
    // later work on the context stream (resolve, readback, the next wave) waits for every part
    for (auto& R : runs) {
      if (R.st == stream) continue;
      RT_TRY(cudaEventRecord(wf_events[3 * R.idx + 2], R.st));
      RT_TRY(cudaStreamWaitEvent(stream, wf_events[3 * R.idx + 2], 0));
    }
  }
  return SNELLY_OK;
}

// Frames of one job with the given integrator on its own buffers, timed with events on the
// context stream: one warm-up frame, then enough frames for about 40 ms (4 to 16) in one call, so
// that overlapping frames are timed over a sequence of several; the per-frame time. The job's
// state is seeded again afterwards by the caller.
int Context::time_frames(Job& j, int kernel, float* ms_per_frame) {
  void* tables = j.tables.ptr;
  void* bstart = (char*)j.tables.ptr + 128;
  int njobs = 1;
  void* gparams = j.gparams.ptr;
  void* margs[] = {&tables, &bstart, &njobs, &gparams};
  auto frames = [&](int n) -> int {
    if (kernel == SNELLY_KERNEL_WAVEFRONT) return enqueue_wavefront_frames(j, n);
    for (int f = 0; f < n; ++f)
      if (int rc = launch(j.module->f_frame_mega, j.blocks, SNELLY_BLOCK, margs)) return rc;
    return SNELLY_OK;
  };
  cudaEvent_t e[3] = {nullptr, nullptr, nullptr};
  for (auto& ev : e)
    if (cudaEventCreate(&ev) != cudaSuccess) {
      for (auto& x : e)
        if (x) cudaEventDestroy(x);
      return fail(SNELLY_EDEVICE, "autotune event creation failed");
    }
  int rc = SNELLY_OK;
  float warm = 0.0f, ms = 0.0f;
  int n = 2;
  if (!(rc = (cudaEventRecord(e[0], stream) == cudaSuccess ? frames(1) : SNELLY_EDEVICE))) {
    cudaEventRecord(e[1], stream);
    if (cudaEventSynchronize(e[1]) != cudaSuccess) rc = fail(SNELLY_EDEVICE, "autotune timing failed");
    else cudaEventElapsedTime(&warm, e[0], e[1]);
  }
  if (!rc) {
    n = std::max(4, std::min(16, (int)std::ceil(40.0f / std::max(warm, 1e-3f))));
    rc = frames(n);
  }
  if (!rc) {
    cudaEventRecord(e[2], stream);
    if (cudaEventSynchronize(e[2]) != cudaSuccess) rc = fail(SNELLY_EDEVICE, "autotune timing failed");
    else cudaEventElapsedTime(&ms, e[1], e[2]);
  }
  for (auto& x : e) cudaEventDestroy(x);
  *ms_per_frame = ms / n;
  return rc;
}

// The integrator choice of SNELLY_KERNEL_AUTO and the wavefront's launch configuration, per
// (scene module, image-size class): the first such job times, on its own buffers, the wavefront
// with each value of one configuration field in turn (the best so far for the others; one pass
// over pixel ranges, per-material shading, drain steps, refill chunk, claim size, refill threshold,
// block shape, the unfinished-path fraction below which parking stops and, for jobs with subsurface
// walks, the persistent walker against one thread per walk, the extend grid's rays per lane, and
// overlapping frames against frame after frame, and the share of the GPU a shade launch may fill;
// then a second pass over the pixel ranges and the rays per lane; fields fixed by the environment
// are not varied), then the path-per-thread
// kernel, keeps the fastest and caches the decision; the job's state is seeded again afterwards
// by the caller. The size class is the power of two nearest the pixel count (tail effects make
// the choice size-dependent). A candidate must beat the best so far by 1.5% to replace it.
// A candidate replaces the best configuration so far only when it is faster by more than the
// timing noise of one short window (about 1-2%), so that noise does not walk the choice away
// from the defaults (measured on the 1080p fractal workload) or from a better earlier value.
static constexpr float kTuneMargin = 0.985f;

int Context::autotune(Job& j) {
  const long long npix = (long long)j.desc.width * j.desc.height;
  int cls = 0;
  while ((1ll << (cls + 1)) <= npix) ++cls;
  if (npix - (1ll << cls) > (1ll << (cls + 1)) - npix) ++cls;
  const std::string key = j.module->key + "/" + std::to_string(cls);
  auto it = tuned.find(key);
  Tuned best{SNELLY_KERNEL_WAVEFRONT, j.wfc};  // the context's defaults, pixel ranges as allocated
  if (it != tuned.end()) {
    best = it->second;
  } else {
    int rc = upload_slot(j, 0);
    if (rc) return rc;
    void* tables = j.tables.ptr;
    void* bstart = (char*)j.tables.ptr + 128;
    int njobs = 1;
    void* sargs[] = {&tables, &bstart, &njobs};
    if ((rc = launch(j.module->f_seed, j.blocks, SNELLY_BLOCK, sargs))) return rc;
    auto try_cfg = [&](const WfConfig& cfg, float* ms) -> int {
      if (cfg.parts != j.wfc.parts || cfg.interleave != j.wfc.interleave) {  // another split into pixel ranges: new buffers
        if (cudaStreamSynchronize(stream) != cudaSuccess) return fail(SNELLY_EDEVICE, "autotune sync failed");
        release_wavefront(j);
        j.wfc = cfg;
        if (int r = alloc_wavefront(j)) return r;
      }
      j.wfc = cfg;
      return time_frames(j, SNELLY_KERNEL_WAVEFRONT, ms);
    };
    float best_ms = 0.0f;
    if ((rc = try_cfg(best.cfg, &best_ms))) return rc;
    struct Field {
      int WfConfig::*f;
      std::vector<int> values;
    } fields[] = {{&WfConfig::parts, {1, 2, 3, 4, 6, 8}}, {&WfConfig::shade_split, {0, 1}},
                  {&WfConfig::drain, {16, 32, 64}},       {&WfConfig::chunk, {4, 8, 16}},
                  {&WfConfig::grab, {16, 32, 64}},        {&WfConfig::refill, {2, 4, 8}},
                  {&WfConfig::block, {64, 128}},          {&WfConfig::park_left, {0, 8, 32, 128}},
                  {&WfConfig::walker, {0, 1}},            {&WfConfig::lane_rays, {1, 2, 4, 8, 16}},
                  {&WfConfig::overlap, {0, 1}},           {&WfConfig::shade_share, {3, 5, 8}},
                  {&WfConfig::interleave, {0, 1}},        {&WfConfig::vol_stage, {0, 1}}};
    const unsigned nfields = sizeof fields / sizeof fields[0];
    const bool walks = j.module->f_wf_walk && j.params.subsurfaceMFP > 0.0f;
    auto descend = [&](unsigned k) -> int {  // try every value of field k against the best so far
      if (wf_fixed & (1u << k)) return SNELLY_OK;
      if (fields[k].f == &WfConfig::walker && !walks) return SNELLY_OK;  // no subsurface walks to time
      if (fields[k].f == &WfConfig::vol_stage && !j.module->f_wf_volume) return SNELLY_OK;  // no medium
      for (int v : fields[k].values) {
        WfConfig cfg = best.cfg;
        if (cfg.*(fields[k].f) == v) continue;
        cfg.*(fields[k].f) = v;
        if (fields[k].f == &WfConfig::parts && v > 1 && npix < (long long)v * 65536)
          continue;  // too small for that many ranges
        float ms = 0.0f;
        if (int r = try_cfg(cfg, &ms)) return r;
        if (ms < best_ms * kTuneMargin) {
          best_ms = ms;
          best.cfg = cfg;
        }
      }
      return SNELLY_OK;
    };
    for (unsigned k = 0; k < nfields; ++k)
      if ((rc = descend(k))) return rc;
    // the pixel ranges (their number and how they deal out the rows) and the extend grid's rays
    // per lane decide together how the ranges' launches share the GPU: a second pass over them
    for (unsigned k = 0; k < nfields; ++k)
      if ((fields[k].f == &WfConfig::parts || fields[k].f == &WfConfig::lane_rays ||
           fields[k].f == &WfConfig::interleave) &&
          (rc = descend(k)))
        return rc;
    float mega_ms = 0.0f;
    if ((rc = time_frames(j, SNELLY_KERNEL_MEGA, &mega_ms))) return rc;
    best.kernel = mega_ms < best_ms ? SNELLY_KERNEL_MEGA : SNELLY_KERNEL_WAVEFRONT;
    tuned[key] = best;
  }
  j.kernel_mode = best.kernel;
  if (best.kernel == SNELLY_KERNEL_MEGA) {
    if (cudaStreamSynchronize(stream) != cudaSuccess) return fail(SNELLY_EDEVICE, "autotune sync failed");
    release_wavefront(j);
    return SNELLY_OK;
  }
  if (best.cfg.parts != j.wfc.parts || best.cfg.interleave != j.wfc.interleave) {
    if (cudaStreamSynchronize(stream) != cudaSuccess) return fail(SNELLY_EDEVICE, "autotune sync failed");
    release_wavefront(j);
    j.wfc = best.cfg;
    return alloc_wavefront(j);
  }
  j.wfc = best.cfg;
  return SNELLY_OK;
}

}  // namespace snelly
