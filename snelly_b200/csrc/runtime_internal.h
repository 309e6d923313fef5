// runtime_internal.h - internal types of libsnelly (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "glsl_transform.h"
#include "kernels/pt_launch.h"

// Return SNELLY_EDEVICE with the failing call and CUDA's message (needs `fail` in scope).
#define RT_TRY(expr)                                                                        \
  do {                                                                                      \
    cudaError_t e_ = (expr);                                                                \
    if (e_ != cudaSuccess) return fail(SNELLY_EDEVICE, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define SNELLY_WF_MAX_PARTS 8  // concurrent wavefront pixel ranges of one job, at most
#include "snelly.h"

static_assert(JOB_MODE_PT == SNELLY_MODE_PT && JOB_MODE_NORMALS == SNELLY_MODE_NORMALS &&
                  JOB_MODE_AO == SNELLY_MODE_AO && JOB_MODE_PICK == SNELLY_MODE_PICK &&
                  JOB_MODE_PTSIMPLE == SNELLY_MODE_PTSIMPLE,
              "kernel render-mode values follow the ABI's");
static_assert(sizeof(JobRec) <= 128, "a single-job table holds one JobRec before the block starts at byte 128");

#ifndef SNELLY_MAX_BATCH
#define SNELLY_MAX_BATCH 32
#endif

namespace snelly {

int fail(int code, const std::string& msg);

struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
};

// The scene string after the host-side assembly of js/renderer.js:217-316.
struct SceneSource {
  std::string glsl;     // with default hooks appended
  std::string defines;  // HAS_* / MAX_* preprocessor lines
  GlslTransformResult xf;
  bool has_custom_camera = false, has_surface = false, has_metal = false, has_dielectric = false;
  bool has_surface_nm = false, has_metal_nm = false, has_dielectric_nm = false, has_volume_emission = false;
};

struct Module {
  std::string key;
  cudaLibrary_t lib = nullptr;
  cudaKernel_t f_seed = nullptr, f_frame_mega = nullptr, f_resolve = nullptr;
  cudaKernel_t f_wf_generate = nullptr, f_wf_extend = nullptr, f_wf_shade = nullptr, f_wf_sss = nullptr;
  cudaKernel_t f_wf_walk = nullptr, f_wf_walk_exit = nullptr;  // the persistent subsurface walker
  cudaKernel_t f_wf_volume = nullptr;  // the heterogeneous medium's scatter stage (null without one)
  int walk_blocks_per_sm = 8;  // resident 128-thread blocks of the walker (occupancy query)
  // the shade stage split by queue segment: misses/finishing, surface, metal, dielectric (null
  // for a material the scene does not have)
  cudaKernel_t f_wf_shade_seg[4] = {nullptr, nullptr, nullptr, nullptr};
  int wf_rec_f4 = 0;  // float4 slots of the module's wavefront path record
  cudaKernel_t f_firsthit = nullptr, f_ptsimple = nullptr;
  int extend_blocks_per_sm = 8;  // resident 128-thread blocks of the persistent extend stage (occupancy query)
  int extend_blocks_per_sm64 = 16;  // the same for 64-thread blocks
  int shade_blocks_per_sm = 4;      // resident 128-thread blocks of the shade stage (occupancy query)
  char* c_params = nullptr;  // device addresses of the constant banks
  char* c_uniforms = nullptr;
  size_t c_uniforms_bytes = 0, slot_uniform_bytes = 0;
};

// Launch configuration of a wavefront job: chosen per (scene module, image-size class) by the
// autotuner, or the context's defaults.
struct WfConfig {
  int parts = 8;        // concurrent pixel ranges (one per 65,536 pixels at most)
  int shade_split = 0;  // the shade stage as one launch per material segment
  int drain = 32;       // steps an extend warp marches once its work runs out before parking (0: never)
  int chunk = 8;        // sphere-tracing steps between refills of idle lanes
  int grab = 32;        // work items a warp claims from the work head at a time
  int refill = 8;       // idle lanes of a warp that trigger a refill
  int block = 128;      // threads per block of the extend and shade launches (64 or 128)
  int park_left = 0;    // stop parking once at most park_left / 1024 of the paths are unfinished
  int walker = 0;       // subsurface walks by the persistent walker (1) or one thread per walk (0)
  int lane_rays = 16;   // extend grid: one lane per lane_rays rays the iteration may hold (a
                        // smaller grid lets the ranges' extend launches share the GPU)
  int overlap = 1;      // the frames of one advance overlap (a path that finishes its pixel's sample
                        // starts the pixel's next) rather than run one after another
  int shade_share = 8;  // shade grid: at most shade_share / 8 of the stage's resident blocks, so that
                        // other ranges' extend blocks fit beside a range's shade stage
  int interleave = 1;   // pixel ranges as the image's rows dealt to the ranges in turn (1), so that every
                        // range holds a like share of the scene, or as contiguous runs of rows (0)
  int vol_stage = 1;    // vertices that collide in a heterogeneous medium scatter in a stage of their
                        // own (1) rather than inside the shade stage (0)
};

struct Scene {
  uint64_t id = 0;
  SceneSource src;
  snelly_scene_opts opts{};
  int kernel_mode = SNELLY_KERNEL_MEGA;
  std::vector<unsigned char> ublock;  // uniform block (host copy), snapshotted by jobs
  std::map<std::string, DevBuf> textures;
  std::vector<DevBuf> retired_textures;  // replaced while jobs referenced them; freed with the scene
  std::shared_ptr<Module> module;
  // IEEE-mode build of the same program for the first-hit passes (normals, AO, pick), compiled on
  // first use when `module` is a fast-math build: those passes are deterministic and must agree
  // with the reference per pixel, and they trace one ray per pixel, so exact arithmetic costs
  // little there.
  std::shared_ptr<Module> strict_module;
};

struct Job {
  uint64_t id = 0;
  Scene* scene = nullptr;
  Module* module = nullptr;  // the build this job's kernels run from
  snelly_render_desc desc{};
  SnellyParams params{};
  std::vector<unsigned char> ublock;
  DevBuf rng, acc, comp, acc64, out, icdf, env, gparams, tables;
  DevBuf display;  // tonemapped image (snelly_tonemap), allocated on first use
  DevBuf wf;  // wavefront path state and queues
  WfBuffers wfb[SNELLY_WF_MAX_PARTS]{};  // one set per pixel range, each run on its own stream
  int wf_parts = 0;
  WfConfig wfc;  // its launch configuration
  int blocks = 0;
  int kernel_mode = SNELLY_KERNEL_MEGA;  // the integrator this job's frames run (after tuning)
  int pick_at = 0;           // a one-pixel pick job (snelly_pick)
  float pick_x = 0.0f, pick_y = 0.0f;
  int frames_enqueued = 0;
  bool cancelled = false;
  cudaEvent_t done = nullptr;
  cudaEvent_t read_done = nullptr;  // the last SNELLY_READ_ASYNC copy of `out` (on the copy stream)
  bool read_pending = false;
};

// Device-side tables of a batched launch, one set per batch stream.
struct BatchLane {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  DevBuf recs;     // JobRec[SNELLY_MAX_BATCH] + block starts
  DevBuf gparams;  // SnellyParams[SNELLY_MAX_BATCH]
};

struct Context {
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;  // SNELLY_READ_ASYNC device-to-host copies (created on first use)
  std::mutex mu;
  std::map<uint64_t, Scene> scenes;
  std::map<uint64_t, Job> jobs;
  std::map<std::string, std::shared_ptr<Module>> module_cache;
  DevBuf xyz;
  size_t budget = 0, used = 0;
  uint64_t next_id = 0;
  uint64_t launches = 0;
  std::string csrc_dir, kernel_dir, include_dir, cache_dir;
  std::vector<BatchLane> lanes;  // batch streams (created on first use)
  struct Tuned {
    int kernel;
    WfConfig cfg;
  };
  std::map<std::string, Tuned> tuned;  // autotuner decisions per (module, image-size class)
  // Wavefront defaults; a field set from the environment (SNELLY_WF_SPLIT, SNELLY_WF_DRAIN,
  // SNELLY_WF_SHADE_SPLIT, SNELLY_WF_CHUNK, SNELLY_WF_GRAB, SNELLY_WF_REFILL, SNELLY_WF_BLOCK,
  // SNELLY_WF_PARK_LEFT, SNELLY_WF_WALKER, SNELLY_WF_LANE_RAYS, SNELLY_WF_OVERLAP,
  // SNELLY_WF_SHADE_SHARE, SNELLY_WF_INTERLEAVE, SNELLY_WF_VOLUME) is also kept fixed by the autotuner.
  WfConfig wf_default;
  unsigned wf_fixed = 0;             // bit per WfConfig field, in declaration order
  int wf_park_iters = -1;            // iterations that may park rays; -1: 3 x (max_bounces + 2) (SNELLY_WF_PARK_ITERS)
  int wf_pdl = 0;                    // programmatic dependent launch of the wavefront kernels (SNELLY_WF_PDL)
  int* poll_host = nullptr;          // pinned words the wavefront's paths-left reads land in (2 per part)
  size_t poll_cap = 0;
  std::vector<cudaStream_t> wf_pool;  // one stream per concurrently running wavefront part
  std::vector<cudaEvent_t> wf_events;  // per part: two progress reads and a join
  cudaEvent_t wf_fork = nullptr;
  DevBuf stats_scratch;          // image-statistics partial sums
  void* static_stats_scratch = nullptr;  // device address of the allocation-free statistics scratch
  void* flush_buf = nullptr;     // L2 eviction buffer of snelly_flush_l2 (freed with the context)
  size_t flush_bytes = 0;

  ~Context();
  int alloc(DevBuf& b, size_t bytes);
  void release(DevBuf& b);
  int compile_module(const std::string& src, int math_mode, std::shared_ptr<Module>* out, std::string* log);
  int launch(cudaKernel_t f, int blocks, int threads, void** args);
  int upload_slot(Job& j, int slot);
  int single_job_tables(Job& j);
  int enqueue_frames(Job& j, int frames);
  int advance_batch(const std::vector<Job*>& jobs, const std::vector<int>& frames);
  void free_job(Job& j);
  // wavefront integrator (wavefront.cpp)
  int alloc_wavefront(Job& j);
  void release_wavefront(Job& j);
  int enqueue_wavefront_frames(Job& j, int frames);
  int enqueue_wavefront(const std::vector<Job*>& js, const std::vector<int>& frames,
                        const std::map<Module*, cudaEvent_t>& after, bool slot0_ready = false);
  int autotune(Job& j);
  int time_frames(Job& j, int kernel, float* ms_per_frame);
};

int assemble_scene(const std::string& glsl, const snelly_scene_opts& o, SceneSource* out);
std::string program_source(const SceneSource& ss);

// Wait for (or, with SNELLY_READ_POLL, test) the completion of a job's enqueued frames.
int wait_job(Context& c, Job& j, int flags);

}  // namespace snelly

// The opaque handle of the C ABI.
struct snelly_ctx {
  std::unique_ptr<snelly::Context> c;
};
