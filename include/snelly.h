/* snelly.h - C ABI of the B200 spectral SDF path tracer (libsnelly.so).
 *
 * This is the drop-in boundary for the reference's hot path. In the reference, the host
 * (js/renderer.js) compiles the scene's GLSL into a fragment shader (compileShaders,
 * js/renderer.js:217-359), uploads uniforms (js/renderer.js:520-611, js/materials.js syncShader
 * functions) and draws one full-screen quad per frame (js/renderer.js:613-617, the CPU->GPU
 * boundary gl.drawArrays, js/gl.js:468); readback happens through gl.readPixels
 * (js/renderer.js:455). The entry points below replace those steps:
 *
 *   snelly_create_scene   <- Renderer.compileShaders   js/renderer.js:217-359 (+ GLU.Shader js/gl.js:179)
 *   snelly_set_uniforms   <- Scene.syncShader / shader.uniform*   js/renderer.js:604-611, js/gl.js:262-408
 *   snelly_render         <- Renderer.render (uniform upload + draw, per frame)   js/renderer.js:462-673
 *   snelly_advance        <- further Renderer.render calls on an unchanged scene (progressive frames)
 *   snelly_readback       <- gl.readPixels of the radiance target   js/renderer.js:453-455
 *   snelly_cancel / snelly_destroy_job   <- Renderer.reset   js/renderer.js:191-201
 *   snelly_last_error     <- GLU.fail reporting   js/gl.js:603-626
 *
 * Conventions: 0 = success, negative = error (SNELLY_E*); the message of the last error on the
 * calling thread is returned by snelly_last_error(). Strings and arrays are copied during the
 * call; all device memory is owned by the library. Images are row-major with row 0 the bottom
 * row (gl_FragCoord / GL texture convention). No exceptions cross this boundary.
 */
#ifndef SNELLY_H
#define SNELLY_H

#include <stddef.h>
#include <stdint.h>

#include "snelly_params.h"

#ifdef __cplusplus
extern "C" {
#endif

#define SNELLY_OK 0
#define SNELLY_EINVAL (-1)        /* bad argument */
#define SNELLY_ECOMPILE (-2)      /* scene GLSL did not translate or compile (log returned) */
#define SNELLY_ENOMEM_BUDGET (-3) /* allocation refused by the HBM budget */
#define SNELLY_EBUSY (-4)         /* job not finished (POLL readback) */
#define SNELLY_ETIMEOUT (-5)      /* a bounded wait ran out */
#define SNELLY_EDEVICE (-6)       /* CUDA driver / runtime error */
#define SNELLY_ENOTFOUND (-7)     /* unknown scene / job id or uniform name */
#define SNELLY_ECANCELLED (-8)    /* job was cancelled */

typedef struct snelly_ctx snelly_ctx;

/* Kernel organisation for a scene (SNELLY_KERNEL_AUTO lets the autotuner choose). */
#define SNELLY_KERNEL_AUTO 0
#define SNELLY_KERNEL_MEGA 1      /* one thread per pixel runs the whole camera path */
#define SNELLY_KERNEL_WAVEFRONT 2 /* per-stage kernels over queues of rays in HBM */

/* Floating-point mode of the compiled scene module. */
#define SNELLY_MATH_FAST 0   /* fused multiply-add, fast transcendentals (production) */
#define SNELLY_MATH_STRICT 1 /* no contraction, IEEE div/sqrt (matches the CPU oracle closely) */

/* Compile-time options of a scene (the reference's shader defines, js/renderer.js:292-316). */
typedef struct snelly_scene_opts {
  int max_bounces;             /* __MAX_BOUNCES__ */
  int max_march_steps;         /* __MAX_MARCH_STEPS__ */
  int max_atmosphere_scatters; /* __MAX_ATMOSPHERE_SCATTERS__ */
  int max_samples_per_frame;   /* __MAX_SAMPLES_PER_FRAME__ */
  int dispersive;              /* DISPERSION_ENABLED */
  int interactive;             /* INTERACTIVE_MODE */
  int has_atmosphere;          /* HAS_ATMOSPHERE: volume scattering or absorption colour non-zero */
  int has_fog;                 /* HAS_FOG */
  int has_sphere_light;        /* HAS_SPHERE_LIGHT: sphereLightPower > -7 */
  int math_mode;               /* SNELLY_MATH_* */
  int kernel_mode;             /* SNELLY_KERNEL_* */
} snelly_scene_opts;

/* Uniform value types (GLSL types of `uniform` declarations in the scene string). */
#define SNELLY_U_FLOAT 0
#define SNELLY_U_INT 1
#define SNELLY_U_BOOL 2
#define SNELLY_U_VEC2 3
#define SNELLY_U_VEC3 4
#define SNELLY_U_VEC4 5
#define SNELLY_U_IVEC2 6
#define SNELLY_U_IVEC3 7
#define SNELLY_U_IVEC4 8
#define SNELLY_U_MAT2 9
#define SNELLY_U_MAT3 10
#define SNELLY_U_MAT4 11
#define SNELLY_U_SAMPLER2D 12
#define SNELLY_U_SAMPLER3D 13

/* One uniform assignment: `count` elements of `type` (arrays: count = array length). Float-based
 * types read `f`, int/bool types read `i`. Samplers are set with snelly_set_texture. */
typedef struct snelly_uniform {
  const char* name;
  int type;
  int count;
  const float* f;
  const int* i;
} snelly_uniform;

/* Emission spectrum sampled for the wavelength of each pixel and frame (js/spectra.js). */
#define SNELLY_SPECTRUM_BLACKBODY 0 /* BlackbodySpectrum(temperature), the reference default */
#define SNELLY_SPECTRUM_FLAT 1      /* FlatSpectrum(band_min, band_max) */
#define SNELLY_SPECTRUM_MONO 2      /* MonochromaticSpectrum(wavelength) */
typedef struct snelly_spectrum {
  int kind;
  float temperature; /* K */
  float band_min, band_max, wavelength; /* nm */
} snelly_spectrum;

/* Render modes (js/renderer.js:507-516). */
#define SNELLY_MODE_PT 0      /* spectral path tracer (pathtracer-fragment-shader.glsl) */
#define SNELLY_MODE_NORMALS 1 /* first-hit normals (normals-fragment-shader.glsl) */
#define SNELLY_MODE_AO 2      /* first-hit ambient occlusion (ao-fragment-shader.glsl) */
#define SNELLY_MODE_PICK 3    /* first-hit distance and material (pick-fragment-shader.glsl) */
#define SNELLY_MODE_PTSIMPLE 4 /* RGB surface-only path tracer (renderMode 'ptsimple',
                                  simplepathtracer-fragment-shader.glsl) */

typedef struct snelly_render_desc {
  int width, height;
  int frames;         /* progressive frames to enqueue now (each = max_samples_per_frame samples) */
  int mode;           /* SNELLY_MODE_* */
  uint64_t seed;      /* per-pixel RNG seeding */
  SnellyParams params;        /* uniform-level values; the device-pointer fields are ignored */
  snelly_spectrum spectrum;   /* emission spectrum for wavelength sampling */
  const uint8_t* env_map;     /* optional lat-long sRGB8 RGB environment, env_h rows of env_w */
  int env_w, env_h;
  int accum_fp64;     /* also accumulate in FP64 (precision study) */
  int reserved;
} snelly_render_desc;

/* Context: one per process and device. hbm_budget_bytes = 0 means "free memory minus 2 GiB". */
int snelly_init(snelly_ctx** ctx, int device, size_t hbm_budget_bytes);
int snelly_shutdown(snelly_ctx* ctx);
const char* snelly_last_error(void);
const char* snelly_version(void);

/* Compile a scene: the GLSL string a Scene.shader() returns. Missing hooks get the reference's
 * default bodies (js/renderer.js:228-263). On SNELLY_ECOMPILE the translation/NVRTC log is
 * copied into `log`. */
int snelly_create_scene(snelly_ctx* ctx, const char* scene_glsl, const snelly_scene_opts* opts,
                        uint64_t* scene_id, char* log, size_t log_cap);
int snelly_destroy_scene(snelly_ctx* ctx, uint64_t scene_id);
/* Scene uniforms, snapshotted by each subsequent snelly_render. */
int snelly_set_uniforms(snelly_ctx* ctx, uint64_t scene_id, const snelly_uniform* u, size_t n);
/* Texture for a sampler2D/sampler3D scene uniform: texel data (fmt 0 = f32, 1 = f16, 2 = u8)
 * of w x h x d texels with `channels` components, row-major, copied to the device. */
int snelly_set_texture(snelly_ctx* ctx, uint64_t scene_id, const char* name, const void* data, int w, int h,
                       int d, int channels, int fmt, int linear);

/* Start a job: allocates its per-pixel state, seeds it and enqueues desc->frames frames. Returns
 * without waiting for the frames, except that a wavefront job's frame is enqueued in pairs of
 * iterations until a progress read shows the frame complete, so the call returns roughly one
 * pair of iterations before its last frame ends. A SNELLY_KERNEL_AUTO scene's first job of a
 * module and image-size class also runs the autotuner's trial frames. */
int snelly_render(snelly_ctx* ctx, uint64_t scene_id, const snelly_render_desc* desc, uint64_t* job_id);
/* Enqueue more frames on an existing job (progressive accumulation); same timing as snelly_render. */
int snelly_advance(snelly_ctx* ctx, uint64_t job_id, int frames);

/* Replace an existing job's camera, renderer and material parameters, its emission spectrum and
 * its snapshot of the scene's uniforms (taken now from the scene, after snelly_set_uniforms /
 * snelly_set_texture) for the frames enqueued after this call; the accumulated samples and the
 * RNG state are kept. Replaces the per-frame uniform upload of Renderer.render
 * (js/renderer.js:520-611: camera, renderer, Materials.syncShader and Scene.syncShader run every
 * frame, so a preframeCallback's changes reach the next frame without a reset,
 * js/sceneAPI.js:287-358). desc->width, height and mode must equal the job's (SNELLY_EINVAL
 * otherwise: the reference resizes through a reset); desc->frames, seed, accum_fp64 and the
 * environment-map fields are ignored (the job keeps its own). The module's compile-time bounds
 * (maxBounces above the compiled value, maxMarchSteps, ...) do not change, as in the reference
 * without a recompile. Returns after the new parameters are on the device. */
int snelly_update_job(snelly_ctx* ctx, uint64_t job_id, const snelly_render_desc* desc);

/* Enqueue frames[i] more frames on each job_ids[i], batched: for every frame, the jobs that share
 * a scene module run in one launch (up to 32 jobs per launch, each with its own parameter slot),
 * and the launches of different modules go to separate streams so that they overlap on the GPU.
 * Jobs keep their per-pixel RNG streams, so each job's image is the same as when rendered alone.
 * Path-per-thread integrator. */
int snelly_advance_batch(snelly_ctx* ctx, const uint64_t* job_ids, const int* frames, size_t n);

#define SNELLY_READ_WAIT 1 /* block until the job's enqueued frames are done */
#define SNELLY_READ_POLL 2 /* return SNELLY_EBUSY if not done */
/* Enqueue the copy after the job's enqueued frames on a separate copy stream and return at once,
 * so that the copy overlaps the frames enqueued next (no reference counterpart: gl.readPixels
 * blocks). out_xyzn must stay valid until the copy is done: snelly_sync, or a later
 * SNELLY_READ_WAIT readback of the same job, returns after it; page-locked memory makes the copy
 * asynchronous. Frames enqueued afterwards write the job's mean image only once the copy is done. */
#define SNELLY_READ_ASYNC 4
/* Mean XYZ and sample count per pixel: width*height*4 floats (X, Y, Z, N). */
int snelly_readback(snelly_ctx* ctx, uint64_t job_id, float* out_xyzn, size_t bytes, int flags);
/* Mean values per pixel of a first-hit job: NORMALS and AO give mean XYZ and the frame count;
 * PICK gives (first-hit distance or maxLengthScale on a miss, material id, 0, 1) for the ray
 * through the centre of each pixel (pick-fragment-shader.glsl at every pixel). */

/* First-hit distance and material id (-1 none, 0 dielectric, 1 metal, 2 surface) along the
 * pinhole camera ray through pixel coordinate (x, y) of a desc->width x desc->height frame, in
 * gl_FragCoord units: Renderer.prototype.pick (js/renderer.js:398-461, pick-fragment-shader.glsl).
 * A miss gives maxLengthScale. desc->params supplies the camera; frames/mode are ignored.
 * Synchronous. */
int snelly_pick(snelly_ctx* ctx, uint64_t scene_id, const snelly_render_desc* desc, float x, float y, float* distance,
                float* material);
/* Complete progressive state (for checkpoint/resume): RNG lanes (4 uint32 per pixel), Kahan sums
 * and compensations (4 floats each per pixel); acc64 (4 doubles per pixel) when enabled, else
 * may be NULL. Waits for the job. */
int snelly_readback_state(snelly_ctx* ctx, uint64_t job_id, uint32_t* rng, float* acc, float* comp, double* acc64);
/* The integrator a job's frames run: SNELLY_KERNEL_MEGA or SNELLY_KERNEL_WAVEFRONT (a scene
 * created with SNELLY_KERNEL_AUTO gets the autotuner's choice for its module and image size, once
 * per size class: the wavefront's launch configuration by coordinate descent (one pass over every
 * field, a second over the pixel ranges and the extend grid's rays per lane), each
 * candidate timed over a warm-up frame and about 40 ms of frames, then the path-per-thread
 * kernel). No counterpart in the reference, which has one fragment program. */
int snelly_job_kernel(snelly_ctx* ctx, uint64_t job_id, int* kernel_mode);
/* A wavefront job's launch configuration, SNELLY_WF_CONFIG_FIELDS ints: concurrent pixel ranges,
 * per-material shade launches (0/1), drain steps before parking, sphere-tracing steps between
 * refills, work items claimed per warp, idle lanes that trigger a refill, threads per block, the
 * fraction of unfinished paths (in 1/1024) below which rays are no longer parked, subsurface
 * walks by the persistent walker (1) or one thread per walk (0), the rays an iteration may hold
 * per lane of the extend grid, whether the frames of one advance overlap (1: a path that
 * finishes its pixel's sample starts the pixel's next one; 0: frame after frame), the eighths
 * of the shade stage's resident blocks its grid may fill, whether the pixel ranges are the
 * image's rows dealt to the ranges in turn (1) or contiguous runs of rows (0), and whether
 * vertices that collide in a heterogeneous medium scatter in a stage of their own (1) or inside
 * the shade stage (0). */
#define SNELLY_WF_CONFIG_FIELDS 14
int snelly_job_wavefront_config(snelly_ctx* ctx, uint64_t job_id, int* out);
/* Start a job from saved state instead of seeding (resume). */
int snelly_restore(snelly_ctx* ctx, uint64_t scene_id, const snelly_render_desc* desc, const uint32_t* rng,
                   const float* acc, const float* comp, uint64_t* job_id);
int snelly_job_status(snelly_ctx* ctx, uint64_t job_id, int* frames_enqueued, int* frames_done);
int snelly_cancel(snelly_ctx* ctx, uint64_t job_id);
int snelly_destroy_job(snelly_ctx* ctx, uint64_t job_id);
/* Wait for all enqueued work. */
int snelly_sync(snelly_ctx* ctx);
/* The CUDA stream (cudaStream_t) the context launches on, for event timing by the caller. */
void* snelly_stream(snelly_ctx* ctx);
/* Kernel launches issued by this context so far (instrumentation). */
uint64_t snelly_launch_count(snelly_ctx* ctx);

/* Statistics of a job's image after the frames enqueued so far (waits for them): out5 = the sums
 * over pixels of the per-pixel mean X, Y, Z and of Y^2, and the total sample count. Used by the
 * serving loop's noise criterion. Deterministic (fixed-order two-pass reduction in FP64). */
int snelly_image_stats(snelly_ctx* ctx, uint64_t job_id, double* out5);

/* Measured FP32 FMA throughput of this GPU (TFLOP/s), from an FMA-chain microbenchmark; the
 * roofline denominator of the path tracer. ms_out: best kernel time of 5 runs. */
int snelly_measure_fp32_peak(snelly_ctx* ctx, double* tflops, double* ms_out);
/* Overwrite `bytes` of scratch memory on the context's stream, evicting L2 between timings. */
int snelly_flush_l2(snelly_ctx* ctx, size_t bytes);

/* The wavelength-sampling table a job uses for `s`: SNELLY_ICDF_SAMPLES (4096) floats, the inverse
 * CDF of the emission spectrum over 390..750 nm (js/spectra.js:28-61). */
int snelly_inverse_cdf(const snelly_spectrum* s, float* out);

/* snelly_image_stats without any device allocation. No counterpart in the reference (whose host
 * reads statistics back through gl.readPixels).
 * Same results as snelly_image_stats up to the summation order of the double-precision sums; for
 * callers that cannot allocate device memory at that point: a serving loop whose HBM budget is fully
 * committed to resident jobs (the budgeted allocator would refuse the scratch), and code that must
 * not call cudaFree, which synchronises the whole device. Its scratch is a fixed 160 KiB of
 * file-scope device memory per device (4096 partial records), so it handles jobs of at most
 * 4096 x 2048 = 8,388,608 pixels and returns SNELLY_EINVAL, naming the limit, for larger ones.
 * The first call through a context looks up the scratch address (cudaGetSymbolAddress, with the
 * context's device made current for the lookup) and keeps it with the context; make that first
 * call before any stream capture. After a device reset every context on that device is invalid,
 * this address included: create a new context, whose first call looks it up again. The scratch is
 * shared by every context and thread of the process on that device, so overlapping calls race;
 * calls through one context are serialised by the context. It clears its completion counter
 * before each launch and allocates nothing (no cudaMalloc, cudaFree or allocating library call). */
int snelly_image_stats_static(snelly_ctx* ctx, uint64_t job_id, double* out5);

/* Display transform of a job's mean image: shaders/tonemapper-fragment-shader.glsl as uploaded by
 * Renderer.render (js/renderer.js:619-638): XYZ -> linear sRGB, gamut shift, pow(., invGamma),
 * 2^exposure, L/(1+L), saturation, contrast, hue shift. Fields are the shader's uniforms (the
 * host passes invGamma = 1/gamma). Output row 0 is the bottom row. RGBA8: the colour-buffer
 * conversion clamp(c, 0, 1) * 255 rounded to nearest, 4 bytes per pixel; RGBA32F: the shader's
 * output colour, 16 bytes per pixel. Waits for the job's enqueued frames. */
typedef struct snelly_tonemap_params {
  float exposure, invGamma, contrast, saturation, hueShift;
} snelly_tonemap_params;
#define SNELLY_TONEMAP_RGBA8 0
#define SNELLY_TONEMAP_RGBA32F 1
int snelly_tonemap(snelly_ctx* ctx, uint64_t job_id, const snelly_tonemap_params* params, void* out, size_t bytes,
                   int format);

/* Exhaustive device self-test of the arithmetic replacement the scene kernels' random number
 * generator uses (no counterpart in the reference): which = 0 checks its integer-to-float
 * conversion and its quotients against float() and __fdiv_rn for every state of each of the four
 * lanes. *mismatches = number of differing results. */
int snelly_selftest(snelly_ctx* ctx, int which, uint64_t* mismatches);

/* Reconstruct 8-bit PNG image bytes from decompressed scanlines (each a filter-type byte and
 * width*channels filtered bytes; PNG specification section 9) into out (height*width*channels).
 * Used by the host to load environment maps (Scene.envMap, js/renderer.js:143-157) and the
 * SDF-PNG assets of scripts/pngPacker.html. No device work. */
int snelly_png_unfilter(const uint8_t* raw, size_t raw_bytes, int width, int height, int channels, uint8_t* out);

/* sizeof of the ABI structs, for bindings to check their layouts: 0 SnellyParams,
 * 1 snelly_render_desc, 2 snelly_scene_opts, 3 snelly_uniform, 4 snelly_spectrum. */
size_t snelly_abi_sizeof(int which);

/* Translate and compile a scene for sm_100a without a device (no module is loaded): a build and
 * test-time check. The NVRTC log, with the assembler's per-kernel register, spill and shared
 * memory report, goes to `log`; the cubin size to cubin_bytes. */
int snelly_compile_check(const char* scene_glsl, const snelly_scene_opts* opts, char* log, size_t log_cap,
                         size_t* cubin_bytes);

/* GLSL -> C++ translation of a scene string (what snelly_create_scene compiles), for tools that
 * build CPU code from the same source. extra_members: C++ member declarations to add to the
 * struct (NULL: the scene defaults, i.e. the reference's rand()). Writes the C++ text into out
 * (NUL-terminated). */
int snelly_glsl_to_cpp(const char* glsl, const char* struct_name, const char* extra_members, char* out,
                       size_t out_cap);

#ifdef __cplusplus
}
#endif
#endif /* SNELLY_H */
