// runtime.cpp - libsnelly: the C ABI of include/snelly.h.
//
// Owns the CUDA context use (primary context of one device), one launch stream, the NVRTC
// module cache (one module per scene source + compile-time options), scenes, jobs and their
// device buffers, and an HBM budget that every allocation is checked against.
#include <cuda_runtime.h>
#include <dirent.h>
#include <dlfcn.h>
#include <nvrtc.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "glsl_transform.h"
#include "kernels/pt_launch.h"
#include "runtime_internal.h"
#include "snelly.h"
#include "spectrum.h"

namespace snelly {

thread_local std::string t_last_error;

int fail(int code, const std::string& msg) {
  t_last_error = msg;
  return code;
}

static const float kXyzTable[4 * SNELLY_XYZ_SAMPLES] = {
#include "cie_xyz_table.inc"
};

// ---- device buffers under the context's HBM budget --------------------------------------------
int Context::alloc(DevBuf& b, size_t bytes) {
  b.bytes = 0;
  b.ptr = nullptr;
  if (bytes == 0) return SNELLY_OK;
  if (used + bytes > budget)
    return fail(SNELLY_ENOMEM_BUDGET, "HBM budget exceeded: need " + std::to_string(bytes) + " bytes, " +
                                          std::to_string(budget - used) + " left");
  cudaError_t e = cudaMalloc(&b.ptr, bytes);
  if (e != cudaSuccess) {
    b.ptr = nullptr;
    return fail(SNELLY_EDEVICE, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  b.bytes = bytes;
  used += bytes;
  return SNELLY_OK;
}

void Context::release(DevBuf& b) {
  if (b.ptr) {
    cudaFree(b.ptr);
    used -= b.bytes;
  }
  b.ptr = nullptr;
  b.bytes = 0;
}

// ---- locating the kernel sources ---------------------------------------------------------------
static std::string library_dir() {
  Dl_info info;
  if (dladdr((void*)&library_dir, &info) && info.dli_fname) {
    std::string p = info.dli_fname;
    size_t s = p.rfind('/');
    if (s != std::string::npos) return p.substr(0, s);
  }
  return ".";
}

static bool file_exists(const std::string& p) {
  struct stat st;
  return stat(p.c_str(), &st) == 0;
}

// ---- scene assembly (js/renderer.js:217-316) ---------------------------------------------------
// Hook defaults: identity functions with the reference's signatures, appended when the scene
// string does not mention the hook name.
struct HookDefault {
  const char* needle;
  const char* body;
};
static const HookDefault kHookDefaults[] = {
    {"INIT(", "void INIT() {}"},
    {"SURFACE_DIFFUSE_REFLECTANCE(", "vec3 SURFACE_DIFFUSE_REFLECTANCE(in vec3 C, in vec3 X, in vec3 N, in vec3 V) { return C; }"},
    {"SURFACE_SPECULAR_REFLECTANCE(", "vec3 SURFACE_SPECULAR_REFLECTANCE(in vec3 C, in vec3 X, in vec3 N, in vec3 V) { return C; }"},
    {"SURFACE_ROUGHNESS(", "float SURFACE_ROUGHNESS(in float roughness, in vec3 X, in vec3 N) { return roughness; }"},
    {"SUBSURFACE_ALBEDO(", "vec3 SUBSURFACE_ALBEDO(in vec3 C, in vec3 X, in vec3 N) { return C; }"},
    {"METAL_SPECULAR_REFLECTANCE(", "vec3 METAL_SPECULAR_REFLECTANCE(in vec3 C, in vec3 X, in vec3 N, in vec3 V) { return C; }"},
    {"METAL_ROUGHNESS(", "float METAL_ROUGHNESS(in float roughness, in vec3 X, in vec3 N) { return roughness; }"},
    {"DIELECTRIC_SPECULAR_REFLECTANCE(", "vec3 DIELECTRIC_SPECULAR_REFLECTANCE(in vec3 C, in vec3 X, in vec3 N, in vec3 V) { return C; }"},
    {"DIELECTRIC_ROUGHNESS(", "float DIELECTRIC_ROUGHNESS(in float roughness, in vec3 X, in vec3 N) { return roughness; }"},
    {"DIELECTRIC_ABSORPTION(", "vec3 DIELECTRIC_ABSORPTION(vec3 absorption_ui, vec3 X) { return absorption_ui; }"},
    {"VOLUME_EXTINCTION(", "float VOLUME_EXTINCTION(float extinction_ui, vec3 X) { return extinction_ui; }"},
    {"VOLUME_EXTINCTION_MAX(", "float VOLUME_EXTINCTION_MAX(float extinction_ui) { return extinction_ui; }"},
    {"VOLUME_SCATTERING_COLOR(", "vec3 VOLUME_SCATTERING_COLOR(vec3 scattering_color_ui, vec3 X) { return scattering_color_ui; }"},
    {"VOLUME_ABSORPTION_COLOR(", "vec3 VOLUME_ABSORPTION_COLOR(vec3 absorption_color_ui, vec3 X) { return absorption_color_ui; }"},
    {"VOLUME_ANISOTROPY(", "float VOLUME_ANISOTROPY(float anisotropy, vec3 X) { return anisotropy; }"},
    {"VOLUME_EMISSION(", "vec3 VOLUME_EMISSION(vec3 emission, vec3 X) { return emission; }"},
};

// The reference's float RNG (PT:119-130), made available to scene hooks that call rand(rnd).
static const char* kSceneExtraMembers = R"(
  gfloat rand(vec4& rnd) {
    const vec4 q = vec4(1225.0f, 1585.0f, 2457.0f, 2098.0f);
    const vec4 r = vec4(1112.0f, 367.0f, 92.0f, 265.0f);
    const vec4 a = vec4(3423.0f, 2646.0f, 1707.0f, 1999.0f);
    const vec4 m = vec4(4194287.0f, 4194277.0f, 4194191.0f, 4194167.0f);
    vec4 beta = floor(rnd / q);
    vec4 p = a * (rnd - beta * q) - beta * r;
    beta = (1.0f - sign(p)) * 0.5f * m;
    rnd = p + beta;
    return fract(dot(rnd / m, vec4(1.0f, -1.0f, 1.0f, -1.0f)));
  }
)";

int assemble_scene(const std::string& glsl, const snelly_scene_opts& o, SceneSource* out) {
  std::string s = glsl;
  auto has = [&](const char* needle) { return s.find(needle) != std::string::npos; };
  SceneSource r;
  r.has_custom_camera = glsl.find("CONSTRUCT_PRIMARY_RAY(") != std::string::npos;
  r.has_surface = glsl.find("SDF_SURFACE(") != std::string::npos;
  r.has_metal = glsl.find("SDF_METAL(") != std::string::npos;
  r.has_dielectric = glsl.find("SDF_DIELECTRIC(") != std::string::npos;
  r.has_surface_nm = glsl.find("SURFACE_NORMAL_MAP(") != std::string::npos;
  r.has_metal_nm = glsl.find("METAL_NORMAL_MAP(") != std::string::npos;
  r.has_dielectric_nm = glsl.find("DIELECTRIC_NORMAL_MAP(") != std::string::npos;
  r.has_volume_emission = glsl.find("VOLUME_EMISSION(") != std::string::npos;
  for (const HookDefault& h : kHookDefaults)
    if (!has(h.needle)) s += std::string("\n ") + h.body + "\n";
  if (!(r.has_surface || r.has_metal || r.has_dielectric))
    return fail(SNELLY_ECOMPILE, "Scene must define at least one of: SDF_SURFACE, SDF_METAL, SDF_DIELECTRIC");
  std::ostringstream d;
  if (r.has_custom_camera) d << "#define HAS_CUSTOM_CAMERA\n";
  if (r.has_surface) d << "#define HAS_SURFACE\n";
  if (r.has_metal) d << "#define HAS_METAL\n";
  if (r.has_dielectric) d << "#define HAS_DIELECTRIC\n";
  // A scene that defines VOLUME_EXTINCTION itself has a heterogeneous medium in the atmosphere's
  // box (an extension of this build: the reference declares the hook but never calls it), which
  // takes the place of the homogeneous atmosphere.
  const bool hetero = glsl.find("VOLUME_EXTINCTION(") != std::string::npos;
  if (hetero) d << "#define HAS_HETERO_VOLUME\n";
  else if (o.has_atmosphere) d << "#define HAS_ATMOSPHERE\n";
  if (o.has_fog) d << "#define HAS_FOG\n";
  if (r.has_volume_emission) d << "#define HAS_VOLUME_EMISSION\n";
  d << "#define HAS_GEOMETRY\n";
  if (r.has_surface_nm || r.has_metal_nm || r.has_dielectric_nm) d << "#define HAS_NORMALMAP\n";
  if (r.has_surface_nm) d << "#define HAS_SURFACE_NORMALMAP\n";
  if (r.has_metal_nm) d << "#define HAS_METAL_NORMALMAP\n";
  if (r.has_dielectric_nm) d << "#define HAS_DIELECTRIC_NORMALMAP\n";
  if (o.interactive) d << "#define INTERACTIVE_MODE\n";
  if (o.dispersive) d << "#define DISPERSION_ENABLED\n";
  if (o.has_sphere_light) d << "#define HAS_SPHERE_LIGHT\n";
  d << "#define MAX_MARCH_STEPS " << o.max_march_steps << "\n";
  d << "#define MAX_BOUNCES " << o.max_bounces << "\n";
  d << "#define MAX_ATMOSPHERE_SCATTERS " << o.max_atmosphere_scatters << "\n";
  d << "#define MAX_SAMPLES_PER_FRAME " << o.max_samples_per_frame << "\n";
  r.defines = d.str();
  r.glsl = s;
  if (!glsl_transform(s, "Scene", kSceneExtraMembers, &r.xf))
    return fail(SNELLY_ECOMPILE, "GLSL translation failed: " + r.xf.error);
  *out = r;
  return SNELLY_OK;
}

std::string program_source(const SceneSource& ss) {
  std::ostringstream p;
  p << "// generated by libsnelly: scene module\n" << ss.defines << "#include \"glslcompat.h\"\nnamespace glsl {\n"
    << ss.xf.code << "\n}  // namespace glsl\n#include \"pt_kernels.cu\"\n";
  return p.str();
}

// ---- NVRTC ----------------------------------------------------------------------------------------
static std::string hex64(uint64_t v) {
  char b[17];
  snprintf(b, sizeof b, "%016llx", (unsigned long long)v);
  return b;
}
static uint64_t fnv1a(const std::string& s, uint64_t h = 1469598103934665603ull) {
  for (unsigned char c : s) {
    h ^= c;
    h *= 1099511628211ull;
  }
  return h;
}

static std::vector<std::string> nvrtc_options(const std::string& kernel_dir, const std::string& csrc_dir,
                                              const std::string& include_dir, int math_mode) {
  // --ptxas-options=-v: the log lists registers, spills and shared memory per kernel
  std::vector<std::string> opts = {"--gpu-architecture=sm_100a", "-std=c++17", "-default-device", "-lineinfo",
                                   "-diag-suppress=550,177", "--ptxas-options=-v", "-I" + kernel_dir, "-I" + csrc_dir,
                                   "-I" + include_dir};
  if (math_mode == SNELLY_MATH_STRICT) {
    opts.push_back("--fmad=false");
    opts.push_back("--prec-div=true");
    opts.push_back("--prec-sqrt=true");
    opts.push_back("--ftz=false");
  } else {
    opts.push_back("--use_fast_math");
  }
  // extra compiler options, space-separated (e.g. -DWF_CHUNK=4 or --ptxas-options=-v); they are
  // part of the module cache key
  if (const char* x = getenv("SNELLY_NVRTC_EXTRA")) {
    std::istringstream in(x);
    std::string o;
    while (in >> o) opts.push_back(o);
  }
  return opts;
}

// NVRTC compile of a scene module to an sm_100a cubin.
static int nvrtc_cubin(const std::string& src, const std::vector<std::string>& opts, std::vector<char>* cubin,
                       std::string* log) {
  nvrtcProgram prog;
  if (nvrtcCreateProgram(&prog, src.c_str(), "scene_module.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS)
    return fail(SNELLY_ECOMPILE, "nvrtcCreateProgram failed");
  std::vector<const char*> copts;
  for (auto& o : opts) copts.push_back(o.c_str());
  nvrtcResult rc = nvrtcCompileProgram(prog, (int)copts.size(), copts.data());
  size_t lsz = 0;
  nvrtcGetProgramLogSize(prog, &lsz);
  std::string lg(lsz, '\0');
  if (lsz) nvrtcGetProgramLog(prog, &lg[0]);
  if (log) *log = lg;
  if (rc != NVRTC_SUCCESS) {
    nvrtcDestroyProgram(&prog);
    return fail(SNELLY_ECOMPILE, std::string("NVRTC: ") + nvrtcGetErrorString(rc) + "\n" + lg);
  }
  size_t csz = 0;
  nvrtcGetCUBINSize(prog, &csz);
  cubin->resize(csz);
  nvrtcGetCUBIN(prog, cubin->data());
  nvrtcDestroyProgram(&prog);
  return SNELLY_OK;
}

static std::string read_file(const std::string& path) {
  std::ifstream in(path);
  std::stringstream ss;
  ss << in.rdbuf();
  return ss.str();
}

// Cache key of a module: its program source, the compiler options but the include paths, every source file the program
// includes (all of the kernel directory, the GLSL compatibility header and its swizzle table, the
// parameter block) and the NVRTC version.
static std::string module_key(const std::string& src, const std::vector<std::string>& opts,
                              const std::string& kernel_dir, const std::string& csrc_dir,
                              const std::string& include_dir) {
  std::string key_text = src;
  for (auto& o : opts)  // include paths differ between machines; the files they hold are hashed below
    if (o.compare(0, 2, "-I") != 0) key_text += "\n" + o;
  std::vector<std::string> kfiles;
  if (DIR* d = opendir(kernel_dir.c_str())) {
    while (dirent* e = readdir(d))
      if (e->d_name[0] != '.') kfiles.push_back(e->d_name);
    closedir(d);
  }
  std::sort(kfiles.begin(), kfiles.end());
  for (auto& f : kfiles) key_text += "\n//" + f + "\n" + read_file(kernel_dir + "/" + f);
  key_text += read_file(csrc_dir + "/glslcompat.h") + read_file(csrc_dir + "/glsl_swizzles.inc") +
              read_file(include_dir + "/snelly_params.h");
  int nv_major = 0, nv_minor = 0;
  nvrtcVersion(&nv_major, &nv_minor);
  key_text += "\nnvrtc " + std::to_string(nv_major) + "." + std::to_string(nv_minor);
  return hex64(fnv1a(key_text));
}

// Store a compiled module under its key: written whole to a temporary file, then renamed.
static void cache_store(const std::string& cache_path, const std::vector<char>& cubin) {
  if (cache_path.empty()) return;
  std::string tmp = cache_path + ".tmp" + std::to_string((long)getpid());
  std::ofstream o(tmp, std::ios::binary);
  o.write(cubin.data(), (std::streamsize)cubin.size());
  o.close();
  if (o.good()) rename(tmp.c_str(), cache_path.c_str());
  else unlink(tmp.c_str());
}

int Context::compile_module(const std::string& src, int math_mode, std::shared_ptr<Module>* out, std::string* log) {
  std::vector<std::string> opts = nvrtc_options(kernel_dir, csrc_dir, include_dir, math_mode);
  const std::string key = module_key(src, opts, kernel_dir, csrc_dir, include_dir);
  auto it = module_cache.find(key);
  if (it != module_cache.end()) {
    *out = it->second;
    return SNELLY_OK;
  }
  std::vector<char> cubin;
  std::string cache_path = cache_dir.empty() ? "" : cache_dir + "/" + key + ".cubin";
  bool from_cache = false;
  if (!cache_path.empty() && file_exists(cache_path)) {
    std::ifstream in(cache_path, std::ios::binary);
    cubin.assign(std::istreambuf_iterator<char>(in), std::istreambuf_iterator<char>());
    from_cache = !cubin.empty();
  }
  auto m = std::make_shared<Module>();
  m->key = key;
  for (int attempt = 0;; ++attempt) {
    if (cubin.empty()) {
      int rc = nvrtc_cubin(src, opts, &cubin, log);
      if (rc) return rc;
      from_cache = false;
      cache_store(cache_path, cubin);
    }
    cudaError_t lr = cudaLibraryLoadData(&m->lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
    if (lr == cudaSuccess) break;
    cudaGetLastError();
    if (!from_cache || attempt > 0)
      return fail(SNELLY_EDEVICE, std::string("cudaLibraryLoadData: ") + cudaGetErrorString(lr));
    unlink(cache_path.c_str());  // an unusable cached cubin (truncated, or from another build): compile again
    cubin.clear();
  }
  struct Fn {
    const char* name;
    cudaKernel_t* f;
    bool required;
  } fns[] = {{"snelly_seed", &m->f_seed, true},
             {"snelly_frame_mega", &m->f_frame_mega, true},
             {"snelly_resolve", &m->f_resolve, true},
             {"snelly_wf_generate", &m->f_wf_generate, false},
             {"snelly_wf_extend", &m->f_wf_extend, false},
             {"snelly_wf_shade", &m->f_wf_shade, false},
             {"snelly_wf_shade_miss", &m->f_wf_shade_seg[0], false},
             {"snelly_wf_shade_surface", &m->f_wf_shade_seg[1], false},
             {"snelly_wf_shade_metal", &m->f_wf_shade_seg[2], false},
             {"snelly_wf_shade_dielectric", &m->f_wf_shade_seg[3], false},
             {"snelly_wf_sss", &m->f_wf_sss, false},
             {"snelly_wf_walk", &m->f_wf_walk, false},
             {"snelly_wf_walk_exit", &m->f_wf_walk_exit, false},
             {"snelly_wf_volume", &m->f_wf_volume, false},
             {"snelly_firsthit", &m->f_firsthit, false},
             {"snelly_ptsimple", &m->f_ptsimple, false}};
  for (auto& f : fns) {
    cudaError_t r = cudaLibraryGetKernel(f.f, m->lib, f.name);
    if (r != cudaSuccess) {
      cudaGetLastError();
      *f.f = nullptr;
      if (f.required) return fail(SNELLY_ECOMPILE, std::string("kernel missing from module: ") + f.name);
    }
  }
  if (m->f_wf_extend) {  // the extend stage is persistent: one wave of resident blocks
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, (const void*)m->f_wf_extend, SNELLY_BLOCK, 0) == cudaSuccess &&
        nb > 0)
      m->extend_blocks_per_sm = nb;
    else
      cudaGetLastError();
    nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, (const void*)m->f_wf_extend, 64, 0) == cudaSuccess && nb > 0)
      m->extend_blocks_per_sm64 = nb;
    else
      cudaGetLastError();
  }
  if (m->f_wf_walk) {  // the walker is persistent too: one resident wave
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, (const void*)m->f_wf_walk, SNELLY_BLOCK, 0) == cudaSuccess && nb > 0)
      m->walk_blocks_per_sm = nb;
    else
      cudaGetLastError();
  }
  if (m->f_wf_shade) {  // one resident wave of the shade stage's grid-stride loop
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, (const void*)m->f_wf_shade, SNELLY_BLOCK, 0) == cudaSuccess &&
        nb > 0)
      m->shade_blocks_per_sm = nb;
    else
      cudaGetLastError();
  }
  size_t sz = 0;
  if (m->f_wf_generate) {  // the path-record size the wavefront kernels were compiled for
    int* rp = nullptr;
    RT_TRY(cudaLibraryGetGlobal((void**)&rp, &sz, m->lib, "snelly_wf_rec_f4"));
    RT_TRY(cudaMemcpy(&m->wf_rec_f4, rp, sizeof(int), cudaMemcpyDeviceToHost));
  }
  RT_TRY(cudaLibraryGetGlobal((void**)&m->c_params, &sz, m->lib, "c_params"));
  RT_TRY(cudaLibraryGetGlobal((void**)&m->c_uniforms, &m->c_uniforms_bytes, m->lib, "c_uniforms"));
  m->slot_uniform_bytes = m->c_uniforms_bytes / SNELLY_MAX_BATCH;
  module_cache[key] = m;
  *out = m;
  return SNELLY_OK;
}

// ---- launches --------------------------------------------------------------------------------------
int Context::launch(cudaKernel_t f, int blocks, int threads, void** args) {
  if (blocks <= 0) return SNELLY_OK;
  RT_TRY(cudaLaunchKernel((const void*)f, dim3((unsigned)blocks), dim3((unsigned)threads), args, 0, stream));
  launches++;
  return SNELLY_OK;
}

// Upload a job's parameter and uniform blocks into constant-memory slot `slot` of its module.
int Context::upload_slot(Job& j, int slot) {
  Module& m = *j.module;
  RT_TRY(cudaMemcpyAsync(m.c_params + slot * sizeof(SnellyParams), &j.params, sizeof(SnellyParams),
                         cudaMemcpyHostToDevice, stream));
  size_t ub = std::min(j.ublock.size(), m.slot_uniform_bytes);
  if (ub)
    RT_TRY(cudaMemcpyAsync(m.c_uniforms + slot * m.slot_uniform_bytes, j.ublock.data(), ub, cudaMemcpyHostToDevice,
                           stream));
  return SNELLY_OK;
}

// Job record + block table for a single-job launch over all pixels.
int Context::single_job_tables(Job& j) {
  JobRec r{};
  r.rng = (uint4*)j.rng.ptr;
  r.acc = (float4*)j.acc.ptr;
  r.comp = (float4*)j.comp.ptr;
  r.acc64 = (double*)j.acc64.ptr;
  r.out = (float4*)j.out.ptr;
  r.seed = j.desc.seed;
  r.width = j.desc.width;
  r.height = j.desc.height;
  r.pixel_begin = 0;
  r.pixel_count = j.desc.width * j.desc.height;
  r.slot = 0;
  r.mode = j.desc.mode;
  r.pick_at = j.pick_at;
  r.pick_x = j.pick_x;
  r.pick_y = j.pick_y;
  int bs[2] = {0, (r.pixel_count + SNELLY_BLOCK - 1) / SNELLY_BLOCK};
  RT_TRY(cudaMemcpyAsync(j.tables.ptr, &r, sizeof r, cudaMemcpyHostToDevice, stream));
  RT_TRY(cudaMemcpyAsync((char*)j.tables.ptr + 128, bs, sizeof bs, cudaMemcpyHostToDevice, stream));
  j.blocks = bs[1];
  return SNELLY_OK;
}

int Context::enqueue_frames(Job& j, int frames) {
  if (frames <= 0) return SNELLY_OK;
  Module& m = *j.module;
  int rc = upload_slot(j, 0);
  if (rc) return rc;
  void* tables = j.tables.ptr;
  void* bstart = (char*)j.tables.ptr + 128;
  int njobs = 1;
  void* gparams = j.gparams.ptr;
  void* args[] = {&tables, &bstart, &njobs, &gparams};
  const bool wavefront = j.desc.mode == SNELLY_MODE_PT && j.kernel_mode == SNELLY_KERNEL_WAVEFRONT && m.f_wf_generate;
  if (wavefront && (rc = enqueue_wavefront_frames(j, frames))) return rc;  // every frame, pipelined by pixel range
  for (int f = 0; f < frames && !wavefront; ++f) {
    if (j.desc.mode == SNELLY_MODE_PT) {
      rc = launch(m.f_frame_mega, j.blocks, SNELLY_BLOCK, args);
    } else if (j.desc.mode == SNELLY_MODE_PTSIMPLE) {
      if (!m.f_ptsimple) return fail(SNELLY_EINVAL, "the simplified path tracer is not available in this module");
      rc = launch(m.f_ptsimple, j.blocks, SNELLY_BLOCK, args);
    } else {
      if (!m.f_firsthit) return fail(SNELLY_EINVAL, "first-hit render modes are not available in this module");
      rc = launch(m.f_firsthit, j.blocks, SNELLY_BLOCK, args);
    }
    if (rc) return rc;
  }
  void* rargs[] = {&tables, &bstart, &njobs};
  if (j.read_pending) RT_TRY(cudaStreamWaitEvent(stream, j.read_done, 0));  // `out` is being copied out
  rc = launch(m.f_resolve, j.blocks, SNELLY_BLOCK, rargs);
  if (rc) return rc;
  j.frames_enqueued += frames;
  RT_TRY(cudaEventRecord(j.done, stream));
  return SNELLY_OK;
}

// Batched frames (see snelly_advance_batch). Jobs the autotuner gave the wavefront run as pixel
// ranges on their own streams, all of them at once (enqueue_wavefront). The others are grouped by
// module; each group gets a lane (stream + device tables); per frame, one path-per-thread launch
// covers the group's jobs that still need frames. Lanes and wavefront ranges run concurrently; a
// module's wavefront jobs take over its constant-memory slots after its lane is done.
int Context::advance_batch(const std::vector<Job*>& js, const std::vector<int>& frames) {
  std::map<Module*, std::vector<size_t>> groups;
  std::vector<Job*> wjobs;
  std::vector<int> wframes;
  for (size_t k = 0; k < js.size(); ++k) {
    if (frames[k] <= 0) continue;
    Job& j = *js[k];
    if (j.desc.mode == SNELLY_MODE_PT && j.kernel_mode == SNELLY_KERNEL_WAVEFRONT && j.module->f_wf_generate) {
      wjobs.push_back(&j);
      wframes.push_back(frames[k]);
    } else {
      groups[j.module].push_back(k);
    }
  }
  // all earlier work on the main stream (job seeding, single-job frames) comes first
  cudaEvent_t start;
  RT_TRY(cudaEventCreateWithFlags(&start, cudaEventDisableTiming));
  RT_TRY(cudaEventRecord(start, stream));
  size_t lane_idx = 0;
  std::map<Module*, cudaEvent_t> after;
  for (auto& g : groups) {
    Module& m = *g.first;
    std::vector<size_t>& idx = g.second;
    // one lane per module: its constant-memory slots are reused chunk after chunk, in order
    for (size_t c0 = 0; c0 < idx.size(); c0 += SNELLY_MAX_BATCH) {
      if (lane_idx >= lanes.size()) {
        BatchLane L;
        RT_TRY(cudaStreamCreateWithFlags(&L.stream, cudaStreamNonBlocking));
        RT_TRY(cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming));
        int rc = alloc(L.recs, SNELLY_MAX_BATCH * sizeof(JobRec) + 4 * (SNELLY_MAX_BATCH + 1) + 256);
        if (!rc) rc = alloc(L.gparams, SNELLY_MAX_BATCH * sizeof(SnellyParams));
        if (rc) return rc;
        lanes.push_back(L);
      }
      BatchLane& L = lanes[lane_idx];
      if (c0 == 0) RT_TRY(cudaStreamWaitEvent(L.stream, start, 0));
      size_t c1 = std::min(idx.size(), c0 + SNELLY_MAX_BATCH);
      int maxf = 0;
      for (size_t q = c0; q < c1; ++q) maxf = std::max(maxf, frames[idx[q]]);
      // parameter slots: one per job of the chunk
      for (size_t q = c0; q < c1; ++q) {
        Job& j = *js[idx[q]];
        int slot = (int)(q - c0);
        RT_TRY(cudaMemcpyAsync(m.c_params + slot * sizeof(SnellyParams), &j.params, sizeof(SnellyParams),
                               cudaMemcpyHostToDevice, L.stream));
        size_t ub = std::min(j.ublock.size(), m.slot_uniform_bytes);
        if (ub)
          RT_TRY(cudaMemcpyAsync(m.c_uniforms + slot * m.slot_uniform_bytes, j.ublock.data(), ub,
                                 cudaMemcpyHostToDevice, L.stream));
        RT_TRY(cudaMemcpyAsync((char*)L.gparams.ptr + slot * sizeof(SnellyParams), &j.params, sizeof(SnellyParams),
                               cudaMemcpyHostToDevice, L.stream));
      }
      for (int f = 0; f < maxf; ++f) {
        std::vector<JobRec> recs;
        std::vector<int> bs(1, 0);
        for (size_t q = c0; q < c1; ++q) {
          Job& j = *js[idx[q]];
          if (frames[idx[q]] <= f) continue;
          JobRec r{};
          r.rng = (uint4*)j.rng.ptr;
          r.acc = (float4*)j.acc.ptr;
          r.comp = (float4*)j.comp.ptr;
          r.acc64 = (double*)j.acc64.ptr;
          r.out = (float4*)j.out.ptr;
          r.seed = j.desc.seed;
          r.width = j.desc.width;
          r.height = j.desc.height;
          r.pixel_begin = 0;
          r.pixel_count = j.desc.width * j.desc.height;
          r.slot = (int)(q - c0);
          r.mode = j.desc.mode;
          recs.push_back(r);
          bs.push_back(bs.back() + (r.pixel_count + SNELLY_BLOCK - 1) / SNELLY_BLOCK);
        }
        // the tables are rewritten for every frame: the copy is ordered after the previous launch
        RT_TRY(cudaMemcpyAsync(L.recs.ptr, recs.data(), recs.size() * sizeof(JobRec), cudaMemcpyHostToDevice, L.stream));
        char* bsp = (char*)L.recs.ptr + SNELLY_MAX_BATCH * sizeof(JobRec);
        RT_TRY(cudaMemcpyAsync(bsp, bs.data(), bs.size() * sizeof(int), cudaMemcpyHostToDevice, L.stream));
        void* recp = L.recs.ptr;
        void* bsv = bsp;
        int nj = (int)recs.size();
        void* gp = L.gparams.ptr;
        void* args[] = {&recp, &bsv, &nj, &gp};
        RT_TRY(cudaLaunchKernel((const void*)m.f_frame_mega, dim3((unsigned)bs.back()), dim3(SNELLY_BLOCK), args, 0,
                                L.stream));
        launches++;
      }
      // resolve each job once at the end of the batch (single-job launches on the lane)
      for (size_t q = c0; q < c1; ++q) {
        Job& j = *js[idx[q]];
        void* tables = j.tables.ptr;
        void* bstart = (char*)j.tables.ptr + 128;
        int one = 1;
        void* rargs[] = {&tables, &bstart, &one};
        if (j.read_pending) RT_TRY(cudaStreamWaitEvent(L.stream, j.read_done, 0));  // `out` is being copied out
        RT_TRY(cudaLaunchKernel((const void*)m.f_resolve, dim3((unsigned)j.blocks), dim3(SNELLY_BLOCK), rargs, 0,
                                L.stream));
        launches++;
        j.frames_enqueued += frames[idx[q]];
      }
    }
    BatchLane& L = lanes[lane_idx];
    RT_TRY(cudaEventRecord(L.done, L.stream));
    after[&m] = L.done;
    ++lane_idx;
  }
  // the wavefront jobs, overlapping the lanes (a module's after its lane, for the slots)
  int rc = enqueue_wavefront(wjobs, wframes, after);
  if (rc) {
    cudaEventDestroy(start);
    return rc;
  }
  for (size_t l = 0; l < lane_idx; ++l) RT_TRY(cudaStreamWaitEvent(stream, lanes[l].done, 0));
  for (size_t q = 0; q < wjobs.size(); ++q) {  // each wavefront job's mean image
    Job& j = *wjobs[q];
    void* tables = j.tables.ptr;
    void* bstart = (char*)j.tables.ptr + 128;
    int one = 1;
    void* rargs[] = {&tables, &bstart, &one};
    if (j.read_pending) RT_TRY(cudaStreamWaitEvent(stream, j.read_done, 0));  // `out` is being copied out
    if ((rc = launch(j.module->f_resolve, j.blocks, SNELLY_BLOCK, rargs))) {
      cudaEventDestroy(start);
      return rc;
    }
    j.frames_enqueued += wframes[q];
  }
  // later main-stream work (and every job's completion event) is ordered after all of it
  for (size_t k = 0; k < js.size(); ++k) RT_TRY(cudaEventRecord(js[k]->done, stream));
  cudaEventDestroy(start);
  return SNELLY_OK;
}

Context::~Context() {
  cudaStreamSynchronize(stream);
  for (auto& L : lanes) {
    cudaStreamSynchronize(L.stream);
    release(L.recs);
    release(L.gparams);
    cudaEventDestroy(L.done);
    cudaStreamDestroy(L.stream);
  }
  for (auto& kv : jobs) free_job(kv.second);
  for (auto& kv : scenes) {
    for (auto& t : kv.second.textures) release(t.second);
    for (auto& t : kv.second.retired_textures) release(t);
  }
  if (copy_stream) cudaStreamSynchronize(copy_stream);
  release(xyz);
  release(stats_scratch);
  if (flush_buf) cudaFree(flush_buf);
  if (poll_host) cudaFreeHost(poll_host);
  for (auto& e : wf_events) cudaEventDestroy(e);
  for (auto& st : wf_pool) {
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
  if (wf_fork) cudaEventDestroy(wf_fork);
  for (auto& kv : module_cache) cudaLibraryUnload(kv.second->lib);
  if (copy_stream) cudaStreamDestroy(copy_stream);
  cudaStreamDestroy(stream);
}

void Context::free_job(Job& j) {
  if (j.read_done) {  // an asynchronous readback may still be copying `out`
    cudaEventSynchronize(j.read_done);
    cudaEventDestroy(j.read_done);
    j.read_done = nullptr;
    j.read_pending = false;
  }
  release(j.rng);
  release(j.acc);
  release(j.comp);
  release(j.acc64);
  release(j.out);
  release(j.icdf);
  release(j.env);
  release(j.gparams);
  release(j.tables);
  release(j.display);
  release_wavefront(j);
  if (j.done) cudaEventDestroy(j.done);
  j.done = nullptr;
}

}  // namespace snelly

using namespace snelly;

extern "C" {

const char* snelly_last_error(void) { return t_last_error.c_str(); }
const char* snelly_version(void) { return "snelly-b200 0.1.0 (sm_100a)"; }

int snelly_init(snelly_ctx** out, int device, size_t budget) {
  if (!out) return fail(SNELLY_EINVAL, "ctx pointer is null");
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) return fail(SNELLY_EDEVICE, "no CUDA device available");
  if (device < 0 || device >= n) return fail(SNELLY_EINVAL, "device index out of range");
  RT_TRY(cudaSetDevice(device));
  RT_TRY(cudaFree(0));  // create / retain the primary context
  cudaDeviceProp prop;
  RT_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) return fail(SNELLY_EDEVICE, "libsnelly requires an sm_100 (Blackwell) GPU");
  auto c = std::make_unique<Context>();
  c->device = device;
  c->sm_count = prop.multiProcessorCount;
  RT_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  size_t freeb = 0, total = 0;
  RT_TRY(cudaMemGetInfo(&freeb, &total));
  size_t reserve = size_t(2) << 30;
  c->budget = budget ? budget : (freeb > reserve ? freeb - reserve : freeb / 2);
  std::string dir = library_dir();
  const char* env = getenv("SNELLY_KERNEL_DIR");
  c->csrc_dir = env ? std::string(env) : dir + "/csrc";
  c->kernel_dir = c->csrc_dir + "/kernels";
  c->include_dir = env ? std::string(env) + "/../../include" : dir + "/../include";
  if (!file_exists(c->kernel_dir + "/pt_kernels.cu"))
    return fail(SNELLY_EINVAL, "kernel sources not found under " + c->kernel_dir);
  if (const char* pi = getenv("SNELLY_WF_PARK_ITERS")) c->wf_park_iters = atoi(pi);
  if (const char* pd = getenv("SNELLY_WF_PDL")) c->wf_pdl = atoi(pd) ? 1 : 0;
  {  // wavefront defaults from the environment; those given are not tuned
    WfConfig& d = c->wf_default;
    struct {
      const char* name;
      int* field;
      int lo, hi;
    } knobs[] = {{"SNELLY_WF_SPLIT", &d.parts, 1, SNELLY_WF_MAX_PARTS}, {"SNELLY_WF_SHADE_SPLIT", &d.shade_split, 0, 1},
                 {"SNELLY_WF_DRAIN", &d.drain, 0, 4096},  // 0: never park rays
                 {"SNELLY_WF_CHUNK", &d.chunk, 1, 64}, {"SNELLY_WF_GRAB", &d.grab, 1, 1024},
                 {"SNELLY_WF_REFILL", &d.refill, 1, 32}, {"SNELLY_WF_BLOCK", &d.block, 64, 128},
                 {"SNELLY_WF_PARK_LEFT", &d.park_left, 0, 1024}, {"SNELLY_WF_WALKER", &d.walker, 0, 1},
                 {"SNELLY_WF_LANE_RAYS", &d.lane_rays, 1, 64}, {"SNELLY_WF_OVERLAP", &d.overlap, 0, 1},
                 {"SNELLY_WF_SHADE_SHARE", &d.shade_share, 1, 8}, {"SNELLY_WF_INTERLEAVE", &d.interleave, 0, 1},
                 {"SNELLY_WF_VOLUME", &d.vol_stage, 0, 1}};
    for (unsigned k = 0; k < sizeof knobs / sizeof knobs[0]; ++k)
      if (const char* v = getenv(knobs[k].name)) {
        *knobs[k].field = std::max(knobs[k].lo, std::min(atoi(v), knobs[k].hi));
        c->wf_fixed |= 1u << k;
      }
    d.block = d.block < 128 ? 64 : 128;
  }
  const char* cdir = getenv("SNELLY_CACHE_DIR");
  c->cache_dir = cdir ? std::string(cdir) : dir + "/_build/kcache";
  mkdir((dir + "/_build").c_str(), 0755);
  if (mkdir(c->cache_dir.c_str(), 0755) != 0 && !file_exists(c->cache_dir)) c->cache_dir.clear();
  int rc = c->alloc(c->xyz, sizeof(kXyzTable));
  if (rc) return rc;
  RT_TRY(cudaMemcpy(c->xyz.ptr, kXyzTable, sizeof(kXyzTable), cudaMemcpyHostToDevice));
  auto* h = new snelly_ctx;
  h->c = std::move(c);
  *out = h;
  return SNELLY_OK;
}

int snelly_shutdown(snelly_ctx* ctx) {
  if (!ctx) return fail(SNELLY_EINVAL, "ctx is null");
  delete ctx;
  return SNELLY_OK;
}

int snelly_create_scene(snelly_ctx* ctx, const char* glsl, const snelly_scene_opts* opts, uint64_t* scene_id,
                        char* log, size_t log_cap) {
  if (!ctx || !glsl || !opts || !scene_id) return fail(SNELLY_EINVAL, "null argument to snelly_create_scene");
  Context& c = *ctx->c;
  std::lock_guard<std::mutex> lk(c.mu);
  snelly_scene_opts o = *opts;
  if (o.max_bounces < 0 || o.max_bounces > 64) return fail(SNELLY_EINVAL, "max_bounces out of range [0, 64]");
  if (o.max_march_steps < 1 || o.max_march_steps > 100000) return fail(SNELLY_EINVAL, "max_march_steps out of range");
  if (o.max_samples_per_frame < 1 || o.max_samples_per_frame > 1024)
    return fail(SNELLY_EINVAL, "max_samples_per_frame out of range");
  if (o.max_atmosphere_scatters < 0 || o.max_atmosphere_scatters > 64)
    return fail(SNELLY_EINVAL, "max_atmosphere_scatters out of range");
  Scene s;
  int rc = assemble_scene(glsl, o, &s.src);
  if (rc) {
    if (log && log_cap) snprintf(log, log_cap, "%s", t_last_error.c_str());
    return rc;
  }
  s.opts = o;
  // The wavefront integrator serves one sample per pixel per frame (the reference default);
  // more samples per frame consume one pixel's RNG stream sequentially and use the per-pixel kernel.
  // SNELLY_KERNEL_AUTO is decided per job by the autotuner (wavefront.cpp).
  s.kernel_mode = o.max_samples_per_frame == 1 && (o.kernel_mode == SNELLY_KERNEL_WAVEFRONT || o.kernel_mode == SNELLY_KERNEL_AUTO)
                      ? o.kernel_mode
                      : SNELLY_KERNEL_MEGA;
  std::string nvlog;
  rc = c.compile_module(program_source(s.src), o.math_mode, &s.module, &nvlog);
  if (log && log_cap) snprintf(log, log_cap, "%s", rc ? t_last_error.c_str() : nvlog.c_str());
  if (rc) return rc;
  s.ublock.assign(s.src.xf.block_size, 0);
  s.id = ++c.next_id;
  *scene_id = s.id;
  c.scenes[s.id] = std::move(s);
  return SNELLY_OK;
}

int snelly_destroy_scene(snelly_ctx* ctx, uint64_t scene_id) {
  if (!ctx) return fail(SNELLY_EINVAL, "ctx is null");
  Context& c = *ctx->c;
  std::lock_guard<std::mutex> lk(c.mu);
  auto it = c.scenes.find(scene_id);
  if (it == c.scenes.end()) return fail(SNELLY_ENOTFOUND, "unknown scene id");
  for (auto& kv : c.jobs)
    if (kv.second.scene == &it->second) return fail(SNELLY_EBUSY, "scene has live jobs");
  for (auto& t : it->second.textures) c.release(t.second);
  for (auto& t : it->second.retired_textures) c.release(t);
  c.scenes.erase(it);
  return SNELLY_OK;
}

int snelly_set_uniforms(snelly_ctx* ctx, uint64_t scene_id, const snelly_uniform* u, size_t n) {
  if (!ctx || (!u && n)) return fail(SNELLY_EINVAL, "null argument to snelly_set_uniforms");
  Context& c = *ctx->c;
  std::lock_guard<std::mutex> lk(c.mu);
  auto it = c.scenes.find(scene_id);
  if (it == c.scenes.end()) return fail(SNELLY_ENOTFOUND, "unknown scene id");
  Scene& s = it->second;
  for (size_t k = 0; k < n; ++k) {
    const snelly_uniform& v = u[k];
    if (!v.name) return fail(SNELLY_EINVAL, "uniform name is null");
    const GlslUniform* g = nullptr;
    for (auto& q : s.src.xf.uniforms)
      if (q.name == v.name) g = &q;
    if (!g) return fail(SNELLY_ENOTFOUND, std::string("scene declares no uniform '") + v.name + "'");
    if (g->kind == UK_SAMPLER2D || g->kind == UK_SAMPLER3D)
      return fail(SNELLY_EINVAL, std::string("uniform '") + v.name + "' is a sampler: use snelly_set_texture");
    bool is_int = (g->kind == UK_INT || g->kind == UK_BOOL || g->kind == UK_IVEC2 || g->kind == UK_IVEC3 ||
                   g->kind == UK_IVEC4);
    int type_ok = (v.type == g->kind) || (g->kind == UK_BOOL && v.type == SNELLY_U_INT) ||
                  (g->kind == UK_INT && v.type == SNELLY_U_BOOL);
    if (!type_ok) return fail(SNELLY_EINVAL, std::string("type mismatch for uniform '") + v.name + "'");
    int maxn = g->array_len ? g->array_len : 1;
    if (v.count < 1 || v.count > maxn) return fail(SNELLY_EINVAL, std::string("bad element count for '") + v.name + "'");
    if (is_int ? !v.i : !v.f) return fail(SNELLY_EINVAL, std::string("missing values for '") + v.name + "'");
    for (int e = 0; e < v.count; ++e)
      for (int q = 0; q < g->components; ++q) {
        size_t off = g->offset + e * g->elem_size + 4 * q;
        if (is_int) memcpy(&s.ublock[off], &v.i[e * g->components + q], 4);
        else memcpy(&s.ublock[off], &v.f[e * g->components + q], 4);
      }
  }
  return SNELLY_OK;
}

int snelly_set_texture(snelly_ctx* ctx, uint64_t scene_id, const char* name, const void* data, int w, int h, int d,
                       int channels, int fmt, int linear) {
  if (!ctx || !name || !data) return fail(SNELLY_EINVAL, "null argument to snelly_set_texture");
  if (w < 1 || h < 1 || d < 1 || channels < 1 || channels > 4 || fmt < 0 || fmt > 2)
    return fail(SNELLY_EINVAL, "bad texture dimensions or format");
  Context& c = *ctx->c;
  std::lock_guard<std::mutex> lk(c.mu);
  auto it = c.scenes.find(scene_id);
  if (it == c.scenes.end()) return fail(SNELLY_ENOTFOUND, "unknown scene id");
  Scene& s = it->second;
  const GlslUniform* g = nullptr;
  for (auto& q : s.src.xf.uniforms)
    if (q.name == name) g = &q;
  if (!g || (g->kind != UK_SAMPLER2D && g->kind != UK_SAMPLER3D))
    return fail(SNELLY_ENOTFOUND, std::string("scene declares no sampler '") + name + "'");
  if (g->kind == UK_SAMPLER2D && d != 1) return fail(SNELLY_EINVAL, "sampler2D texture must have depth 1");
  size_t esz = fmt == 0 ? 4 : (fmt == 1 ? 2 : 1);
  size_t bytes = (size_t)w * h * d * channels * esz;
  DevBuf& b = s.textures[name];
  // Jobs of this scene hold the old texture's address in their uniform snapshot: it stays
  // allocated until the scene is destroyed (which needs the jobs gone).
  bool referenced = false;
  for (auto& kv : c.jobs)
    if (kv.second.scene == &s) referenced = true;
  if (referenced && b.ptr) {
    s.retired_textures.push_back(b);
    b = DevBuf{};
  } else {
    c.release(b);
  }
  int rc = c.alloc(b, bytes);
  if (rc) return rc;
  RT_TRY(cudaMemcpy(b.ptr, data, bytes, cudaMemcpyHostToDevice));
  // sampler2D {data, w, h, ch, fmt, filter, srgb}; sampler3D {data, w, h, d, ch, fmt, filter}
  struct {
    const void* p;
    int a[6];
  } rec;
  rec.p = b.ptr;
  if (g->kind == UK_SAMPLER2D) {
    int v[6] = {w, h, channels, fmt, linear ? 1 : 0, 0};
    memcpy(rec.a, v, sizeof v);
  } else {
    int v[6] = {w, h, d, channels, fmt, linear ? 1 : 0};
    memcpy(rec.a, v, sizeof v);
  }
  memcpy(&s.ublock[g->offset], &rec, sizeof rec);
  return SNELLY_OK;
}

// A one-pixel job of snelly_pick: the pixel coordinate and the frame it belongs to.
struct PickAt {
  float x, y;
  int width, height;
};

static int start_job(Context& c, uint64_t scene_id, const snelly_render_desc* desc, const uint32_t* rng,
                     const float* acc, const float* comp, uint64_t* job_id, const PickAt* pick = nullptr) {
  auto it = c.scenes.find(scene_id);
  if (it == c.scenes.end()) return fail(SNELLY_ENOTFOUND, "unknown scene id");
  if (desc->width < 1 || desc->height < 1 || (long long)desc->width * desc->height > (1ll << 30))
    return fail(SNELLY_EINVAL, "bad image size");
  if (desc->frames < 0) return fail(SNELLY_EINVAL, "frames must be >= 0");
  if (desc->mode < SNELLY_MODE_PT || desc->mode > SNELLY_MODE_PTSIMPLE) return fail(SNELLY_EINVAL, "bad render mode");
  const SnellyParams& p = desc->params;
  if (p.dieleModel < SNELLY_IOR_ABBE || p.dieleModel > SNELLY_IOR_CAUCHY || p.dieleNumCoeffs < 0 ||
      p.dieleNumCoeffs > SNELLY_MAX_IOR_COEFFS)
    return fail(SNELLY_EINVAL, "bad dielectric model");
  if (desc->env_map && (desc->env_w < 1 || desc->env_h < 1)) return fail(SNELLY_EINVAL, "bad environment map size");
  Scene& s = it->second;
  Job j;
  j.scene = &s;
  j.module = s.module.get();
  if (desc->mode != SNELLY_MODE_PT && desc->mode != SNELLY_MODE_PTSIMPLE) {  // first-hit passes
    if (s.opts.math_mode == SNELLY_MATH_STRICT) {
      s.strict_module = s.module;
    } else if (!s.strict_module) {
      std::string nvlog;
      int rc0 = c.compile_module(program_source(s.src), SNELLY_MATH_STRICT, &s.strict_module, &nvlog);
      if (rc0) return rc0;
    }
    j.module = s.strict_module.get();
  }
  j.desc = *desc;
  j.desc.env_map = nullptr;
  j.params = desc->params;
  j.params.resolution[0] = (float)desc->width;
  j.params.resolution[1] = (float)desc->height;
  if (pick) {
    j.params.resolution[0] = (float)pick->width;
    j.params.resolution[1] = (float)pick->height;
    j.pick_at = 1;
    j.pick_x = pick->x;
    j.pick_y = pick->y;
  }
  j.ublock = s.ublock;
  fill_renderer_uniforms(s.src.xf.uniforms, &j.params, j.ublock);  // renderer uniforms the scene reads
  size_t npix = (size_t)desc->width * desc->height;
  int rc;
  auto bail = [&](int code) {
    c.free_job(j);
    return code;
  };
  if ((rc = c.alloc(j.rng, npix * 16)) || (rc = c.alloc(j.acc, npix * 16)) || (rc = c.alloc(j.comp, npix * 16)) ||
      (rc = c.alloc(j.out, npix * 16)) || (rc = c.alloc(j.icdf, 4 * SNELLY_ICDF_SAMPLES)) ||
      (rc = c.alloc(j.gparams, sizeof(SnellyParams))) || (rc = c.alloc(j.tables, 256)))
    return bail(rc);
  if (desc->accum_fp64 && (rc = c.alloc(j.acc64, npix * 32))) return bail(rc);
  if (desc->env_map) {
    size_t eb = (size_t)desc->env_w * desc->env_h * 3;
    if ((rc = c.alloc(j.env, eb))) return bail(rc);
    if (cudaMemcpy(j.env.ptr, desc->env_map, eb, cudaMemcpyHostToDevice) != cudaSuccess)
      return bail(fail(SNELLY_EDEVICE, "environment map upload failed"));
    j.params.envMap = (const unsigned char*)j.env.ptr;
    j.params.envMapW = desc->env_w;
    j.params.envMapH = desc->env_h;
    j.params.haveEnvMap = 1;
  } else {
    j.params.envMap = nullptr;
    j.params.envMapW = j.params.envMapH = 0;
    j.params.haveEnvMap = 0;
  }
  std::vector<float> icdf = inverse_cdf(desc->spectrum);
  if (cudaMemcpy(j.icdf.ptr, icdf.data(), icdf.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(fail(SNELLY_EDEVICE, "ICDF upload failed"));
  j.params.xyzTable = (const float*)c.xyz.ptr;
  j.params.icdfTable = (const float*)j.icdf.ptr;
  if (cudaMemcpy(j.gparams.ptr, &j.params, sizeof(SnellyParams), cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(fail(SNELLY_EDEVICE, "parameter upload failed"));
  if (cudaEventCreateWithFlags(&j.done, cudaEventDisableTiming) != cudaSuccess)
    return bail(fail(SNELLY_EDEVICE, "event creation failed"));
  if ((rc = c.single_job_tables(j))) return bail(rc);
  j.kernel_mode = SNELLY_KERNEL_MEGA;
  if (desc->mode == SNELLY_MODE_PT && s.kernel_mode != SNELLY_KERNEL_MEGA && j.module->f_wf_generate)
    j.kernel_mode = s.kernel_mode;
  j.wfc = c.wf_default;
  if (j.kernel_mode != SNELLY_KERNEL_MEGA && (rc = c.alloc_wavefront(j))) return bail(rc);
  if (j.kernel_mode == SNELLY_KERNEL_AUTO && (rc = c.autotune(j))) return bail(rc);
  if (rng) {
    if (cudaMemcpy(j.rng.ptr, rng, npix * 16, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(j.acc.ptr, acc, npix * 16, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(j.comp.ptr, comp, npix * 16, cudaMemcpyHostToDevice) != cudaSuccess)
      return bail(fail(SNELLY_EDEVICE, "state upload failed"));
    if (j.acc64.ptr) cudaMemsetAsync(j.acc64.ptr, 0, j.acc64.bytes, c.stream);
  } else {
    void* tables = j.tables.ptr;
    void* bstart = (char*)j.tables.ptr + 128;
    int njobs = 1;
    void* args[] = {&tables, &bstart, &njobs};
    if ((rc = c.launch(j.module->f_seed, j.blocks, SNELLY_BLOCK, args))) return bail(rc);
  }
  if (desc->frames == 0) {  // the mean image of the seeded or restored state, for readback
    void* tables = j.tables.ptr;
    void* bstart = (char*)j.tables.ptr + 128;
    int njobs = 1;
    void* rargs[] = {&tables, &bstart, &njobs};
    if ((rc = c.launch(j.module->f_resolve, j.blocks, SNELLY_BLOCK, rargs))) return bail(rc);
  }
  j.id = ++c.next_id;
  uint64_t id = j.id;
  c.jobs[id] = std::move(j);
  Job& jj = c.jobs[id];
  if ((rc = c.enqueue_frames(jj, desc->frames))) {
    c.free_job(jj);
    c.jobs.erase(id);
    return rc;
  }
  if (desc->frames == 0) cudaEventRecord(jj.done, c.stream);
  *job_id = id;
  return SNELLY_OK;
}

int snelly_render(snelly_ctx* ctx, uint64_t scene_id, const snelly_render_desc* desc, uint64_t* job_id) {
  if (!ctx || !desc || !job_id) return fail(SNELLY_EINVAL, "null argument to snelly_render");
  Context& c = *ctx->c;
  std::lock_guard<std::mutex> lk(c.mu);
  return start_job(c, scene_id, desc, nullptr, nullptr, nullptr, job_id);
}

int snelly_restore(snelly_ctx* ctx, uint64_t scene_id, const snelly_render_desc* desc, const uint32_t* rng,
                   const float* acc, const float* comp, uint64_t* job_id) {
  if (!ctx || !desc || !job_id || !rng || !acc || !comp) return fail(SNELLY_EINVAL, "null argument to snelly_restore");
  Context& c = *ctx->c;
  std::lock_guard<std::mutex> lk(c.mu);
  return start_job(c, scene_id, desc, rng, acc, comp, job_id);
}

int snelly_advance(snelly_ctx* ctx, uint64_t job_id, int frames) {
  if (!ctx) return fail(SNELLY_EINVAL, "ctx is null");
  if (frames < 0) return fail(SNELLY_EINVAL, "frames must be >= 0");
  Context& c = *ctx->c;
  std::lock_guard<std::mutex> lk(c.mu);
  auto it = c.jobs.find(job_id);
  if (it == c.jobs.end()) return fail(SNELLY_ENOTFOUND, "unknown job id");
  if (it->second.cancelled) return fail(SNELLY_ECANCELLED, "job was cancelled");
  return c.enqueue_frames(it->second, frames);
}

int snelly_update_job(snelly_ctx* ctx, uint64_t job_id, const snelly_render_desc* desc) {
  if (!ctx || !desc) return fail(SNELLY_EINVAL, "null argument to snelly_update_job");
  Context& c = *ctx->c;
  std::lock_guard<std::mutex> lk(c.mu);
  auto it = c.jobs.find(job_id);
  if (it == c.jobs.end()) return fail(SNELLY_ENOTFOUND, "unknown job id");
  Job& j = it->second;
  if (j.cancelled) return fail(SNELLY_ECANCELLED, "job was cancelled");
  if (j.pick_at) return fail(SNELLY_EINVAL, "pick jobs cannot be updated");
  if (desc->width != j.desc.width || desc->height != j.desc.height || desc->mode != j.desc.mode)
    return fail(SNELLY_EINVAL, "image size and render mode are fixed for a job: reset and render a new one");
  const SnellyParams& p = desc->params;
  if (p.dieleModel < SNELLY_IOR_ABBE || p.dieleModel > SNELLY_IOR_CAUCHY || p.dieleNumCoeffs < 0 ||
      p.dieleNumCoeffs > SNELLY_MAX_IOR_COEFFS)
    return fail(SNELLY_EINVAL, "bad dielectric model");
  // The job's own resources stay: resolution, environment map and the table pointers.
  SnellyParams np = p;
  np.resolution[0] = j.params.resolution[0];
  np.resolution[1] = j.params.resolution[1];
  np.envMap = j.params.envMap;
  np.envMapW = j.params.envMapW;
  np.envMapH = j.params.envMapH;
  np.haveEnvMap = j.params.haveEnvMap;
  np.xyzTable = j.params.xyzTable;
  np.icdfTable = j.params.icdfTable;
  // Every upload below is ordered on the context stream after the frames already enqueued.
  if (memcmp(&desc->spectrum, &j.desc.spectrum, sizeof(snelly_spectrum)) != 0) {
    std::vector<float> icdf = inverse_cdf(desc->spectrum);
    RT_TRY(cudaMemcpyAsync(j.icdf.ptr, icdf.data(), icdf.size() * 4, cudaMemcpyHostToDevice, c.stream));
    RT_TRY(cudaStreamSynchronize(c.stream));  // the staging vector goes out of scope
    j.desc.spectrum = desc->spectrum;
  }
  j.params = np;
  j.ublock = j.scene->ublock;
  fill_renderer_uniforms(j.scene->src.xf.uniforms, &j.params, j.ublock);
  RT_TRY(cudaMemcpyAsync(j.gparams.ptr, &j.params, sizeof(SnellyParams), cudaMemcpyHostToDevice, c.stream));
  RT_TRY(cudaStreamSynchronize(c.stream));  // j.params may change again before the copy runs
  return SNELLY_OK;
}

int snelly_advance_batch(snelly_ctx* ctx, const uint64_t* job_ids, const int* frames, size_t n) {
  if (!ctx || (n && (!job_ids || !frames))) return fail(SNELLY_EINVAL, "null argument to snelly_advance_batch");
  Context& c = *ctx->c;
  std::lock_guard<std::mutex> lk(c.mu);
  std::vector<Job*> js;
  std::vector<int> fs;
  for (size_t k = 0; k < n; ++k) {
    auto it = c.jobs.find(job_ids[k]);
    if (it == c.jobs.end()) return fail(SNELLY_ENOTFOUND, "unknown job id in batch");
    if (it->second.cancelled) return fail(SNELLY_ECANCELLED, "cancelled job in batch");
    if (frames[k] < 0) return fail(SNELLY_EINVAL, "frames must be >= 0");
    if (it->second.desc.mode != SNELLY_MODE_PT) return fail(SNELLY_EINVAL, "batches run the path tracer only");
    for (Job* q : js)
      if (q == &it->second) return fail(SNELLY_EINVAL, "job listed twice in batch");
    js.push_back(&it->second);
    fs.push_back(frames[k]);
  }
  return c.advance_batch(js, fs);
}

extern "C++" {
int snelly::wait_job(Context& c, Job& j, int flags) {
  if (flags & SNELLY_READ_POLL) {
    cudaError_t e = cudaEventQuery(j.done);
    if (e == cudaErrorNotReady) return fail(SNELLY_EBUSY, "job not finished");
    if (e != cudaSuccess) return fail(SNELLY_EDEVICE, std::string("job failed: ") + cudaGetErrorString(e));
    return SNELLY_OK;
  }
  (void)c;
  cudaError_t e = cudaEventSynchronize(j.done);
  if (e != cudaSuccess) return fail(SNELLY_EDEVICE, std::string("job failed: ") + cudaGetErrorString(e));
  return SNELLY_OK;
}
}  // extern "C++"

int snelly_readback(snelly_ctx* ctx, uint64_t job_id, float* out, size_t bytes, int flags) {
  if (!ctx || !out) return fail(SNELLY_EINVAL, "null argument to snelly_readback");
  Context& c = *ctx->c;
  std::lock_guard<std::mutex> lk(c.mu);
  auto it = c.jobs.find(job_id);
  if (it == c.jobs.end()) return fail(SNELLY_ENOTFOUND, "unknown job id");
  Job& j = it->second;
  if (j.cancelled) return fail(SNELLY_ECANCELLED, "job was cancelled");
  size_t need = (size_t)j.desc.width * j.desc.height * 16;
  if (bytes < need) return fail(SNELLY_EINVAL, "output buffer too small: need " + std::to_string(need) + " bytes");
  if (flags & SNELLY_READ_ASYNC) {  // copy after the enqueued frames, on the copy stream; return now
    if (!c.copy_stream) RT_TRY(cudaStreamCreateWithFlags(&c.copy_stream, cudaStreamNonBlocking));
    if (!j.read_done) RT_TRY(cudaEventCreateWithFlags(&j.read_done, cudaEventDisableTiming));
    RT_TRY(cudaStreamWaitEvent(c.copy_stream, j.done, 0));
    RT_TRY(cudaMemcpyAsync(out, j.out.ptr, need, cudaMemcpyDeviceToHost, c.copy_stream));
    RT_TRY(cudaEventRecord(j.read_done, c.copy_stream));
    j.read_pending = true;
    return SNELLY_OK;
  }
  int rc = wait_job(c, j, flags);
  if (rc) return rc;
  if (j.read_pending) {  // earlier asynchronous copies of this job are complete when this returns
    RT_TRY(cudaEventSynchronize(j.read_done));
    j.read_pending = false;
  }
  RT_TRY(cudaMemcpyAsync(out, j.out.ptr, need, cudaMemcpyDeviceToHost, c.stream));
  RT_TRY(cudaStreamSynchronize(c.stream));
  return SNELLY_OK;
}

int snelly_pick(snelly_ctx* ctx, uint64_t scene_id, const snelly_render_desc* desc, float x, float y, float* distance,
                float* material) {
  if (!ctx || !desc || !distance || !material) return fail(SNELLY_EINVAL, "null argument to snelly_pick");
  if (desc->width < 1 || desc->height < 1) return fail(SNELLY_EINVAL, "bad image size");
  Context& c = *ctx->c;
  std::lock_guard<std::mutex> lk(c.mu);
  snelly_render_desc d = *desc;
  d.width = d.height = 1;
  d.frames = 1;
  d.mode = SNELLY_MODE_PICK;
  d.accum_fp64 = 0;
  PickAt pa{x, y, desc->width, desc->height};
  uint64_t id = 0;
  int rc = start_job(c, scene_id, &d, nullptr, nullptr, nullptr, &id, &pa);
  if (rc) return rc;
  Job& j = c.jobs[id];
  float r[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  rc = wait_job(c, j, SNELLY_READ_WAIT);
  if (!rc && (cudaMemcpyAsync(r, j.out.ptr, sizeof r, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
              cudaStreamSynchronize(c.stream) != cudaSuccess))
    rc = fail(SNELLY_EDEVICE, "pick readback failed");
  c.free_job(j);
  c.jobs.erase(id);
  if (rc) return rc;
  *distance = r[0];
  *material = r[1];
  return SNELLY_OK;
}

int snelly_readback_state(snelly_ctx* ctx, uint64_t job_id, uint32_t* rng, float* acc, float* comp, double* acc64) {
  if (!ctx) return fail(SNELLY_EINVAL, "ctx is null");
  Context& c = *ctx->c;
  std::lock_guard<std::mutex> lk(c.mu);
  auto it = c.jobs.find(job_id);
  if (it == c.jobs.end()) return fail(SNELLY_ENOTFOUND, "unknown job id");
  Job& j = it->second;
  int rc = wait_job(c, j, SNELLY_READ_WAIT);
  if (rc) return rc;
  size_t npix = (size_t)j.desc.width * j.desc.height;
  if (rng) RT_TRY(cudaMemcpy(rng, j.rng.ptr, npix * 16, cudaMemcpyDeviceToHost));
  if (acc) RT_TRY(cudaMemcpy(acc, j.acc.ptr, npix * 16, cudaMemcpyDeviceToHost));
  if (comp) RT_TRY(cudaMemcpy(comp, j.comp.ptr, npix * 16, cudaMemcpyDeviceToHost));
  if (acc64) {
    if (!j.acc64.ptr) return fail(SNELLY_EINVAL, "job has no FP64 accumulation");
    RT_TRY(cudaMemcpy(acc64, j.acc64.ptr, npix * 32, cudaMemcpyDeviceToHost));
  }
  return SNELLY_OK;
}

int snelly_job_kernel(snelly_ctx* ctx, uint64_t job_id, int* kernel_mode) {
  if (!ctx || !kernel_mode) return fail(SNELLY_EINVAL, "null argument to snelly_job_kernel");
  Context& c = *ctx->c;
  std::lock_guard<std::mutex> lk(c.mu);
  auto it = c.jobs.find(job_id);
  if (it == c.jobs.end()) return fail(SNELLY_ENOTFOUND, "unknown job id");
  *kernel_mode = it->second.kernel_mode;
  return SNELLY_OK;
}

int snelly_job_wavefront_config(snelly_ctx* ctx, uint64_t job_id, int* out) {
  if (!ctx || !out) return fail(SNELLY_EINVAL, "null argument to snelly_job_wavefront_config");
  Context& c = *ctx->c;
  std::lock_guard<std::mutex> lk(c.mu);
  auto it = c.jobs.find(job_id);
  if (it == c.jobs.end()) return fail(SNELLY_ENOTFOUND, "unknown job id");
  const WfConfig& w = it->second.wfc;
  const int v[SNELLY_WF_CONFIG_FIELDS] = {it->second.wf_parts, w.shade_split, w.drain,  w.chunk,    w.grab,
                                          w.refill,              w.block,       w.park_left, w.walker, w.lane_rays,
                                          w.overlap,             w.shade_share, w.interleave, w.vol_stage};
  for (int k = 0; k < SNELLY_WF_CONFIG_FIELDS; ++k) out[k] = v[k];
  return SNELLY_OK;
}

int snelly_job_status(snelly_ctx* ctx, uint64_t job_id, int* enq, int* done) {
  if (!ctx) return fail(SNELLY_EINVAL, "ctx is null");
  Context& c = *ctx->c;
  std::lock_guard<std::mutex> lk(c.mu);
  auto it = c.jobs.find(job_id);
  if (it == c.jobs.end()) return fail(SNELLY_ENOTFOUND, "unknown job id");
  Job& j = it->second;
  if (enq) *enq = j.frames_enqueued;
  if (done) *done = cudaEventQuery(j.done) == cudaSuccess ? j.frames_enqueued : -1;
  return SNELLY_OK;
}

int snelly_cancel(snelly_ctx* ctx, uint64_t job_id) {
  if (!ctx) return fail(SNELLY_EINVAL, "ctx is null");
  Context& c = *ctx->c;
  std::lock_guard<std::mutex> lk(c.mu);
  auto it = c.jobs.find(job_id);
  if (it == c.jobs.end()) return fail(SNELLY_ENOTFOUND, "unknown job id");
  it->second.cancelled = true;
  return SNELLY_OK;
}

int snelly_destroy_job(snelly_ctx* ctx, uint64_t job_id) {
  if (!ctx) return fail(SNELLY_EINVAL, "ctx is null");
  Context& c = *ctx->c;
  std::lock_guard<std::mutex> lk(c.mu);
  auto it = c.jobs.find(job_id);
  if (it == c.jobs.end()) return fail(SNELLY_ENOTFOUND, "unknown job id");
  cudaEventSynchronize(it->second.done);
  c.free_job(it->second);
  c.jobs.erase(it);
  return SNELLY_OK;
}

int snelly_sync(snelly_ctx* ctx) {
  if (!ctx) return fail(SNELLY_EINVAL, "ctx is null");
  RT_TRY(cudaStreamSynchronize(ctx->c->stream));
  if (ctx->c->copy_stream) RT_TRY(cudaStreamSynchronize(ctx->c->copy_stream));  // SNELLY_READ_ASYNC copies
  return SNELLY_OK;
}

int snelly_inverse_cdf(const snelly_spectrum* s, float* out) {
  if (!s || !out) return fail(SNELLY_EINVAL, "null argument to snelly_inverse_cdf");
  std::vector<float> v = inverse_cdf(*s);
  memcpy(out, v.data(), v.size() * sizeof(float));
  return SNELLY_OK;
}

size_t snelly_abi_sizeof(int which) {
  switch (which) {
    case 0: return sizeof(SnellyParams);
    case 1: return sizeof(snelly_render_desc);
    case 2: return sizeof(snelly_scene_opts);
    case 3: return sizeof(snelly_uniform);
    case 4: return sizeof(snelly_spectrum);
    default: return 0;
  }
}

void* snelly_stream(snelly_ctx* ctx) { return ctx ? (void*)ctx->c->stream : nullptr; }
uint64_t snelly_launch_count(snelly_ctx* ctx) { return ctx ? ctx->c->launches : 0; }

int snelly_compile_check(const char* glsl, const snelly_scene_opts* opts, char* log, size_t log_cap,
                         size_t* cubin_bytes) {
  if (!glsl || !opts) return fail(SNELLY_EINVAL, "null argument to snelly_compile_check");
  SceneSource ss;
  int rc = assemble_scene(glsl, *opts, &ss);
  if (rc) {
    if (log && log_cap) snprintf(log, log_cap, "%s", t_last_error.c_str());
    return rc;
  }
  std::string dir = library_dir();
  const char* env = getenv("SNELLY_KERNEL_DIR");
  std::string csrc = env ? std::string(env) : dir + "/csrc";
  std::string inc = env ? std::string(env) + "/../../include" : dir + "/../include";
  std::vector<char> cubin;
  std::string lg;
  std::vector<std::string> nopts = nvrtc_options(csrc + "/kernels", csrc, inc, opts->math_mode);
  const std::string src = program_source(ss);
  rc = nvrtc_cubin(src, nopts, &cubin, &lg);
  if (!rc) {  // into the module cache, where a context on a GPU machine finds it
    const char* cdir = getenv("SNELLY_CACHE_DIR");
    std::string cache = cdir ? std::string(cdir) : dir + "/_build/kcache";
    mkdir((dir + "/_build").c_str(), 0755);
    if (mkdir(cache.c_str(), 0755) == 0 || file_exists(cache))
      cache_store(cache + "/" + module_key(src, nopts, csrc + "/kernels", csrc, inc) + ".cubin", cubin);
  }
  if (log && log_cap) snprintf(log, log_cap, "%s", rc ? t_last_error.c_str() : lg.c_str());
  if (cubin_bytes) *cubin_bytes = cubin.size();
  return rc;
}

int snelly_glsl_to_cpp(const char* glsl, const char* struct_name, const char* extra_members, char* out,
                       size_t out_cap) {
  if (!glsl || !out || !out_cap) return fail(SNELLY_EINVAL, "null argument to snelly_glsl_to_cpp");
  GlslTransformResult r;
  if (!glsl_transform(glsl, struct_name ? struct_name : "Scene", extra_members ? extra_members : kSceneExtraMembers, &r))
    return fail(SNELLY_ECOMPILE, "GLSL translation failed: " + r.error);
  if (r.code.size() + 1 > out_cap) return fail(SNELLY_EINVAL, "output buffer too small: need " + std::to_string(r.code.size() + 1));
  memcpy(out, r.code.c_str(), r.code.size() + 1);
  return SNELLY_OK;
}

}  // extern "C"
