// glsl_transform.h - rewrite a GLSL ES 3.00 scene (or whole fragment shader) as a C++ struct.
//
// The scene string a Snelly scene returns from shader() (js/sceneAPI.js:120-198) is GLSL that
// defines SDF_SURFACE/SDF_METAL/SDF_DIELECTRIC and optional hooks, plus `uniform`s that the
// scene's syncShader() sets. glsl_transform() turns it into
//
//   struct <Name>Uniforms { ... };          // one field per `uniform`, fixed layout
//   struct <Name> {                         // everything else, as members
//     const T& uniformName; ...             // bound to a <Name>Uniforms block
//     explicit <Name>(const <Name>Uniforms&);
//     <globals as data members, functions as member functions>
//   };
//
// so that each GPU thread (or CPU oracle thread) owns its own copy of the scene's globals
// (GLSL globals are per-invocation) and the uniforms of the job it is working on.
#pragma once
#include <string>
#include <vector>

namespace snelly {

enum UniformKind {
  UK_FLOAT = 0, UK_INT = 1, UK_BOOL = 2, UK_VEC2 = 3, UK_VEC3 = 4, UK_VEC4 = 5,
  UK_IVEC2 = 6, UK_IVEC3 = 7, UK_IVEC4 = 8, UK_MAT2 = 9, UK_MAT3 = 10, UK_MAT4 = 11,
  UK_SAMPLER2D = 12, UK_SAMPLER3D = 13
};

struct GlslUniform {
  std::string name;
  std::string glsl_type;
  int kind = 0;
  int array_len = 0;     // 0 = not an array
  int components = 1;    // scalars per element (float/int components; samplers: 0)
  size_t offset = 0;     // byte offset in the uniform block
  size_t elem_size = 0;  // bytes per element
  // >= 0: one of the renderer's own uniforms that the scene reads without declaring it (scene
  // code sits inside the reference's fragment shader and sees its uniforms); the value comes from
  // this byte offset of the job's SnellyParams, which holds every such uniform under its name
  long params_offset = -1;
};

struct GlslTransformResult {
  std::string code;               // C++ source: uniform block struct + scene struct
  std::vector<GlslUniform> uniforms;
  size_t block_size = 0;          // sizeof(<Name>Uniforms) (>= 1)
  std::vector<std::string> functions;  // names of the functions the source defines
  std::string error;              // empty on success
};

// extra_members: C++ member declarations prepended to the struct body (used when a whole
// fragment shader is wrapped: gl_FragCoord and the like). A renderer uniform (the path tracer's
// own uniforms, js/renderer.js:520-584) that the source reads but does not declare is added to
// the uniform block after the source's own uniforms, with its params_offset set.
bool glsl_transform(const std::string& src, const std::string& name,
                    const std::string& extra_members, GlslTransformResult* out);

// Replace float literals, `float`, parameter qualifiers etc. in a free-standing fragment of
// GLSL code (no global-scope handling). Used for #define bodies and tests.
std::string glsl_rewrite_fragment(const std::string& src);

// Copy the values of a block's renderer uniforms (params_offset >= 0) from a SnellyParams.
void fill_renderer_uniforms(const std::vector<GlslUniform>& uniforms, const void* params,
                            std::vector<unsigned char>& block);

}  // namespace snelly
