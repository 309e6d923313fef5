// glsl_transform.cpp - token-level GLSL ES 3.00 -> C++ rewrite (see glsl_transform.h).
//
// Rules applied to the token stream:
//   * float literals get an `f` suffix (GLSL literals are single precision; unsuffixed C++
//     literals are double and would promote arithmetic);
//   * `float` becomes `gfloat` (float, or the oracle's operation-counting scalar);
//   * parameter qualifiers: `in` is dropped, `out`/`inout` turn the parameter into a reference;
//   * precision / interpolation qualifiers and `layout(...)` are dropped;
//   * GLSL array constructors `T[N](a, b)` become brace initialisers `{a, b}`;
//   * identifiers that are C++ (but not GLSL) keywords get a `_g` suffix;
//   * at global scope: `uniform` declarations move to the uniform block, function prototypes
//     are dropped (member functions may be used before their definition), `in`/`out`
//     globals become plain members, everything else stays in order inside the struct.
#include "glsl_transform.h"

#include <algorithm>
#include <cctype>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <map>
#include <set>
#include <sstream>

#include "snelly_params.h"

namespace snelly {
namespace {

// The path tracer's own uniforms (the non-sampler `uniform` declarations of
// shaders/pathtracer-fragment-shader.glsl) with their GLSL types; SnellyParams holds each under
// the same name, with the host's conversions applied. Scene code is pasted into that shader, so
// it may read them.
struct RendererUniform {
  const char* name;
  const char* glsl_type;
  size_t params_offset;
};
#define SNELLY_RU(NAME, TYPE) {#NAME, TYPE, offsetof(SnellyParams, NAME)}
const RendererUniform kRendererUniforms[] = {
    SNELLY_RU(resolution, "vec2"), SNELLY_RU(camPos, "vec3"), SNELLY_RU(camDir, "vec3"), SNELLY_RU(camX, "vec3"),
    SNELLY_RU(camY, "vec3"), SNELLY_RU(camFovy, "float"), SNELLY_RU(camAspect, "float"),
    SNELLY_RU(camAperture, "float"), SNELLY_RU(camFocalDistance, "float"), SNELLY_RU(filterRadius, "float"),
    SNELLY_RU(radianceClamp, "float"), SNELLY_RU(skipProbability, "float"), SNELLY_RU(shadowStrength, "float"),
    SNELLY_RU(maxStepsIsMiss, "bool"), SNELLY_RU(wavelengthSamples, "int"), SNELLY_RU(lengthScale, "float"),
    SNELLY_RU(minLengthScale, "float"), SNELLY_RU(maxLengthScale, "float"), SNELLY_RU(haveEnvMap, "bool"),
    SNELLY_RU(envMapVisible, "bool"), SNELLY_RU(envMapPhiRotation, "float"), SNELLY_RU(envMapThetaRotation, "float"),
    SNELLY_RU(envMapTransitionAngle, "float"), SNELLY_RU(skyPower, "float"), SNELLY_RU(skyTintUp, "vec3"),
    SNELLY_RU(skyTintDown, "vec3"), SNELLY_RU(sunPower, "float"), SNELLY_RU(sunAngularSize, "float"),
    SNELLY_RU(sunLatitude, "float"), SNELLY_RU(sunLongitude, "float"), SNELLY_RU(sunColor, "vec3"),
    SNELLY_RU(sunDir, "vec3"), SNELLY_RU(sunVisibleDirectly, "bool"), SNELLY_RU(sphereLightPosition, "vec3"),
    SNELLY_RU(sphereLightRadius, "float"), SNELLY_RU(sphereLightPower, "float"), SNELLY_RU(sphereLightColor, "vec3"),
    SNELLY_RU(metalRoughness, "float"), SNELLY_RU(metalSpecAlbedoRGB, "vec3"), SNELLY_RU(dieleRoughness, "float"),
    SNELLY_RU(dieleAbsorptionRGB, "vec3"), SNELLY_RU(dieleSpecAlbedoRGB, "vec3"),
    SNELLY_RU(surfaceDiffuseAlbedoRGB, "vec3"), SNELLY_RU(surfaceSpecAlbedoRGB, "vec3"),
    SNELLY_RU(surfaceRoughness, "float"), SNELLY_RU(surfaceIor, "float"), SNELLY_RU(subsurface, "float"),
    SNELLY_RU(subsurfaceAlbedoRGB, "vec3"), SNELLY_RU(subsurfaceMFP, "float"), SNELLY_RU(subsurfaceAnisotropy, "float"),
    SNELLY_RU(subsurfaceDiffuseWeight, "float"), SNELLY_RU(maxSSSSteps, "int"), SNELLY_RU(atmosphereBoundsMin, "vec3"),
    SNELLY_RU(atmosphereBoundsMax, "vec3"), SNELLY_RU(atmosphereExtinctionCoeffRGB, "vec3"),
    SNELLY_RU(atmosphereScatteringCoeffRGB, "vec3"), SNELLY_RU(atmosphereMFP, "float"),
    SNELLY_RU(atmosphereAnisotropy, "float"), SNELLY_RU(fogEnable, "bool"), SNELLY_RU(fogMaxOpticalDepth, "float"),
    SNELLY_RU(fogMFP, "float"), SNELLY_RU(fogEmission, "vec3"), SNELLY_RU(fogTint, "vec3"),
    SNELLY_RU(volumeEmission, "float"), SNELLY_RU(volumeEmissionColorRGB, "vec3")};
#undef SNELLY_RU

enum TokKind { T_WS, T_COMMENT, T_PP, T_IDENT, T_NUM, T_PUNCT };
struct Tok {
  TokKind k;
  std::string s;
};

bool is_ident_start(char c) { return std::isalpha((unsigned char)c) || c == '_'; }
bool is_ident_char(char c) { return std::isalnum((unsigned char)c) || c == '_'; }

std::vector<Tok> tokenize(const std::string& s) {
  std::vector<Tok> out;
  size_t i = 0, n = s.size();
  bool line_start = true;
  while (i < n) {
    char c = s[i];
    if (c == '\n') {
      out.push_back({T_WS, "\n"});
      ++i;
      line_start = true;
      continue;
    }
    if (c == ' ' || c == '\t' || c == '\r' || c == '\f' || c == '\v') {
      size_t j = i;
      while (j < n && (s[j] == ' ' || s[j] == '\t' || s[j] == '\r' || s[j] == '\f' || s[j] == '\v')) ++j;
      out.push_back({T_WS, s.substr(i, j - i)});
      i = j;
      continue;
    }
    if (c == '#' && line_start) {
      size_t j = i;
      while (j < n && s[j] != '\n') {
        if (s[j] == '\\' && j + 1 < n && s[j + 1] == '\n') j += 2;
        else ++j;
      }
      out.push_back({T_PP, s.substr(i, j - i)});
      i = j;
      continue;
    }
    line_start = false;
    if (c == '/' && i + 1 < n && s[i + 1] == '/') {
      size_t j = i;
      while (j < n && s[j] != '\n') ++j;
      out.push_back({T_COMMENT, s.substr(i, j - i)});
      i = j;
      continue;
    }
    if (c == '/' && i + 1 < n && s[i + 1] == '*') {
      size_t j = s.find("*/", i + 2);
      j = (j == std::string::npos) ? n : j + 2;
      out.push_back({T_COMMENT, s.substr(i, j - i)});
      i = j;
      continue;
    }
    if (is_ident_start(c)) {
      size_t j = i;
      while (j < n && is_ident_char(s[j])) ++j;
      out.push_back({T_IDENT, s.substr(i, j - i)});
      i = j;
      continue;
    }
    if (std::isdigit((unsigned char)c) || (c == '.' && i + 1 < n && std::isdigit((unsigned char)s[i + 1]))) {
      size_t j = i;
      if (c == '0' && j + 1 < n && (s[j + 1] == 'x' || s[j + 1] == 'X')) {
        j += 2;
        while (j < n && std::isxdigit((unsigned char)s[j])) ++j;
      } else {
        while (j < n && std::isdigit((unsigned char)s[j])) ++j;
        if (j < n && s[j] == '.') {
          ++j;
          while (j < n && std::isdigit((unsigned char)s[j])) ++j;
        }
        if (j < n && (s[j] == 'e' || s[j] == 'E')) {
          size_t k = j + 1;
          if (k < n && (s[k] == '+' || s[k] == '-')) ++k;
          if (k < n && std::isdigit((unsigned char)s[k])) {
            j = k;
            while (j < n && std::isdigit((unsigned char)s[j])) ++j;
          }
        }
      }
      while (j < n && (s[j] == 'f' || s[j] == 'F' || s[j] == 'u' || s[j] == 'U' || s[j] == 'l' || s[j] == 'L')) ++j;
      out.push_back({T_NUM, s.substr(i, j - i)});
      i = j;
      continue;
    }
    static const char* ops3[] = {"<<=", ">>=", nullptr};
    static const char* ops2[] = {"++", "--", "<<", ">>", "<=", ">=", "==", "!=", "&&", "||", "^^",
                                 "+=", "-=", "*=", "/=", "%=", "&=", "|=", "^=", "::", nullptr};
    bool matched = false;
    for (int k = 0; ops3[k]; ++k)
      if (s.compare(i, 3, ops3[k]) == 0) { out.push_back({T_PUNCT, ops3[k]}); i += 3; matched = true; break; }
    if (matched) continue;
    for (int k = 0; ops2[k]; ++k)
      if (s.compare(i, 2, ops2[k]) == 0) { out.push_back({T_PUNCT, ops2[k]}); i += 2; matched = true; break; }
    if (matched) continue;
    out.push_back({T_PUNCT, std::string(1, c)});
    ++i;
  }
  return out;
}

bool is_float_literal(const std::string& t) {
  if (t.size() > 1 && t[0] == '0' && (t[1] == 'x' || t[1] == 'X')) return false;
  bool has_dot_or_exp = false, has_suffix_f = false, has_suffix_u = false;
  for (char c : t) {
    if (c == '.' || c == 'e' || c == 'E') has_dot_or_exp = true;
    if (c == 'f' || c == 'F') has_suffix_f = true;
    if (c == 'u' || c == 'U') has_suffix_u = true;
  }
  return has_dot_or_exp && !has_suffix_f && !has_suffix_u;
}

const std::set<std::string>& dropped_qualifiers() {
  static const std::set<std::string> s = {"highp", "mediump", "lowp", "flat", "smooth", "centroid",
                                          "invariant", "precise", "noperspective"};
  return s;
}

const std::set<std::string>& cxx_only_keywords() {
  static const std::set<std::string> s = {
      "new", "delete", "operator", "friend", "private", "protected", "public", "virtual", "explicit",
      "mutable", "typename", "try", "catch", "throw", "auto", "char", "register", "signed", "namespace",
      "using", "template", "this", "class", "typeid", "export", "constexpr", "decltype", "nullptr",
      "alignas", "alignof", "noexcept", "static_assert", "thread_local", "and", "or", "not", "xor",
      "bitand", "bitor", "compl", "and_eq", "or_eq", "not_eq", "xor_eq", "goto", "union", "enum",
      "typedef", "extern", "static", "inline", "volatile", "sizeof", "short", "long", "double",
      "unsigned", "wchar_t", "char16_t", "char32_t", "concept", "requires", "final", "override",
      "gfloat",
      // identifiers that are macros of the C/C++ math headers
      "HUGE_VAL", "HUGE_VALF", "INFINITY", "NAN", "NULL", "EOF"};
  return s;
}

size_t next_sig(const std::vector<Tok>& t, size_t i) {
  while (i < t.size() && (t[i].k == T_WS || t[i].k == T_COMMENT)) ++i;
  return i;
}

// Find the index of the token that closes the bracket opened at t[i].
size_t match_close(const std::vector<Tok>& t, size_t i) {
  const std::string open = t[i].s;
  const std::string close = open == "(" ? ")" : (open == "[" ? "]" : "}");
  int depth = 0;
  for (size_t j = i; j < t.size(); ++j) {
    if (t[j].k != T_PUNCT) continue;
    if (t[j].s == open) ++depth;
    else if (t[j].s == close && --depth == 0) return j;
  }
  return t.size();
}

std::string rewrite_pp(const std::string& pp);

// Rewrite a token range (no global-scope logic).
std::string rewrite_tokens(const std::vector<Tok>& t, size_t b, size_t e) {
  std::string out;
  bool pending_ref = false;
  std::set<size_t> replace_close;  // ')' of array constructors, emitted as '}'
  // Scalar declarations without initialiser (`float a, b;`) are value-initialised: WebGL
  // implementations zero-initialise uninitialised locals and the reference relies on it.
  int pdepth = 0;
  bool in_decl = false, expect_name = false;
  for (size_t i = b; i < e; ++i) {
    const Tok& k = t[i];
    if (replace_close.count(i)) { out += "}"; --pdepth; continue; }
    if (k.k == T_PUNCT) {
      if (k.s == "(") ++pdepth;
      else if (k.s == ")") --pdepth;
      if (in_decl && pdepth == 0) {
        if (k.s == ",") expect_name = true;
        else if (k.s == ";" || k.s == "{" || k.s == "}") in_decl = expect_name = false;
      }
      if (k.s == "(" && in_decl && expect_name) in_decl = expect_name = false;  // cast: float(x)
    }
    if (k.k == T_IDENT && pdepth == 0) {
      if (k.s == "float" || k.s == "int" || k.s == "bool" || k.s == "uint") {
        in_decl = true;
        expect_name = true;
      } else if (in_decl && expect_name && !dropped_qualifiers().count(k.s) && k.s != "const") {
        expect_name = false;
        size_t nx = next_sig(t, i + 1);
        if (nx < e && t[nx].k == T_PUNCT && (t[nx].s == ";" || t[nx].s == ",")) {
          std::string nm = cxx_only_keywords().count(k.s) ? k.s + "_g" : k.s;
          out += nm + "{}";
          continue;
        }
        if (nx < e && t[nx].k == T_PUNCT && t[nx].s == "(") in_decl = false;  // function
      }
    }
    switch (k.k) {
      case T_WS:
      case T_COMMENT:
        out += k.s;
        break;
      case T_PP:
        out += rewrite_pp(k.s);
        break;
      case T_NUM:
        out += k.s;
        if (is_float_literal(k.s)) out += "f";
        break;
      case T_PUNCT:
        out += k.s;
        break;
      case T_IDENT: {
        const std::string& s = k.s;
        if (dropped_qualifiers().count(s)) {
          size_t j = i + 1;
          if (j < e && t[j].k == T_WS) i = j;  // swallow one whitespace token
          break;
        }
        if (s == "in") {
          size_t j = i + 1;
          if (j < e && t[j].k == T_WS) i = j;
          break;
        }
        if (s == "out" || s == "inout") {
          pending_ref = true;
          size_t j = i + 1;
          if (j < e && t[j].k == T_WS) i = j;
          break;
        }
        if (s == "layout") {
          size_t j = next_sig(t, i + 1);
          if (j < e && t[j].s == "(") {
            i = match_close(t, j);
            size_t w = i + 1;
            if (w < e && t[w].k == T_WS) i = w;
          }
          break;
        }
        std::string name = s;
        if (s == "float") name = "gfloat";
        else if (cxx_only_keywords().count(s)) name = s + "_g";
        // GLSL array constructor: T[N](...) or T[](...) -> {...}
        {
          size_t j = next_sig(t, i + 1);
          if (j < e && t[j].k == T_PUNCT && t[j].s == "[") {
            size_t jc = match_close(t, j);
            size_t jp = next_sig(t, jc + 1);
            bool is_type = (s == "float" || s == "int" || s == "bool" || s == "vec2" || s == "vec3" ||
                            s == "vec4" || s == "ivec2" || s == "ivec3" || s == "ivec4" || s == "mat2" ||
                            s == "mat3" || s == "mat4");
            // preceded by '=' or '(' or ',' means an expression context
            bool expr_ctx = false;
            for (size_t q = i; q-- > b;) {
              if (t[q].k == T_WS || t[q].k == T_COMMENT) continue;
              expr_ctx = (t[q].k == T_PUNCT && (t[q].s == "=" || t[q].s == "(" || t[q].s == ","));
              break;
            }
            if (is_type && expr_ctx && jp < e && t[jp].s == "(") {
              size_t pc = match_close(t, jp);
              out += "{";
              replace_close.insert(pc);
              i = jp;  // continue after '('
              break;
            }
          }
        }
        // GLSL evaluates call arguments left to right; C++ leaves the order of constructor
        // arguments unspecified. Vector/matrix constructors whose arguments call rand() (the
        // one side-effecting call scenes make) become braced initialisations, which are
        // evaluated in order.
        {
          static const std::set<std::string> ctors = {"vec2", "vec3", "vec4", "mat2", "mat3", "mat4"};
          size_t j = next_sig(t, i + 1);
          if (ctors.count(s) && j < e && t[j].k == T_PUNCT && t[j].s == "(") {
            size_t jc = match_close(t, j);
            bool calls_rand = false;
            for (size_t q = j + 1; q < jc && q < e; ++q)
              if (t[q].k == T_IDENT && t[q].s == "rand") calls_rand = true;
            if (calls_rand && jc < e) {
              out += name + "{";
              replace_close.insert(jc);
              i = j;
              break;
            }
          }
        }
        out += name;
        if (pending_ref) {
          // the first identifier after out/inout (skipping const) is the parameter type
          if (s != "const") {
            out += "&";
            pending_ref = false;
          }
        }
        break;
      }
    }
  }
  return out;
}

std::string rewrite_pp(const std::string& pp) {
  // #version / #extension / #pragma have no C++ meaning here.
  size_t p = 1;
  while (p < pp.size() && (pp[p] == ' ' || pp[p] == '\t')) ++p;
  size_t q = p;
  while (q < pp.size() && is_ident_char(pp[q])) ++q;
  std::string dir = pp.substr(p, q - p);
  if (dir == "version" || dir == "extension" || dir == "pragma") return "";
  if (dir != "define") return pp;
  // #define NAME[(args)] body: rewrite the body as code
  size_t r = q;
  while (r < pp.size() && (pp[r] == ' ' || pp[r] == '\t')) ++r;
  size_t nm = r;
  while (nm < pp.size() && is_ident_char(pp[nm])) ++nm;
  if (nm < pp.size() && pp[nm] == '(') {
    size_t c = pp.find(')', nm);
    nm = (c == std::string::npos) ? pp.size() : c + 1;
  }
  std::string head = pp.substr(0, nm);
  std::string body = pp.substr(nm);
  std::vector<Tok> bt = tokenize(body);
  return head + rewrite_tokens(bt, 0, bt.size());
}

struct UTypeInfo {
  int kind;
  int components;
  size_t size;
  size_t align;
  const char* cxx;
};

bool uniform_type(const std::string& t, UTypeInfo* u) {
  static const std::map<std::string, UTypeInfo> m = {
      {"float", {UK_FLOAT, 1, 4, 4, "gfloat"}},     {"int", {UK_INT, 1, 4, 4, "int"}},
      {"bool", {UK_BOOL, 1, 4, 4, "int"}},          {"vec2", {UK_VEC2, 2, 8, 4, "vec2"}},
      {"vec3", {UK_VEC3, 3, 12, 4, "vec3"}},        {"vec4", {UK_VEC4, 4, 16, 4, "vec4"}},
      {"ivec2", {UK_IVEC2, 2, 8, 4, "ivec2"}},      {"ivec3", {UK_IVEC3, 3, 12, 4, "ivec3"}},
      {"ivec4", {UK_IVEC4, 4, 16, 4, "ivec4"}},     {"mat2", {UK_MAT2, 4, 16, 4, "mat2"}},
      {"mat3", {UK_MAT3, 9, 36, 4, "mat3"}},        {"mat4", {UK_MAT4, 16, 64, 4, "mat4"}},
      {"sampler2D", {UK_SAMPLER2D, 0, 32, 8, "sampler2D"}},
      {"sampler3D", {UK_SAMPLER3D, 0, 32, 8, "sampler3D"}}};
  auto it = m.find(t);
  if (it == m.end()) return false;
  *u = it->second;
  return true;
}

// GLSL passes out / inout arguments by copy-in, copy-out, so an argument may be any l-value of the
// parameter's type, a swizzle such as `p.xz` included; the C++ rewrite passes them by reference,
// which takes only a variable of that exact type. For a function with out / inout parameters this
// returns a template overload that takes the other arguments: it copies each such argument into a
// temporary of the parameter's type, calls the function with the temporaries and assigns them
// back. The overload is enabled only when some out / inout argument is not an l-value of the
// parameter's own type (glsl::g_copy_in_out), so every call the reference form accepts still
// resolves to the function itself. Returns "" for functions without out / inout parameters and
// for forms it does not handle (array parameters or results).
std::string copy_in_out_overload(const std::vector<Tok>& t, size_t b, size_t open) {
  size_t close = match_close(t, open);
  if (close >= t.size()) return "";
  size_t nm = open;
  while (nm > b && (t[nm - 1].k == T_WS || t[nm - 1].k == T_COMMENT)) --nm;
  if (nm <= b || t[nm - 1].k != T_IDENT) return "";
  // the name the rewrite gave the function (C++-only keywords get the _g suffix)
  const std::string fname = t[nm - 1].s + (cxx_only_keywords().count(t[nm - 1].s) ? "_g" : "");
  std::string ret;
  for (size_t q = b; q < nm - 1; ++q) {
    if (t[q].k == T_PUNCT) return "";  // an array result or something else unexpected
    if (t[q].k == T_IDENT && !dropped_qualifiers().count(t[q].s))
      ret += (ret.empty() ? "" : " ") + (t[q].s == "float" ? std::string("gfloat") : t[q].s);
  }
  if (ret.empty()) return "";
  struct Param {
    std::string type;
    bool byref = false;
  };
  std::vector<Param> ps;
  std::vector<std::string> seg;
  auto flush = [&]() -> bool {
    if (seg.empty()) return true;
    Param p;
    size_t k = 0;
    for (; k < seg.size(); ++k) {
      const std::string& s = seg[k];
      if (s == "out" || s == "inout") p.byref = true;
      else if (s != "in" && s != "const" && !dropped_qualifiers().count(s)) break;
    }
    if (k >= seg.size()) return false;
    p.type = seg[k] == "float" ? "gfloat" : seg[k];
    if (k + 2 < seg.size() || (k + 1 < seg.size() && !is_ident_start(seg[k + 1][0]))) return false;  // arrays
    if (p.type == "void" && seg.size() == 1) {
      seg.clear();
      return true;
    }
    ps.push_back(p);
    seg.clear();
    return true;
  };
  for (size_t q = open + 1; q < close; ++q) {
    if (t[q].k == T_WS || t[q].k == T_COMMENT) continue;
    if (t[q].k == T_PUNCT && t[q].s == ",") {
      if (!flush()) return "";
      continue;
    }
    if (t[q].k == T_PUNCT && t[q].s != "[" && t[q].s != "]") return "";
    seg.push_back(t[q].s);
  }
  if (!flush()) return "";
  bool any = false;
  for (auto& p : ps) any = any || p.byref;
  if (!any) return "";
  const size_t n = ps.size();
  auto A = [](size_t k) { return "A" + std::to_string(k) + "_g"; };
  auto a = [](size_t k) { return "arg" + std::to_string(k) + "_g"; };
  auto tmp = [](size_t k) { return "tmp" + std::to_string(k) + "_g"; };
  std::ostringstream os;
  os << "\n  template <";
  for (size_t k = 0; k < n; ++k) os << "class " << A(k) << ", ";
  os << "typename glsl::g_enable_if<glsl::g_copy_in_out<";
  for (size_t k = 0; k < n; ++k)
    os << (k ? ", " : "") << "glsl::g_param<" << A(k) << ", " << ps[k].type << ", " << (ps[k].byref ? 1 : 0) << ">";
  os << ">::value>::type = 0>\n  " << ret << " " << fname << "(";
  for (size_t k = 0; k < n; ++k) os << (k ? ", " : "") << A(k) << "&& " << a(k);
  os << ") {";
  for (size_t k = 0; k < n; ++k)
    if (ps[k].byref) os << " " << ps[k].type << " " << tmp(k) << "(" << a(k) << ");";
  std::ostringstream call;
  call << fname << "(";
  for (size_t k = 0; k < n; ++k) call << (k ? ", " : "") << (ps[k].byref ? tmp(k) : a(k));
  call << ")";
  const bool is_void = ret == "void";
  os << (is_void ? " " : " auto ret_g = ") << call.str() << ";";
  for (size_t k = 0; k < n; ++k)
    if (ps[k].byref) os << " " << a(k) << " = " << tmp(k) << ";";
  if (!is_void) os << " return ret_g;";
  os << " }\n";
  return os.str();
}

}  // namespace

std::string glsl_rewrite_fragment(const std::string& src) {
  std::vector<Tok> t = tokenize(src);
  return rewrite_tokens(t, 0, t.size());
}

bool glsl_transform(const std::string& src, const std::string& name, const std::string& extra_members,
                    GlslTransformResult* out) {
  *out = GlslTransformResult();
  std::vector<Tok> t = tokenize(src);
  std::map<std::string, long> int_defines;  // simple `#define NAME <int>` for array sizes
  std::string body;                          // struct body (after reference members)
  size_t offset = 0, max_align = 4;
  // identifiers the source uses (macro bodies included) and the names it declares at global
  // scope, to find the renderer uniforms it reads without declaring
  std::set<std::string> referenced, declared;
  for (const Tok& k : t) {
    if (k.k == T_IDENT) referenced.insert(k.s);
    if (k.k == T_PP)
      for (const Tok& q : tokenize(k.s.substr(1)))
        if (q.k == T_IDENT) referenced.insert(q.s);
  }

  size_t i = 0;
  while (i < t.size()) {
    const Tok& k = t[i];
    if (k.k == T_WS || k.k == T_COMMENT) { body += k.s; ++i; continue; }
    if (k.k == T_PP) {
      std::istringstream ss(k.s.substr(1));
      std::string dir, nm, val;
      ss >> dir >> nm >> val;
      if (dir == "define") declared.insert(nm.substr(0, nm.find('(')));
      if (dir == "define" && !val.empty()) {
        char* endp = nullptr;
        long v = std::strtol(val.c_str(), &endp, 0);
        if (endp && *endp == 0) int_defines[nm] = v;
      }
      body += rewrite_pp(k.s);
      ++i;
      continue;
    }
    // collect one global-scope item
    size_t b = i;
    int paren = 0, brace = 0, bracket = 0;
    bool saw_paren_at0 = false, saw_eq_at0 = false, saw_brace = false, is_struct = false;
    size_t first_paren = std::string::npos;
    {
      size_t f = next_sig(t, b);
      if (f < t.size() && t[f].s == "struct") is_struct = true;
    }
    size_t j = i;
    for (; j < t.size(); ++j) {
      const Tok& q = t[j];
      if (q.k != T_PUNCT) continue;
      if (q.s == "(") { if (paren == 0 && brace == 0 && !saw_paren_at0) { saw_paren_at0 = true; first_paren = j; } ++paren; }
      else if (q.s == ")") --paren;
      else if (q.s == "[") ++bracket;
      else if (q.s == "]") --bracket;
      else if (q.s == "{") { ++brace; saw_brace = true; }
      else if (q.s == "}") {
        --brace;
        if (brace == 0 && paren == 0 && !is_struct && saw_paren_at0 && !saw_eq_at0) break;  // function body end
      } else if (q.s == "=" && paren == 0 && brace == 0) saw_eq_at0 = true;
      else if (q.s == ";" && paren == 0 && brace == 0) break;
    }
    size_t e = (j < t.size()) ? j + 1 : t.size();
    // leading qualifier
    size_t f = next_sig(t, b);
    std::string first = (f < e) ? t[f].s : "";
    if (first == "layout") {
      size_t lp = next_sig(t, f + 1);
      if (lp < e && t[lp].s == "(") f = next_sig(t, match_close(t, lp) + 1);
      first = (f < e) ? t[f].s : "";
    }
    if (first == "precision") { i = e; continue; }
    if (first == "uniform") {
      size_t p = next_sig(t, f + 1);
      while (p < e && dropped_qualifiers().count(t[p].s)) p = next_sig(t, p + 1);
      std::string type = (p < e) ? t[p].s : "";
      UTypeInfo ut;
      if (!uniform_type(type, &ut)) {
        out->error = "unsupported uniform type '" + type + "'";
        return false;
      }
      p = next_sig(t, p + 1);
      while (p < e && t[p].s != ";") {
        if (t[p].k != T_IDENT) { out->error = "bad uniform declaration near '" + t[p].s + "'"; return false; }
        GlslUniform u;
        u.name = t[p].s;
        u.glsl_type = type;
        u.kind = ut.kind;
        u.components = ut.components;
        u.elem_size = ut.size;
        p = next_sig(t, p + 1);
        if (p < e && t[p].s == "[") {
          size_t pc = match_close(t, p);
          size_t v = next_sig(t, p + 1);
          long len = -1;
          if (v < pc && t[v].k == T_NUM) len = std::strtol(t[v].s.c_str(), nullptr, 0);
          else if (v < pc && t[v].k == T_IDENT && int_defines.count(t[v].s)) len = int_defines[t[v].s];
          if (len <= 0) { out->error = "uniform array '" + u.name + "' needs a literal size"; return false; }
          u.array_len = (int)len;
          p = next_sig(t, pc + 1);
        }
        offset = (offset + ut.align - 1) / ut.align * ut.align;
        max_align = std::max(max_align, ut.align);
        u.offset = offset;
        offset += ut.size * (u.array_len ? u.array_len : 1);
        out->uniforms.push_back(u);
        if (p < e && t[p].s == ",") p = next_sig(t, p + 1);
      }
      i = e;
      continue;
    }
    if (first == "in" || first == "out" || first == "varying" || first == "attribute") {
      // shader-stage globals become plain members
      body += rewrite_tokens(t, next_sig(t, f + 1), e);
      i = e;
      continue;
    }
    bool is_function = saw_paren_at0 && !saw_eq_at0 && !is_struct && saw_brace;
    bool is_prototype = saw_paren_at0 && !saw_eq_at0 && !is_struct && !saw_brace;
    if (is_function || is_prototype) {
      // the function name is the identifier before the first '(' at depth 0
      size_t q = first_paren;
      while (q > b && (t[q - 1].k == T_WS || t[q - 1].k == T_COMMENT)) --q;
      if (q > b && t[q - 1].k == T_IDENT && is_function) out->functions.push_back(t[q - 1].s);
      if (q > b && t[q - 1].k == T_IDENT) declared.insert(t[q - 1].s);
    } else {
      // a global variable (`[const] T name ...`) or a struct type (`struct S ...`) declares a name
      size_t q = f;
      while (q < e && t[q].k == T_IDENT && (t[q].s == "const" || dropped_qualifiers().count(t[q].s)))
        q = next_sig(t, q + 1);
      const bool st = q < e && t[q].s == "struct";
      size_t r = next_sig(t, q + 1);
      if (st && r < e && t[r].k == T_IDENT) declared.insert(t[r].s);
      else if (!st && r < e && t[r].k == T_IDENT) declared.insert(t[r].s);
    }
    if (is_prototype) { i = e; continue; }
    body += rewrite_tokens(t, b, e);
    if (is_function) body += copy_in_out_overload(t, b, first_paren);
    i = e;
  }

  // renderer uniforms the source reads but does not declare, after its own uniforms
  for (auto& u : out->uniforms) declared.insert(u.name);
  for (const RendererUniform& ru : kRendererUniforms) {
    if (!referenced.count(ru.name) || declared.count(ru.name)) continue;
    UTypeInfo ut;
    uniform_type(ru.glsl_type, &ut);
    GlslUniform u;
    u.name = ru.name;
    u.glsl_type = ru.glsl_type;
    u.kind = ut.kind;
    u.components = ut.components;
    u.elem_size = ut.size;
    offset = (offset + ut.align - 1) / ut.align * ut.align;
    max_align = std::max(max_align, ut.align);
    u.offset = offset;
    offset += ut.size;
    u.params_offset = (long)ru.params_offset;
    out->uniforms.push_back(u);
  }

  size_t block_size = (offset + max_align - 1) / max_align * max_align;
  std::ostringstream os;
  os << "struct " << name << "Uniforms {\n";
  if (out->uniforms.empty()) os << "  int unused_;\n";
  for (auto& u : out->uniforms) {
    UTypeInfo ut;
    uniform_type(u.glsl_type, &ut);
    os << "  " << ut.cxx << " " << u.name;
    if (u.array_len) os << "[" << u.array_len << "]";
    os << ";  // offset " << u.offset << (u.params_offset >= 0 ? ", renderer uniform" : "") << "\n";
  }
  os << "};\n";
  if (out->uniforms.empty()) block_size = 4;
  os << "static_assert(sizeof(" << name << "Uniforms) == " << block_size << ", \"uniform block layout\");\n";
  os << "#ifndef __CUDACC_RTC__\n";  // NVRTC has no offsetof builtin; the host compilers check
  for (auto& u : out->uniforms)
    os << "static_assert(__builtin_offsetof(" << name << "Uniforms, " << u.name << ") == " << u.offset
       << ", \"uniform offset\");\n";
  os << "#endif\n";
  os << "struct " << name << " {\n";
  for (auto& u : out->uniforms) {
    UTypeInfo ut;
    uniform_type(u.glsl_type, &ut);
    if (u.array_len) os << "  const " << ut.cxx << " (&" << u.name << ")[" << u.array_len << "];\n";
    else os << "  const " << ut.cxx << "& " << u.name << ";\n";
  }
  os << "  explicit " << name << "(const " << name << "Uniforms& u__)";
  for (size_t k = 0; k < out->uniforms.size(); ++k)
    os << (k == 0 ? " : " : ", ") << out->uniforms[k].name << "(u__." << out->uniforms[k].name << ")";
  if (out->uniforms.empty()) os << " { (void)u__; }\n";
  else os << " {}\n";
  os << extra_members << "\n";
  os << body << "\n};\n";
  out->code = os.str();
  out->block_size = block_size;
  return true;
}

void fill_renderer_uniforms(const std::vector<GlslUniform>& uniforms, const void* params,
                            std::vector<unsigned char>& block) {
  for (const GlslUniform& u : uniforms)
    if (u.params_offset >= 0 && u.offset + u.elem_size <= block.size() &&
        (size_t)u.params_offset + u.elem_size <= sizeof(SnellyParams))
      std::memcpy(block.data() + u.offset, (const char*)params + u.params_offset, u.elem_size);
}

}  // namespace snelly
