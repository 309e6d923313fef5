// glslcompat.h - GLSL ES 3.00 types and built-in functions for C++ (host) and CUDA (device).
//
// Scene code for the path tracer is written in GLSL (the `SDF_SURFACE`, `SDF_METAL`,
// `SDF_DIELECTRIC` functions and the optional material hooks a scene's `shader()` string
// defines). After a token-level rewrite (glsl_transform.cpp) that code compiles as C++
// against this header: with NVRTC for sm_100a on the GPU, and with g++ for the CPU oracle.
//
// Semantics follow the GLSL ES 3.00 specification:
//   * vec2/vec3/vec4, ivec2/ivec3/ivec4, mat2/mat3/mat4 (column-major, `m * v` and `v * m`);
//   * swizzles through union members (read any, write when components are distinct);
//   * built-ins with GLSL definitions: mod(x,y) = x - y*floor(x/y), fract(x) = x - floor(x),
//     sign, clamp, mix, step, smoothstep, atan(y,x), inversesqrt, reflect, refract, ...;
//   * texture() on sampler2D/sampler3D with GL ES 3.0 LINEAR or NEAREST filtering,
//     CLAMP_TO_EDGE wrapping and texel-centre addressing (the filtering is done in full
//     float precision; hardware samplers use fixed-point weights).
//
// The scalar type `gfloat` is float unless GLSL_SCALAR_DEFINED is set by a header included
// first (the oracle's operation-counting build substitutes a counting type).
#pragma once

#if defined(__CUDACC__) || defined(__CUDACC_RTC__)
#define GLSL_DEVICE 1
#define GLSL_FN __host__ __device__ __forceinline__
#else
#define GLSL_FN inline
#include <cmath>
#include <cstdint>
#endif

namespace glsl {

#ifndef GLSL_SCALAR_DEFINED
typedef float gfloat;

// ---- scalar primitives (float) ------------------------------------------------------------
#ifdef GLSL_DEVICE
GLSL_FN float s_sqrt(float x) { return sqrtf(x); }
GLSL_FN float s_sin(float x) { return sinf(x); }
GLSL_FN float s_cos(float x) { return cosf(x); }
GLSL_FN float s_tan(float x) { return tanf(x); }
GLSL_FN float s_asin(float x) { return asinf(x); }
GLSL_FN float s_acos(float x) { return acosf(x); }
GLSL_FN float s_atan(float x) { return atanf(x); }
GLSL_FN float s_atan2(float y, float x) { return atan2f(y, x); }
GLSL_FN float s_sinh(float x) { return sinhf(x); }
GLSL_FN float s_cosh(float x) { return coshf(x); }
GLSL_FN float s_tanh(float x) { return tanhf(x); }
GLSL_FN float s_exp(float x) { return expf(x); }
GLSL_FN float s_exp2(float x) { return exp2f(x); }
GLSL_FN float s_log(float x) { return logf(x); }
GLSL_FN float s_log2(float x) { return log2f(x); }
GLSL_FN float s_pow(float x, float y) { return powf(x, y); }
GLSL_FN float s_floor(float x) { return floorf(x); }
GLSL_FN float s_ceil(float x) { return ceilf(x); }
GLSL_FN float s_trunc(float x) { return truncf(x); }
GLSL_FN float s_round(float x) { return roundf(x); }
GLSL_FN float s_abs(float x) { return fabsf(x); }
GLSL_FN float s_min(float a, float b) { return fminf(a, b); }
GLSL_FN float s_max(float a, float b) { return fmaxf(a, b); }
GLSL_FN bool s_isnan(float x) { return isnan(x); }
GLSL_FN bool s_isinf(float x) { return isinf(x); }
#else
GLSL_FN float s_sqrt(float x) { return std::sqrt(x); }
GLSL_FN float s_sin(float x) { return std::sin(x); }
GLSL_FN float s_cos(float x) { return std::cos(x); }
GLSL_FN float s_tan(float x) { return std::tan(x); }
GLSL_FN float s_asin(float x) { return std::asin(x); }
GLSL_FN float s_acos(float x) { return std::acos(x); }
GLSL_FN float s_atan(float x) { return std::atan(x); }
GLSL_FN float s_atan2(float y, float x) { return std::atan2(y, x); }
GLSL_FN float s_sinh(float x) { return std::sinh(x); }
GLSL_FN float s_cosh(float x) { return std::cosh(x); }
GLSL_FN float s_tanh(float x) { return std::tanh(x); }
GLSL_FN float s_exp(float x) { return std::exp(x); }
GLSL_FN float s_exp2(float x) { return std::exp2(x); }
GLSL_FN float s_log(float x) { return std::log(x); }
GLSL_FN float s_log2(float x) { return std::log2(x); }
GLSL_FN float s_pow(float x, float y) { return std::pow(x, y); }
GLSL_FN float s_floor(float x) { return std::floor(x); }
GLSL_FN float s_ceil(float x) { return std::ceil(x); }
GLSL_FN float s_trunc(float x) { return std::trunc(x); }
GLSL_FN float s_round(float x) { return std::round(x); }
GLSL_FN float s_abs(float x) { return std::fabs(x); }
GLSL_FN float s_min(float a, float b) { return std::fmin(a, b); }
GLSL_FN float s_max(float a, float b) { return std::fmax(a, b); }
GLSL_FN bool s_isnan(float x) { return std::isnan(x); }
GLSL_FN bool s_isinf(float x) { return std::isinf(x); }
#endif
GLSL_FN float s_tofloat(float x) { return x; }
#endif  // GLSL_SCALAR_DEFINED

struct vec2;
struct vec3;
struct vec4;

// ---- swizzle views ------------------------------------------------------------------------
// swK<N, I...> aliases the float[N] storage of its owning vector and selects components I.
template <int N, int A, int B>
struct sw2 {
  gfloat d[N];
  GLSL_FN operator vec2() const;
  GLSL_FN sw2& operator=(const vec2& v);
  GLSL_FN sw2& operator=(const sw2& o);
  template <class T> GLSL_FN sw2& operator+=(const T& t);
  template <class T> GLSL_FN sw2& operator-=(const T& t);
  template <class T> GLSL_FN sw2& operator*=(const T& t);
  template <class T> GLSL_FN sw2& operator/=(const T& t);
};
template <int N, int A, int B, int C>
struct sw3 {
  gfloat d[N];
  GLSL_FN operator vec3() const;
  GLSL_FN sw3& operator=(const vec3& v);
  GLSL_FN sw3& operator=(const sw3& o);
  template <class T> GLSL_FN sw3& operator+=(const T& t);
  template <class T> GLSL_FN sw3& operator-=(const T& t);
  template <class T> GLSL_FN sw3& operator*=(const T& t);
  template <class T> GLSL_FN sw3& operator/=(const T& t);
};
template <int N, int A, int B, int C, int D>
struct sw4 {
  gfloat d[N];
  GLSL_FN operator vec4() const;
  GLSL_FN sw4& operator=(const vec4& v);
  GLSL_FN sw4& operator=(const sw4& o);
  template <class T> GLSL_FN sw4& operator+=(const T& t);
  template <class T> GLSL_FN sw4& operator-=(const T& t);
  template <class T> GLSL_FN sw4& operator*=(const T& t);
  template <class T> GLSL_FN sw4& operator/=(const T& t);
};

// Single components. With a counting scalar (which has constructors and so cannot live in an
// anonymous struct) each component is a one-element view convertible to a reference to its
// scalar; with float they are plain struct members.
template <int N, int A>
struct sw1 {
  gfloat d[N];
  GLSL_FN operator gfloat&() { return d[A]; }
  GLSL_FN operator const gfloat&() const { return d[A]; }
  GLSL_FN sw1& operator=(gfloat v) { d[A] = v; return *this; }
  GLSL_FN sw1& operator=(const sw1& o) { d[A] = o.d[A]; return *this; }
  GLSL_FN sw1& operator+=(gfloat v) { d[A] = d[A] + v; return *this; }
  GLSL_FN sw1& operator-=(gfloat v) { d[A] = d[A] - v; return *this; }
  GLSL_FN sw1& operator*=(gfloat v) { d[A] = d[A] * v; return *this; }
  GLSL_FN sw1& operator/=(gfloat v) { d[A] = d[A] / v; return *this; }
};
#ifdef GLSL_SCALAR_DEFINED
#define GLSL_COMPONENTS2 sw1<2, 0> x, r, s; sw1<2, 1> y, g, t;
#define GLSL_COMPONENTS3 sw1<3, 0> x, r, s; sw1<3, 1> y, g, t; sw1<3, 2> z, b, p;
#define GLSL_COMPONENTS4 sw1<4, 0> x, r, s; sw1<4, 1> y, g, t; sw1<4, 2> z, b, p; sw1<4, 3> w, a, q;
#else
#define GLSL_COMPONENTS2 struct { gfloat x, y; }; struct { gfloat r, g; }; struct { gfloat s, t; };
#define GLSL_COMPONENTS3 struct { gfloat x, y, z; }; struct { gfloat r, g, b; }; struct { gfloat s, t, p; };
#define GLSL_COMPONENTS4 \
  struct { gfloat x, y, z, w; }; struct { gfloat r, g, b, a; }; struct { gfloat s, t, p, q; };
#endif

#if defined(__GNUC__) && !defined(__CUDACC_RTC__)
#pragma GCC diagnostic push
#pragma GCC diagnostic ignored "-Wpedantic"
#endif

struct vec2 {
  union {
    gfloat d[2];
    GLSL_COMPONENTS2
#define GLSL_SWIZZLE_STORAGE 2
#include "glsl_swizzles.inc"
#undef GLSL_SWIZZLE_STORAGE
  };
  // GLSL locals are zero-initialised by WebGL implementations; follow that.
  GLSL_FN vec2() { x = gfloat(0); y = gfloat(0); }
  GLSL_FN explicit vec2(gfloat a) { x = a; y = a; }
  GLSL_FN vec2(gfloat a, gfloat b) { x = a; y = b; }
  GLSL_FN explicit vec2(const vec3& v);
  GLSL_FN explicit vec2(const vec4& v);
  // a constructor may take only the leading components of its last argument (GLSL ES 3.00 5.4.2)
  GLSL_FN vec2(gfloat a, const vec2& v) { x = a; y = v.x; }
  // float(v): the first component
  GLSL_FN explicit operator gfloat() const { return d[0]; }
  GLSL_FN vec2& operator=(const vec2& o) { x = o.x; y = o.y; return *this; }
  GLSL_FN gfloat& operator[](int i) { return d[i]; }
  GLSL_FN const gfloat& operator[](int i) const { return d[i]; }
  GLSL_FN vec2& operator+=(const vec2& o) { x = x + o.x; y = y + o.y; return *this; }
  GLSL_FN vec2& operator-=(const vec2& o) { x = x - o.x; y = y - o.y; return *this; }
  GLSL_FN vec2& operator*=(const vec2& o) { x = x * o.x; y = y * o.y; return *this; }
  GLSL_FN vec2& operator/=(const vec2& o) { x = x / o.x; y = y / o.y; return *this; }
  GLSL_FN vec2& operator+=(gfloat a) { x = x + a; y = y + a; return *this; }
  GLSL_FN vec2& operator-=(gfloat a) { x = x - a; y = y - a; return *this; }
  GLSL_FN vec2& operator*=(gfloat a) { x = x * a; y = y * a; return *this; }
  GLSL_FN vec2& operator/=(gfloat a) { x = x / a; y = y / a; return *this; }
};

struct vec3 {
  union {
    gfloat d[3];
    GLSL_COMPONENTS3
#define GLSL_SWIZZLE_STORAGE 3
#include "glsl_swizzles.inc"
#undef GLSL_SWIZZLE_STORAGE
  };
  GLSL_FN vec3() { x = gfloat(0); y = gfloat(0); z = gfloat(0); }
  GLSL_FN explicit vec3(gfloat a) { x = a; y = a; z = a; }
  GLSL_FN vec3(gfloat a, gfloat b, gfloat c) { x = a; y = b; z = c; }
  GLSL_FN vec3(const vec2& v, gfloat c) { x = v.x; y = v.y; z = c; }
  GLSL_FN vec3(gfloat a, const vec2& v) { x = a; y = v.x; z = v.y; }
  GLSL_FN explicit vec3(const vec4& v);
  GLSL_FN vec3(gfloat a, gfloat b, const vec2& v) { x = a; y = b; z = v.x; }
  GLSL_FN vec3(gfloat a, gfloat b, const vec3& v) { x = a; y = b; z = v.x; }
  GLSL_FN vec3(const vec2& u, const vec2& v) { x = u.x; y = u.y; z = v.x; }
  GLSL_FN vec3(gfloat a, const vec3& v) { x = a; y = v.x; z = v.y; }
  GLSL_FN explicit operator gfloat() const { return d[0]; }
  GLSL_FN vec3& operator=(const vec3& o) { x = o.x; y = o.y; z = o.z; return *this; }
  GLSL_FN gfloat& operator[](int i) { return d[i]; }
  GLSL_FN const gfloat& operator[](int i) const { return d[i]; }
  GLSL_FN vec3& operator+=(const vec3& o) { x = x + o.x; y = y + o.y; z = z + o.z; return *this; }
  GLSL_FN vec3& operator-=(const vec3& o) { x = x - o.x; y = y - o.y; z = z - o.z; return *this; }
  GLSL_FN vec3& operator*=(const vec3& o) { x = x * o.x; y = y * o.y; z = z * o.z; return *this; }
  GLSL_FN vec3& operator/=(const vec3& o) { x = x / o.x; y = y / o.y; z = z / o.z; return *this; }
  GLSL_FN vec3& operator+=(gfloat a) { x = x + a; y = y + a; z = z + a; return *this; }
  GLSL_FN vec3& operator-=(gfloat a) { x = x - a; y = y - a; z = z - a; return *this; }
  GLSL_FN vec3& operator*=(gfloat a) { x = x * a; y = y * a; z = z * a; return *this; }
  GLSL_FN vec3& operator/=(gfloat a) { x = x / a; y = y / a; z = z / a; return *this; }
  GLSL_FN vec3& operator*=(const struct mat3& m);
};

struct vec4 {
  union {
    gfloat d[4];
    GLSL_COMPONENTS4
#define GLSL_SWIZZLE_STORAGE 4
#include "glsl_swizzles.inc"
#undef GLSL_SWIZZLE_STORAGE
  };
  GLSL_FN vec4() { x = gfloat(0); y = gfloat(0); z = gfloat(0); w = gfloat(0); }
  GLSL_FN explicit vec4(gfloat v) { x = v; y = v; z = v; w = v; }
  GLSL_FN vec4(gfloat a_, gfloat b_, gfloat c_, gfloat d_) { x = a_; y = b_; z = c_; w = d_; }
  GLSL_FN vec4(const vec3& v, gfloat c) { x = v.x; y = v.y; z = v.z; w = c; }
  GLSL_FN vec4(gfloat c, const vec3& v) { x = c; y = v.x; z = v.y; w = v.z; }
  GLSL_FN vec4(const vec2& u, const vec2& v) { x = u.x; y = u.y; z = v.x; w = v.y; }
  GLSL_FN vec4(const vec2& u, gfloat c, gfloat e) { x = u.x; y = u.y; z = c; w = e; }
  GLSL_FN vec4(gfloat c, gfloat e, const vec2& u) { x = c; y = e; z = u.x; w = u.y; }
  GLSL_FN vec4(gfloat c, const vec2& u, gfloat e) { x = c; y = u.x; z = u.y; w = e; }
  GLSL_FN vec4(gfloat a_, gfloat b_, gfloat c_, const vec2& v) { x = a_; y = b_; z = c_; w = v.x; }
  GLSL_FN vec4(gfloat a_, gfloat b_, gfloat c_, const vec3& v) { x = a_; y = b_; z = c_; w = v.x; }
  GLSL_FN vec4(gfloat a_, gfloat b_, const vec3& v) { x = a_; y = b_; z = v.x; w = v.y; }
  GLSL_FN vec4(const vec3& u, const vec2& v) { x = u.x; y = u.y; z = u.z; w = v.x; }
  GLSL_FN vec4(const vec3& u, const vec3& v) { x = u.x; y = u.y; z = u.z; w = v.x; }
  GLSL_FN vec4(const vec2& u, const vec3& v) { x = u.x; y = u.y; z = v.x; w = v.y; }
  GLSL_FN explicit operator gfloat() const { return d[0]; }
  GLSL_FN vec4& operator=(const vec4& o) { x = o.x; y = o.y; z = o.z; w = o.w; return *this; }
  GLSL_FN gfloat& operator[](int i) { return d[i]; }
  GLSL_FN const gfloat& operator[](int i) const { return d[i]; }
  GLSL_FN vec4& operator+=(const vec4& o) { x = x + o.x; y = y + o.y; z = z + o.z; w = w + o.w; return *this; }
  GLSL_FN vec4& operator-=(const vec4& o) { x = x - o.x; y = y - o.y; z = z - o.z; w = w - o.w; return *this; }
  GLSL_FN vec4& operator*=(const vec4& o) { x = x * o.x; y = y * o.y; z = z * o.z; w = w * o.w; return *this; }
  GLSL_FN vec4& operator/=(const vec4& o) { x = x / o.x; y = y / o.y; z = z / o.z; w = w / o.w; return *this; }
  GLSL_FN vec4& operator+=(gfloat v) { x = x + v; y = y + v; z = z + v; w = w + v; return *this; }
  GLSL_FN vec4& operator-=(gfloat v) { x = x - v; y = y - v; z = z - v; w = w - v; return *this; }
  GLSL_FN vec4& operator*=(gfloat v) { x = x * v; y = y * v; z = z * v; w = w * v; return *this; }
  GLSL_FN vec4& operator/=(gfloat v) { x = x / v; y = y / v; z = z / v; w = w / v; return *this; }
  GLSL_FN vec4& operator*=(const struct mat4& m);
};

#if defined(__GNUC__) && !defined(__CUDACC_RTC__)
#pragma GCC diagnostic pop
#endif

GLSL_FN vec2::vec2(const vec3& v) { x = v.x; y = v.y; }
GLSL_FN vec2::vec2(const vec4& v) { x = v.x; y = v.y; }
GLSL_FN vec3::vec3(const vec4& v) { x = v.x; y = v.y; z = v.z; }

// ---- swizzle view members -----------------------------------------------------------------
template <int N, int A, int B>
GLSL_FN sw2<N, A, B>::operator vec2() const { return vec2(d[A], d[B]); }
template <int N, int A, int B>
GLSL_FN sw2<N, A, B>& sw2<N, A, B>::operator=(const vec2& v) {
  static_assert(A != B, "swizzle with repeated components is not assignable");
  gfloat a = v.x, b = v.y; d[A] = a; d[B] = b; return *this;
}
template <int N, int A, int B>
GLSL_FN sw2<N, A, B>& sw2<N, A, B>::operator=(const sw2& o) { return *this = vec2(o); }
template <int N, int A, int B, int C>
GLSL_FN sw3<N, A, B, C>::operator vec3() const { return vec3(d[A], d[B], d[C]); }
template <int N, int A, int B, int C>
GLSL_FN sw3<N, A, B, C>& sw3<N, A, B, C>::operator=(const vec3& v) {
  static_assert(A != B && A != C && B != C, "swizzle with repeated components is not assignable");
  gfloat a = v.x, b = v.y, c = v.z; d[A] = a; d[B] = b; d[C] = c; return *this;
}
template <int N, int A, int B, int C>
GLSL_FN sw3<N, A, B, C>& sw3<N, A, B, C>::operator=(const sw3& o) { return *this = vec3(o); }
template <int N, int A, int B, int C, int D>
GLSL_FN sw4<N, A, B, C, D>::operator vec4() const { return vec4(d[A], d[B], d[C], d[D]); }
template <int N, int A, int B, int C, int D>
GLSL_FN sw4<N, A, B, C, D>& sw4<N, A, B, C, D>::operator=(const vec4& v) {
  static_assert(A != B && A != C && A != D && B != C && B != D && C != D,
                "swizzle with repeated components is not assignable");
  gfloat a = v.x, b = v.y, c = v.z, e = v.w; d[A] = a; d[B] = b; d[C] = c; d[D] = e; return *this;
}
template <int N, int A, int B, int C, int D>
GLSL_FN sw4<N, A, B, C, D>& sw4<N, A, B, C, D>::operator=(const sw4& o) { return *this = vec4(o); }

// ---- arithmetic ---------------------------------------------------------------------------
#define GLSL_VEC_BINOP(V, OP)                                                           \
  GLSL_FN V operator OP(const V& a, const V& b) { V r(a); r OP## = b; return r; }       \
  GLSL_FN V operator OP(const V& a, gfloat s) { V r(a); r OP## = s; return r; }         \
  GLSL_FN V operator OP(gfloat s, const V& b) { V r(s); r OP## = b; return r; }
#define GLSL_VEC_OPS(V)                                                                 \
  GLSL_VEC_BINOP(V, +) GLSL_VEC_BINOP(V, -) GLSL_VEC_BINOP(V, *) GLSL_VEC_BINOP(V, /)
GLSL_VEC_OPS(vec2)
GLSL_VEC_OPS(vec3)
GLSL_VEC_OPS(vec4)
#undef GLSL_VEC_OPS
#undef GLSL_VEC_BINOP

GLSL_FN vec2 operator-(const vec2& a) { return vec2(-a.x, -a.y); }
GLSL_FN vec3 operator-(const vec3& a) { return vec3(-a.x, -a.y, -a.z); }
GLSL_FN vec4 operator-(const vec4& a) { return vec4(-a.x, -a.y, -a.z, -a.w); }
GLSL_FN vec2 operator+(const vec2& a) { return a; }
GLSL_FN vec3 operator+(const vec3& a) { return a; }
GLSL_FN vec4 operator+(const vec4& a) { return a; }
GLSL_FN bool operator==(const vec2& a, const vec2& b) { return a.x == b.x && a.y == b.y; }
GLSL_FN bool operator==(const vec3& a, const vec3& b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
GLSL_FN bool operator==(const vec4& a, const vec4& b) {
  return a.x == b.x && a.y == b.y && a.z == b.z && a.w == b.w;
}
GLSL_FN bool operator!=(const vec2& a, const vec2& b) { return !(a == b); }
GLSL_FN bool operator!=(const vec3& a, const vec3& b) { return !(a == b); }
GLSL_FN bool operator!=(const vec4& a, const vec4& b) { return !(a == b); }

#define GLSL_SW_COMPOUND(SW, V, TPL, ARGS)                                              \
  template <TPL> template <class T>                                                     \
  GLSL_FN SW<ARGS>& SW<ARGS>::operator+=(const T& t) { return *this = V(*this) + t; }   \
  template <TPL> template <class T>                                                     \
  GLSL_FN SW<ARGS>& SW<ARGS>::operator-=(const T& t) { return *this = V(*this) - t; }   \
  template <TPL> template <class T>                                                     \
  GLSL_FN SW<ARGS>& SW<ARGS>::operator*=(const T& t) { return *this = V(*this) * t; }   \
  template <TPL> template <class T>                                                     \
  GLSL_FN SW<ARGS>& SW<ARGS>::operator/=(const T& t) { return *this = V(*this) / t; }
#define GLSL_COMMA ,
GLSL_SW_COMPOUND(sw2, vec2, int N GLSL_COMMA int A GLSL_COMMA int B, N GLSL_COMMA A GLSL_COMMA B)
GLSL_SW_COMPOUND(sw3, vec3, int N GLSL_COMMA int A GLSL_COMMA int B GLSL_COMMA int C,
                 N GLSL_COMMA A GLSL_COMMA B GLSL_COMMA C)
GLSL_SW_COMPOUND(sw4, vec4,
                 int N GLSL_COMMA int A GLSL_COMMA int B GLSL_COMMA int C GLSL_COMMA int D,
                 N GLSL_COMMA A GLSL_COMMA B GLSL_COMMA C GLSL_COMMA D)
#undef GLSL_SW_COMPOUND

// ---- integer / boolean vectors (no swizzles) ----------------------------------------------
struct ivec2 {
  int x, y;
  GLSL_FN ivec2() : x(0), y(0) {}
  GLSL_FN explicit ivec2(int a) : x(a), y(a) {}
  GLSL_FN ivec2(int a, int b) : x(a), y(b) {}
  GLSL_FN explicit ivec2(const vec2& v) : x(int(s_tofloat(v.x))), y(int(s_tofloat(v.y))) {}
  GLSL_FN int& operator[](int i) { return i == 0 ? x : y; }
  GLSL_FN int operator[](int i) const { return i == 0 ? x : y; }
  GLSL_FN explicit operator vec2() const;
};
struct ivec3 {
  int x, y, z;
  GLSL_FN ivec3() : x(0), y(0), z(0) {}
  GLSL_FN explicit ivec3(int a) : x(a), y(a), z(a) {}
  GLSL_FN ivec3(int a, int b, int c) : x(a), y(b), z(c) {}
  GLSL_FN explicit ivec3(const vec3& v)
      : x(int(s_tofloat(v.x))), y(int(s_tofloat(v.y))), z(int(s_tofloat(v.z))) {}
  GLSL_FN int& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  GLSL_FN int operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  GLSL_FN explicit operator vec3() const;
};
struct ivec4 {
  int x, y, z, w;
  GLSL_FN ivec4() : x(0), y(0), z(0), w(0) {}
  GLSL_FN explicit ivec4(int a) : x(a), y(a), z(a), w(a) {}
  GLSL_FN ivec4(int a, int b, int c, int e) : x(a), y(b), z(c), w(e) {}
  GLSL_FN explicit operator vec4() const;
};
struct bvec2 {
  bool x, y;
  GLSL_FN explicit operator vec2() const;
};
struct bvec3 {
  bool x, y, z;
  GLSL_FN explicit operator vec3() const;
};
struct bvec4 {
  bool x, y, z, w;
  GLSL_FN explicit operator vec4() const;
};
// float vectors from integer and boolean ones: vec3(ivec3(i, j, k)), vec4(bvec4(...)) (0 or 1)
GLSL_FN vec2 to_vec(const ivec2& v) { return vec2(gfloat(float(v.x)), gfloat(float(v.y))); }
GLSL_FN vec3 to_vec(const ivec3& v) { return vec3(gfloat(float(v.x)), gfloat(float(v.y)), gfloat(float(v.z))); }
GLSL_FN vec4 to_vec(const ivec4& v) {
  return vec4(gfloat(float(v.x)), gfloat(float(v.y)), gfloat(float(v.z)), gfloat(float(v.w)));
}
GLSL_FN vec2 to_vec(const bvec2& v) { return to_vec(ivec2(v.x, v.y)); }
GLSL_FN vec3 to_vec(const bvec3& v) { return to_vec(ivec3(v.x, v.y, v.z)); }
GLSL_FN vec4 to_vec(const bvec4& v) { return to_vec(ivec4(v.x, v.y, v.z, v.w)); }
GLSL_FN ivec2::operator vec2() const { return to_vec(*this); }
GLSL_FN ivec3::operator vec3() const { return to_vec(*this); }
GLSL_FN ivec4::operator vec4() const { return to_vec(*this); }
GLSL_FN bvec2::operator vec2() const { return to_vec(*this); }
GLSL_FN bvec3::operator vec3() const { return to_vec(*this); }
GLSL_FN bvec4::operator vec4() const { return to_vec(*this); }
// component-wise comparisons and their reductions (GLSL ES 3.00 8.7); `not` is `not_g` after the
// translator's renaming of C++ keywords
#define GLSL_REL(NAME, OP)                                                                           \
  GLSL_FN bvec2 NAME(const vec2& a, const vec2& b) { return bvec2{a.x OP b.x, a.y OP b.y}; }        \
  GLSL_FN bvec3 NAME(const vec3& a, const vec3& b) { return bvec3{a.x OP b.x, a.y OP b.y, a.z OP b.z}; } \
  GLSL_FN bvec4 NAME(const vec4& a, const vec4& b) {                                                \
    return bvec4{a.x OP b.x, a.y OP b.y, a.z OP b.z, a.w OP b.w};                                   \
  }                                                                                                 \
  GLSL_FN bvec2 NAME(const ivec2& a, const ivec2& b) { return bvec2{a.x OP b.x, a.y OP b.y}; }      \
  GLSL_FN bvec3 NAME(const ivec3& a, const ivec3& b) { return bvec3{a.x OP b.x, a.y OP b.y, a.z OP b.z}; } \
  GLSL_FN bvec4 NAME(const ivec4& a, const ivec4& b) {                                              \
    return bvec4{a.x OP b.x, a.y OP b.y, a.z OP b.z, a.w OP b.w};                                   \
  }
GLSL_REL(lessThan, <)
GLSL_REL(lessThanEqual, <=)
GLSL_REL(greaterThan, >)
GLSL_REL(greaterThanEqual, >=)
GLSL_REL(equal, ==)
GLSL_REL(notEqual, !=)
#undef GLSL_REL
GLSL_FN bool any(const bvec2& v) { return v.x || v.y; }
GLSL_FN bool any(const bvec3& v) { return v.x || v.y || v.z; }
GLSL_FN bool any(const bvec4& v) { return v.x || v.y || v.z || v.w; }
GLSL_FN bool all(const bvec2& v) { return v.x && v.y; }
GLSL_FN bool all(const bvec3& v) { return v.x && v.y && v.z; }
GLSL_FN bool all(const bvec4& v) { return v.x && v.y && v.z && v.w; }
GLSL_FN bvec2 not_g(const bvec2& v) { return bvec2{!v.x, !v.y}; }
GLSL_FN bvec3 not_g(const bvec3& v) { return bvec3{!v.x, !v.y, !v.z}; }
GLSL_FN bvec4 not_g(const bvec4& v) { return bvec4{!v.x, !v.y, !v.z, !v.w}; }

// ---- matrices (column-major) --------------------------------------------------------------
struct mat2 {
  vec2 c[2];
  mat2() = default;
  GLSL_FN explicit mat2(gfloat s) { c[0] = vec2(s, gfloat(0)); c[1] = vec2(gfloat(0), s); }
  GLSL_FN mat2(gfloat a, gfloat b, gfloat e, gfloat f) { c[0] = vec2(a, b); c[1] = vec2(e, f); }
  GLSL_FN mat2(const vec2& a, const vec2& b) { c[0] = a; c[1] = b; }
  GLSL_FN mat2& operator=(const mat2& o) { c[0] = o.c[0]; c[1] = o.c[1]; return *this; }
  GLSL_FN vec2& operator[](int i) { return c[i]; }
  GLSL_FN const vec2& operator[](int i) const { return c[i]; }
};
struct mat3 {
  vec3 c[3];
  mat3() = default;
  GLSL_FN explicit mat3(gfloat s) {
    c[0] = vec3(s, gfloat(0), gfloat(0)); c[1] = vec3(gfloat(0), s, gfloat(0)); c[2] = vec3(gfloat(0), gfloat(0), s);
  }
  GLSL_FN mat3(gfloat a0, gfloat a1, gfloat a2, gfloat b0, gfloat b1, gfloat b2, gfloat c0, gfloat c1, gfloat c2) {
    c[0] = vec3(a0, a1, a2); c[1] = vec3(b0, b1, b2); c[2] = vec3(c0, c1, c2);
  }
  GLSL_FN mat3(const vec3& a, const vec3& b, const vec3& e) { c[0] = a; c[1] = b; c[2] = e; }
  GLSL_FN explicit mat3(const struct mat4& m);
  GLSL_FN mat3& operator=(const mat3& o) { c[0] = o.c[0]; c[1] = o.c[1]; c[2] = o.c[2]; return *this; }
  GLSL_FN vec3& operator[](int i) { return c[i]; }
  GLSL_FN const vec3& operator[](int i) const { return c[i]; }
};
struct mat4 {
  vec4 c[4];
  mat4() = default;
  GLSL_FN explicit mat4(gfloat s) {
    gfloat z(0);
    c[0] = vec4(s, z, z, z); c[1] = vec4(z, s, z, z); c[2] = vec4(z, z, s, z); c[3] = vec4(z, z, z, s);
  }
  GLSL_FN mat4(const vec4& a, const vec4& b, const vec4& e, const vec4& f) { c[0] = a; c[1] = b; c[2] = e; c[3] = f; }
  GLSL_FN mat4(gfloat a0, gfloat a1, gfloat a2, gfloat a3, gfloat b0, gfloat b1, gfloat b2, gfloat b3,
               gfloat c0, gfloat c1, gfloat c2, gfloat c3, gfloat d0, gfloat d1, gfloat d2, gfloat d3) {
    c[0] = vec4(a0, a1, a2, a3); c[1] = vec4(b0, b1, b2, b3); c[2] = vec4(c0, c1, c2, c3); c[3] = vec4(d0, d1, d2, d3);
  }
  GLSL_FN mat4& operator=(const mat4& o) { for (int i = 0; i < 4; ++i) c[i] = o.c[i]; return *this; }
  GLSL_FN vec4& operator[](int i) { return c[i]; }
  GLSL_FN const vec4& operator[](int i) const { return c[i]; }
};
GLSL_FN mat3::mat3(const mat4& m) { c[0] = vec3(m.c[0]); c[1] = vec3(m.c[1]); c[2] = vec3(m.c[2]); }

GLSL_FN gfloat dot(const vec2& a, const vec2& b) { return a.x * b.x + a.y * b.y; }
GLSL_FN gfloat dot(const vec3& a, const vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
GLSL_FN gfloat dot(const vec4& a, const vec4& b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
GLSL_FN gfloat dot(gfloat a, gfloat b) { return a * b; }

// m * v: linear combination of columns; v * m: dot with each column.
GLSL_FN vec2 operator*(const mat2& m, const vec2& v) { return m.c[0] * v.x + m.c[1] * v.y; }
GLSL_FN vec3 operator*(const mat3& m, const vec3& v) { return m.c[0] * v.x + m.c[1] * v.y + m.c[2] * v.z; }
GLSL_FN vec4 operator*(const mat4& m, const vec4& v) {
  return m.c[0] * v.x + m.c[1] * v.y + m.c[2] * v.z + m.c[3] * v.w;
}
GLSL_FN vec2 operator*(const vec2& v, const mat2& m) { return vec2(dot(v, m.c[0]), dot(v, m.c[1])); }
GLSL_FN vec3 operator*(const vec3& v, const mat3& m) {
  return vec3(dot(v, m.c[0]), dot(v, m.c[1]), dot(v, m.c[2]));
}
GLSL_FN vec4 operator*(const vec4& v, const mat4& m) {
  return vec4(dot(v, m.c[0]), dot(v, m.c[1]), dot(v, m.c[2]), dot(v, m.c[3]));
}
GLSL_FN mat2 operator*(const mat2& a, const mat2& b) { return mat2(a * b.c[0], a * b.c[1]); }
GLSL_FN mat3 operator*(const mat3& a, const mat3& b) { return mat3(a * b.c[0], a * b.c[1], a * b.c[2]); }
GLSL_FN mat4 operator*(const mat4& a, const mat4& b) {
  return mat4(a * b.c[0], a * b.c[1], a * b.c[2], a * b.c[3]);
}
GLSL_FN mat2 operator*(const mat2& a, gfloat s) { return mat2(a.c[0] * s, a.c[1] * s); }
GLSL_FN mat3 operator*(const mat3& a, gfloat s) { return mat3(a.c[0] * s, a.c[1] * s, a.c[2] * s); }
GLSL_FN mat4 operator*(const mat4& a, gfloat s) { return mat4(a.c[0] * s, a.c[1] * s, a.c[2] * s, a.c[3] * s); }
GLSL_FN mat2 operator*(gfloat s, const mat2& a) { return a * s; }
GLSL_FN mat3 operator*(gfloat s, const mat3& a) { return a * s; }
GLSL_FN mat4 operator*(gfloat s, const mat4& a) { return a * s; }
GLSL_FN mat2 operator+(const mat2& a, const mat2& b) { return mat2(a.c[0] + b.c[0], a.c[1] + b.c[1]); }
GLSL_FN mat3 operator+(const mat3& a, const mat3& b) {
  return mat3(a.c[0] + b.c[0], a.c[1] + b.c[1], a.c[2] + b.c[2]);
}
GLSL_FN mat4 operator+(const mat4& a, const mat4& b) {
  return mat4(a.c[0] + b.c[0], a.c[1] + b.c[1], a.c[2] + b.c[2], a.c[3] + b.c[3]);
}
GLSL_FN vec3& vec3::operator*=(const mat3& m) { return *this = (*this) * m; }
GLSL_FN vec4& vec4::operator*=(const mat4& m) { return *this = (*this) * m; }
// the remaining component-wise matrix operators and the compound assignments GLSL defines
// (m *= n is m = m * n, the linear-algebra product)
GLSL_FN mat2 operator/(const mat2& a, gfloat s) { return mat2(a.c[0] / s, a.c[1] / s); }
GLSL_FN mat3 operator/(const mat3& a, gfloat s) { return mat3(a.c[0] / s, a.c[1] / s, a.c[2] / s); }
GLSL_FN mat4 operator/(const mat4& a, gfloat s) { return mat4(a.c[0] / s, a.c[1] / s, a.c[2] / s, a.c[3] / s); }
#define GLSL_MAT_OPS(M)                                                                   \
  GLSL_FN M operator-(const M& a) { return a * gfloat(-1); }                              \
  GLSL_FN M operator-(const M& a, const M& b) { return a + (-b); }                        \
  GLSL_FN M& operator*=(M& a, gfloat s) { return a = a * s; }                             \
  GLSL_FN M& operator/=(M& a, gfloat s) { return a = a / s; }                             \
  GLSL_FN M& operator*=(M& a, const M& b) { return a = a * b; }                           \
  GLSL_FN M& operator+=(M& a, const M& b) { return a = a + b; }                           \
  GLSL_FN M& operator-=(M& a, const M& b) { return a = a - b; }
GLSL_MAT_OPS(mat2)
GLSL_MAT_OPS(mat3)
GLSL_MAT_OPS(mat4)
#undef GLSL_MAT_OPS
GLSL_FN mat2 transpose(const mat2& m) { return mat2(m.c[0].x, m.c[1].x, m.c[0].y, m.c[1].y); }
GLSL_FN mat3 transpose(const mat3& m) {
  return mat3(m.c[0].x, m.c[1].x, m.c[2].x, m.c[0].y, m.c[1].y, m.c[2].y, m.c[0].z, m.c[1].z, m.c[2].z);
}
GLSL_FN mat4 transpose(const mat4& m) {
  mat4 r;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) r.c[i][j] = m.c[j][i];
  return r;
}
GLSL_FN gfloat determinant(const mat2& m) { return m.c[0].x * m.c[1].y - m.c[1].x * m.c[0].y; }
GLSL_FN gfloat determinant(const mat3& m) {
  return m.c[0].x * (m.c[1].y * m.c[2].z - m.c[2].y * m.c[1].z) -
         m.c[1].x * (m.c[0].y * m.c[2].z - m.c[2].y * m.c[0].z) +
         m.c[2].x * (m.c[0].y * m.c[1].z - m.c[1].y * m.c[0].z);
}
GLSL_FN mat2 inverse(const mat2& m) {
  gfloat id = gfloat(1) / determinant(m);
  return mat2(m.c[1].y * id, -m.c[0].y * id, -m.c[1].x * id, m.c[0].x * id);
}
GLSL_FN mat3 inverse(const mat3& m) {
  // adjugate / determinant, written with cofactors of the column-major storage
  const vec3 &a = m.c[0], &b = m.c[1], &e = m.c[2];
  vec3 r0(b.y * e.z - e.y * b.z, e.y * a.z - a.y * e.z, a.y * b.z - b.y * a.z);
  vec3 r1(e.x * b.z - b.x * e.z, a.x * e.z - e.x * a.z, b.x * a.z - a.x * b.z);
  vec3 r2(b.x * e.y - e.x * b.y, e.x * a.y - a.x * e.y, a.x * b.y - b.x * a.y);
  gfloat id = gfloat(1) / (a.x * r0.x + b.x * r0.y + e.x * r0.z);
  return mat3(r0 * id, r1 * id, r2 * id);
}

// ---- out / inout arguments ----------------------------------------------------------------
// The translator gives each scene function with out / inout parameters a template overload
// that passes those arguments by copy-in, copy-out, as GLSL does, so that a swizzle or a
// component view can be passed (f(p.xz) writes back into p). These traits decide which calls it
// takes: every argument must convert to its parameter's type, every out / inout argument must
// also take the result back by assignment, and at least one out / inout argument must not be an
// l-value of the parameter's own type (those calls go to the function itself).
#ifdef GLSL_DEVICE
#define GLSL_DECL __host__ __device__
#else
#define GLSL_DECL
#endif
template <class T> GLSL_DECL T&& g_declval() noexcept;  // unevaluated use only
template <bool B> struct g_enable_if {};
template <> struct g_enable_if<true> { typedef int type; };
template <class A, class B> struct g_same { static constexpr bool value = false; };
template <class A> struct g_same<A, A> { static constexpr bool value = true; };
template <class T> struct g_sink { GLSL_DECL static char take(T); };  // unevaluated use only
template <class A, class T, class = void> struct g_converts { static constexpr bool value = false; };
template <class A, class T>
struct g_converts<A, T, decltype(void(g_sink<T>::take(g_declval<A>())))> { static constexpr bool value = true; };
template <class A, class T, class = void> struct g_assigns { static constexpr bool value = false; };
template <class A, class T>
struct g_assigns<A, T, decltype(void(g_declval<A>() = g_declval<const T&>()))> { static constexpr bool value = true; };
template <class A, class T, int ByRef> struct g_param;
template <class A, class T> struct g_param<A, T, 0> {
  static constexpr bool ok = g_converts<A, T>::value;
  static constexpr bool exact = true;
};
template <class A, class T> struct g_param<A, T, 1> {
  static constexpr bool ok = g_converts<A, T>::value && g_assigns<A, T>::value;
  static constexpr bool exact = g_same<A, T&>::value;
};
template <class... P> struct g_copy_in_out_all { static constexpr bool ok = true, exact = true; };
template <class P, class... R> struct g_copy_in_out_all<P, R...> {
  static constexpr bool ok = P::ok && g_copy_in_out_all<R...>::ok;
  static constexpr bool exact = P::exact && g_copy_in_out_all<R...>::exact;
};
template <class... P> struct g_copy_in_out {
  static constexpr bool value = g_copy_in_out_all<P...>::ok && !g_copy_in_out_all<P...>::exact;
};
#undef GLSL_DECL

// ---- built-in functions -------------------------------------------------------------------
#define GLSL_MAP1(NAME, IMPL)                                                                  \
  GLSL_FN gfloat NAME(gfloat a) { return IMPL(a); }                                            \
  GLSL_FN vec2 NAME(const vec2& a) { return vec2(IMPL(a.x), IMPL(a.y)); }                      \
  GLSL_FN vec3 NAME(const vec3& a) { return vec3(IMPL(a.x), IMPL(a.y), IMPL(a.z)); }           \
  GLSL_FN vec4 NAME(const vec4& a) { return vec4(IMPL(a.x), IMPL(a.y), IMPL(a.z), IMPL(a.w)); }
#define GLSL_MAP2(NAME, IMPL)                                                                  \
  GLSL_FN gfloat NAME(gfloat a, gfloat b) { return IMPL(a, b); }                               \
  GLSL_FN vec2 NAME(const vec2& a, const vec2& b) { return vec2(IMPL(a.x, b.x), IMPL(a.y, b.y)); } \
  GLSL_FN vec3 NAME(const vec3& a, const vec3& b) {                                            \
    return vec3(IMPL(a.x, b.x), IMPL(a.y, b.y), IMPL(a.z, b.z));                               \
  }                                                                                            \
  GLSL_FN vec4 NAME(const vec4& a, const vec4& b) {                                            \
    return vec4(IMPL(a.x, b.x), IMPL(a.y, b.y), IMPL(a.z, b.z), IMPL(a.w, b.w));               \
  }
// vector-with-scalar second argument (min, max, mod, pow is vector-only in GLSL)
#define GLSL_MAP2S(NAME, IMPL)                                                                 \
  GLSL_FN vec2 NAME(const vec2& a, gfloat b) { return vec2(IMPL(a.x, b), IMPL(a.y, b)); }      \
  GLSL_FN vec3 NAME(const vec3& a, gfloat b) { return vec3(IMPL(a.x, b), IMPL(a.y, b), IMPL(a.z, b)); } \
  GLSL_FN vec4 NAME(const vec4& a, gfloat b) {                                                 \
    return vec4(IMPL(a.x, b), IMPL(a.y, b), IMPL(a.z, b), IMPL(a.w, b));                       \
  }

GLSL_FN gfloat g_radians(gfloat d) { return d * gfloat(0.017453292519943295f); }
GLSL_FN gfloat g_degrees(gfloat r) { return r * gfloat(57.29577951308232f); }
GLSL_FN gfloat g_inversesqrt(gfloat x) { return gfloat(1) / s_sqrt(x); }
GLSL_FN gfloat g_sign(gfloat x) { return x > gfloat(0) ? gfloat(1) : (x < gfloat(0) ? gfloat(-1) : gfloat(0)); }
GLSL_FN gfloat g_fract(gfloat x) { return x - s_floor(x); }
GLSL_FN gfloat g_mod(gfloat x, gfloat y) { return x - y * s_floor(x / y); }
GLSL_FN gfloat g_step(gfloat e, gfloat x) { return x < e ? gfloat(0) : gfloat(1); }

GLSL_MAP1(radians, g_radians)
GLSL_MAP1(degrees, g_degrees)
GLSL_MAP1(sin, s_sin)
GLSL_MAP1(cos, s_cos)
GLSL_MAP1(tan, s_tan)
GLSL_MAP1(asin, s_asin)
GLSL_MAP1(acos, s_acos)
GLSL_MAP1(atan, s_atan)
GLSL_MAP2(atan, s_atan2)
GLSL_MAP1(sinh, s_sinh)
GLSL_MAP1(cosh, s_cosh)
GLSL_MAP1(tanh, s_tanh)
GLSL_MAP2(pow, s_pow)
GLSL_MAP1(exp, s_exp)
GLSL_MAP1(log, s_log)
GLSL_MAP1(exp2, s_exp2)
GLSL_MAP1(log2, s_log2)
GLSL_MAP1(sqrt, s_sqrt)
GLSL_MAP1(inversesqrt, g_inversesqrt)
GLSL_MAP1(abs, s_abs)
GLSL_MAP1(sign, g_sign)
GLSL_MAP1(floor, s_floor)
GLSL_MAP1(ceil, s_ceil)
GLSL_MAP1(trunc, s_trunc)
GLSL_MAP1(round, s_round)
GLSL_MAP1(roundEven, s_round)
GLSL_MAP1(fract, g_fract)
GLSL_MAP2(mod, g_mod)
GLSL_MAP2S(mod, g_mod)
GLSL_MAP2(min, s_min)
GLSL_MAP2S(min, s_min)
GLSL_MAP2(max, s_max)
GLSL_MAP2S(max, s_max)
GLSL_MAP2(step, g_step)

GLSL_FN int abs(int x) { return x < 0 ? -x : x; }
GLSL_FN int min(int a, int b) { return b < a ? b : a; }
GLSL_FN int max(int a, int b) { return a < b ? b : a; }
GLSL_FN int clamp(int x, int a, int b) { return min(max(x, a), b); }
GLSL_FN int sign(int x) { return x > 0 ? 1 : (x < 0 ? -1 : 0); }

GLSL_FN gfloat clamp(gfloat x, gfloat a, gfloat b) { return min(max(x, a), b); }
GLSL_FN vec2 clamp(const vec2& x, gfloat a, gfloat b) { return min(max(x, a), b); }
GLSL_FN vec3 clamp(const vec3& x, gfloat a, gfloat b) { return min(max(x, a), b); }
GLSL_FN vec4 clamp(const vec4& x, gfloat a, gfloat b) { return min(max(x, a), b); }
GLSL_FN vec2 clamp(const vec2& x, const vec2& a, const vec2& b) { return min(max(x, a), b); }
GLSL_FN vec3 clamp(const vec3& x, const vec3& a, const vec3& b) { return min(max(x, a), b); }
GLSL_FN vec4 clamp(const vec4& x, const vec4& a, const vec4& b) { return min(max(x, a), b); }

GLSL_FN gfloat mix(gfloat x, gfloat y, gfloat a) { return x * (gfloat(1) - a) + y * a; }
GLSL_FN vec2 mix(const vec2& x, const vec2& y, gfloat a) { return x * (gfloat(1) - a) + y * a; }
GLSL_FN vec3 mix(const vec3& x, const vec3& y, gfloat a) { return x * (gfloat(1) - a) + y * a; }
GLSL_FN vec4 mix(const vec4& x, const vec4& y, gfloat a) { return x * (gfloat(1) - a) + y * a; }
GLSL_FN vec2 mix(const vec2& x, const vec2& y, const vec2& a) { return x * (vec2(gfloat(1)) - a) + y * a; }
GLSL_FN vec3 mix(const vec3& x, const vec3& y, const vec3& a) { return x * (vec3(gfloat(1)) - a) + y * a; }
GLSL_FN vec4 mix(const vec4& x, const vec4& y, const vec4& a) { return x * (vec4(gfloat(1)) - a) + y * a; }
GLSL_FN gfloat mix(gfloat x, gfloat y, bool a) { return a ? y : x; }

GLSL_FN vec2 step(gfloat e, const vec2& x) { return step(vec2(e), x); }
GLSL_FN vec3 step(gfloat e, const vec3& x) { return step(vec3(e), x); }
GLSL_FN vec4 step(gfloat e, const vec4& x) { return step(vec4(e), x); }

GLSL_FN gfloat smoothstep(gfloat e0, gfloat e1, gfloat x) {
  gfloat t = clamp((x - e0) / (e1 - e0), gfloat(0), gfloat(1));
  return t * t * (gfloat(3) - gfloat(2) * t);
}
GLSL_FN vec2 smoothstep(gfloat e0, gfloat e1, const vec2& x) {
  return vec2(smoothstep(e0, e1, x.x), smoothstep(e0, e1, x.y));
}
GLSL_FN vec3 smoothstep(gfloat e0, gfloat e1, const vec3& x) {
  return vec3(smoothstep(e0, e1, x.x), smoothstep(e0, e1, x.y), smoothstep(e0, e1, x.z));
}
GLSL_FN vec3 smoothstep(const vec3& e0, const vec3& e1, const vec3& x) {
  return vec3(smoothstep(e0.x, e1.x, x.x), smoothstep(e0.y, e1.y, x.y), smoothstep(e0.z, e1.z, x.z));
}

GLSL_FN gfloat length(gfloat x) { return s_abs(x); }
GLSL_FN gfloat length(const vec2& v) { return s_sqrt(dot(v, v)); }
GLSL_FN gfloat length(const vec3& v) { return s_sqrt(dot(v, v)); }
GLSL_FN gfloat length(const vec4& v) { return s_sqrt(dot(v, v)); }
GLSL_FN gfloat distance(gfloat a, gfloat b) { return length(a - b); }
GLSL_FN gfloat distance(const vec2& a, const vec2& b) { return length(a - b); }
GLSL_FN gfloat distance(const vec3& a, const vec3& b) { return length(a - b); }
GLSL_FN gfloat distance(const vec4& a, const vec4& b) { return length(a - b); }
GLSL_FN gfloat normalize(gfloat x) { return g_sign(x); }
GLSL_FN vec2 normalize(const vec2& v) { return v * g_inversesqrt(dot(v, v)); }
GLSL_FN vec3 normalize(const vec3& v) { return v * g_inversesqrt(dot(v, v)); }
GLSL_FN vec4 normalize(const vec4& v) { return v * g_inversesqrt(dot(v, v)); }
GLSL_FN vec3 cross(const vec3& a, const vec3& b) {
  return vec3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
GLSL_FN vec3 reflect(const vec3& i, const vec3& n) { return i - gfloat(2) * dot(n, i) * n; }
GLSL_FN vec2 reflect(const vec2& i, const vec2& n) { return i - gfloat(2) * dot(n, i) * n; }
GLSL_FN vec3 refract(const vec3& i, const vec3& n, gfloat eta) {
  gfloat ni = dot(n, i);
  gfloat k = gfloat(1) - eta * eta * (gfloat(1) - ni * ni);
  if (k < gfloat(0)) return vec3(gfloat(0));
  return eta * i - (eta * ni + s_sqrt(k)) * n;
}
GLSL_FN vec3 faceforward(const vec3& n, const vec3& i, const vec3& nref) {
  return dot(nref, i) < gfloat(0) ? n : -n;
}
GLSL_FN bool isnan(gfloat x) { return s_isnan(x); }
GLSL_FN bool isinf(gfloat x) { return s_isinf(x); }

// ---- textures -----------------------------------------------------------------------------
// A sampler is a plain view of row-major texel data (row 0 = t=0, i.e. the bottom row in GL).
// fmt: 0 = float32 texels, 1 = IEEE binary16 texels, 2 = unorm8 texels (sRGB-decoded when
// srgb != 0). filter: 0 = NEAREST, 1 = LINEAR. Wrap mode is CLAMP_TO_EDGE.
struct sampler2D {
  const void* data;
  int w, h, ch, fmt, filter, srgb;
};
struct sampler3D {
  const void* data;
  int w, h, d, ch, fmt, filter;
};

GLSL_FN float half_bits_to_float(unsigned short h) {
  // IEEE 754 binary16 -> binary32 (sign, 5-bit exponent with bias 15, 10-bit mantissa)
  unsigned int sign = (unsigned int)(h & 0x8000u) << 16;
  unsigned int e = (h >> 10) & 0x1fu;
  unsigned int m = h & 0x3ffu;
  unsigned int bits;
  if (e == 0) {
    if (m == 0) {
      bits = sign;
    } else {  // subnormal half: renormalise
      int shift = 0;
      while (!(m & 0x400u)) { m <<= 1; ++shift; }
      m &= 0x3ffu;
      bits = sign | ((unsigned int)(127 - 15 + 1 - shift) << 23) | (m << 13);
    }
  } else if (e == 31) {
    bits = sign | 0x7f800000u | (m << 13);
  } else {
    bits = sign | ((e - 15 + 127) << 23) | (m << 13);
  }
  union { unsigned int u; float f; } cvt;
  cvt.u = bits;
  return cvt.f;
}

GLSL_FN float srgb8_to_linear(unsigned int v) {
  float c = float(v) * (1.0f / 255.0f);
  return c <= 0.04045f ? c * (1.0f / 12.92f) : s_tofloat(s_pow(gfloat((c + 0.055f) * (1.0f / 1.055f)), gfloat(2.4f)));
}

GLSL_FN float texel_component(const void* data, int fmt, int srgb, long long idx) {
  if (fmt == 0) return ((const float*)data)[idx];
  if (fmt == 1) return half_bits_to_float(((const unsigned short*)data)[idx]);
  unsigned int v = ((const unsigned char*)data)[idx];
  return srgb ? srgb8_to_linear(v) : float(v) * (1.0f / 255.0f);
}

GLSL_FN vec4 texel2D(const sampler2D& s, int i, int j) {
  i = i < 0 ? 0 : (i >= s.w ? s.w - 1 : i);
  j = j < 0 ? 0 : (j >= s.h ? s.h - 1 : j);
  long long base = ((long long)j * s.w + i) * s.ch;
  float c[4] = {0.0f, 0.0f, 0.0f, 1.0f};
  for (int k = 0; k < s.ch && k < 4; ++k) c[k] = texel_component(s.data, s.fmt, s.srgb && k < 3, base + k);
  return vec4(c[0], c[1], c[2], c[3]);
}

GLSL_FN vec4 texture(const sampler2D& s, const vec2& uv) {
  if (!s.filter) {
    int i = int(s_tofloat(s_floor(uv.x * gfloat(float(s.w)))));
    int j = int(s_tofloat(s_floor(uv.y * gfloat(float(s.h)))));
    return texel2D(s, i, j);
  }
  gfloat x = uv.x * gfloat(float(s.w)) - gfloat(0.5f);
  gfloat y = uv.y * gfloat(float(s.h)) - gfloat(0.5f);
  gfloat x0 = s_floor(x), y0 = s_floor(y);
  gfloat fx = x - x0, fy = y - y0;
  int i0 = int(s_tofloat(x0)), j0 = int(s_tofloat(y0));
  vec4 a = texel2D(s, i0, j0), b = texel2D(s, i0 + 1, j0);
  vec4 c = texel2D(s, i0, j0 + 1), e = texel2D(s, i0 + 1, j0 + 1);
  return mix(mix(a, b, fx), mix(c, e, fx), fy);
}

GLSL_FN vec4 texelFetch(const sampler2D& s, const ivec2& p, int) { return texel2D(s, p.x, p.y); }

GLSL_FN vec4 texel3D(const sampler3D& s, int i, int j, int k) {
  i = i < 0 ? 0 : (i >= s.w ? s.w - 1 : i);
  j = j < 0 ? 0 : (j >= s.h ? s.h - 1 : j);
  k = k < 0 ? 0 : (k >= s.d ? s.d - 1 : k);
  long long base = (((long long)k * s.h + j) * s.w + i) * s.ch;
  float c[4] = {0.0f, 0.0f, 0.0f, 1.0f};
  for (int q = 0; q < s.ch && q < 4; ++q) c[q] = texel_component(s.data, s.fmt, 0, base + q);
  return vec4(c[0], c[1], c[2], c[3]);
}

GLSL_FN vec4 texture(const sampler3D& s, const vec3& uvw) {
  if (!s.filter) {
    int i = int(s_tofloat(s_floor(uvw.x * gfloat(float(s.w)))));
    int j = int(s_tofloat(s_floor(uvw.y * gfloat(float(s.h)))));
    int k = int(s_tofloat(s_floor(uvw.z * gfloat(float(s.d)))));
    return texel3D(s, i, j, k);
  }
  gfloat x = uvw.x * gfloat(float(s.w)) - gfloat(0.5f);
  gfloat y = uvw.y * gfloat(float(s.h)) - gfloat(0.5f);
  gfloat z = uvw.z * gfloat(float(s.d)) - gfloat(0.5f);
  gfloat x0 = s_floor(x), y0 = s_floor(y), z0 = s_floor(z);
  gfloat fx = x - x0, fy = y - y0, fz = z - z0;
  int i0 = int(s_tofloat(x0)), j0 = int(s_tofloat(y0)), k0 = int(s_tofloat(z0));
  vec4 c000 = texel3D(s, i0, j0, k0), c100 = texel3D(s, i0 + 1, j0, k0);
  vec4 c010 = texel3D(s, i0, j0 + 1, k0), c110 = texel3D(s, i0 + 1, j0 + 1, k0);
  vec4 c001 = texel3D(s, i0, j0, k0 + 1), c101 = texel3D(s, i0 + 1, j0, k0 + 1);
  vec4 c011 = texel3D(s, i0, j0 + 1, k0 + 1), c111 = texel3D(s, i0 + 1, j0 + 1, k0 + 1);
  vec4 lo = mix(mix(c000, c100, fx), mix(c010, c110, fx), fy);
  vec4 hi = mix(mix(c001, c101, fx), mix(c011, c111, fx), fy);
  return mix(lo, hi, fz);
}

}  // namespace glsl
