// counted.h - an operation-counting float for the oracle (algorithmic FLOP count per path sample).
//
// TEST INFRASTRUCTURE. Included before glslcompat.h in the oracle's counting build
// (-DORACLE_COUNT_OPS): every float operation the restated algorithm performs (scene SDFs and
// hooks included) is tallied per thread. Convention: add, sub, mul, min, max, compare, floor
// count 1 FP32 op each (so a fused multiply-add counts 2); division, sqrt, exp, log, pow, sin,
// cos, tan, asin, acos, atan are tallied separately as special-function operations; abs and
// negation are free (operand modifiers on the GPU).
#pragma once
#define GLSL_SCALAR_DEFINED 1
#include <cmath>
#include <cstdint>

namespace glsl {

struct OpCounts {
  uint64_t flops;
  uint64_t special;
};
inline OpCounts& op_counts() {
  static thread_local OpCounts c{0, 0};
  return c;
}
inline void count_f(uint64_t n = 1) { op_counts().flops += n; }
inline void count_s(uint64_t n = 1) { op_counts().special += n; }

struct Counted {
  float v;
  Counted() = default;
  Counted(float x) : v(x) {}
  Counted(double x) : v((float)x) {}
  Counted(int x) : v((float)x) {}
  explicit operator int() const { return (int)v; }
  explicit operator unsigned() const { return (unsigned)v; }
  explicit operator float() const { return v; }
  Counted& operator+=(Counted o) { count_f(); v += o.v; return *this; }
  Counted& operator-=(Counted o) { count_f(); v -= o.v; return *this; }
  Counted& operator*=(Counted o) { count_f(); v *= o.v; return *this; }
  Counted& operator/=(Counted o) { count_s(); v /= o.v; return *this; }
};
inline Counted operator+(Counted a, Counted b) { count_f(); return Counted(a.v + b.v); }
inline Counted operator-(Counted a, Counted b) { count_f(); return Counted(a.v - b.v); }
inline Counted operator*(Counted a, Counted b) { count_f(); return Counted(a.v * b.v); }
inline Counted operator/(Counted a, Counted b) { count_s(); return Counted(a.v / b.v); }
inline Counted operator-(Counted a) { return Counted(-a.v); }
inline Counted operator+(Counted a) { return a; }
inline bool operator<(Counted a, Counted b) { count_f(); return a.v < b.v; }
inline bool operator>(Counted a, Counted b) { count_f(); return a.v > b.v; }
inline bool operator<=(Counted a, Counted b) { count_f(); return a.v <= b.v; }
inline bool operator>=(Counted a, Counted b) { count_f(); return a.v >= b.v; }
inline bool operator==(Counted a, Counted b) { count_f(); return a.v == b.v; }
inline bool operator!=(Counted a, Counted b) { count_f(); return a.v != b.v; }

typedef Counted gfloat;

inline float s_tofloat(Counted x) { return x.v; }
inline Counted s_sqrt(Counted x) { count_s(); return std::sqrt(x.v); }
inline Counted s_sin(Counted x) { count_s(); return std::sin(x.v); }
inline Counted s_cos(Counted x) { count_s(); return std::cos(x.v); }
inline Counted s_tan(Counted x) { count_s(); return std::tan(x.v); }
inline Counted s_asin(Counted x) { count_s(); return std::asin(x.v); }
inline Counted s_acos(Counted x) { count_s(); return std::acos(x.v); }
inline Counted s_atan(Counted x) { count_s(); return std::atan(x.v); }
inline Counted s_atan2(Counted y, Counted x) { count_s(); return std::atan2(y.v, x.v); }
inline Counted s_sinh(Counted x) { count_s(); return std::sinh(x.v); }
inline Counted s_cosh(Counted x) { count_s(); return std::cosh(x.v); }
inline Counted s_tanh(Counted x) { count_s(); return std::tanh(x.v); }
inline Counted s_exp(Counted x) { count_s(); return std::exp(x.v); }
inline Counted s_exp2(Counted x) { count_s(); return std::exp2(x.v); }
inline Counted s_log(Counted x) { count_s(); return std::log(x.v); }
inline Counted s_log2(Counted x) { count_s(); return std::log2(x.v); }
inline Counted s_pow(Counted x, Counted y) { count_s(); return std::pow(x.v, y.v); }
inline Counted s_floor(Counted x) { count_f(); return std::floor(x.v); }
inline Counted s_ceil(Counted x) { count_f(); return std::ceil(x.v); }
inline Counted s_trunc(Counted x) { count_f(); return std::trunc(x.v); }
inline Counted s_round(Counted x) { count_f(); return std::round(x.v); }
inline Counted s_abs(Counted x) { return std::fabs(x.v); }
inline Counted s_min(Counted a, Counted b) { count_f(); return std::fmin(a.v, b.v); }
inline Counted s_max(Counted a, Counted b) { count_f(); return std::fmax(a.v, b.v); }
inline bool s_isnan(Counted x) { return std::isnan(x.v); }
inline bool s_isinf(Counted x) { return std::isinf(x.v); }

}  // namespace glsl
