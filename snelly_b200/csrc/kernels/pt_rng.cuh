// pt_rng.cuh - the reference's random number generator (PT:119-130) on integer states, written
// without conversion or reciprocal instructions: the path tracer's kernels keep the GPU's
// transcendental unit (XU) near saturation, and every path draws dozens of random numbers.
//
// The reference evaluates a four-lane combined multiplicative LCG in float arithmetic with
// Schrage's decomposition. For integer states below 2^22 every float operation there is exact, so
// the same sequence comes out of 32-bit integer Schrage steps: x' = a*(x mod q) - r*(x div q),
// plus m if negative. The output u = fract(x0/m0 - x1/m1 + x2/m2 - x3/m3) takes IEEE
// round-to-nearest quotients, so the result is bit-identical to the reference's.
//
// Scene-independent: included by pt_device.cuh (NVRTC scene modules) and by aot_kernels.cu (the
// exhaustive self-test of these routines against CUDA's own division).
#pragma once
#include "glslcompat.h"

namespace sdev {

struct Rng {
  unsigned s[4];
};

// One Schrage step of a lane.
__device__ __forceinline__ unsigned schrage(unsigned x, int a, unsigned q, int r, int m) {
  unsigned hi = x / q;
  unsigned lo = x - hi * q;
  int p = a * int(lo) - r * int(hi);
  return unsigned(p < 0 ? p + m : p);
}

// float(x) for 0 <= x < 2^23 without a conversion instruction: placing x in the mantissa of
// 2^23 gives the float 2^23 + x exactly; subtracting 2^23 is exact.
__device__ __forceinline__ float small_uint_to_float(unsigned x) {
  return __fsub_rn(__uint_as_float(0x4B000000u | x), 8388608.0f);
}

// The correctly rounded quotient x / m for integers 0 <= x < m < 2^22, from the correctly rounded
// reciprocal inv_m = RN(1/m) by Markstein's correction step (P. Markstein, "IA-64 and Elementary
// Functions", 2000, ch. 8): q0 = RN(x * inv_m), the residual x - q0*m computed exactly by one
// fused multiply-add, then q = RN(q0 + residual * inv_m). Checked against __fdiv_rn for every x
// of each modulus used below (snelly_selftest).
__device__ __forceinline__ float quotient_small(float x, float m, float inv_m) {
  float q0 = __fmul_rn(x, inv_m);
  float r = __fmaf_rn(-q0, m, x);
  return __fmaf_rn(r, inv_m, q0);
}

// RN(1/m) of the four moduli (exact float32 values).
#define SNELLY_RNG_INV_M0 0x1.000044p-22f  // 1 / 4194287
#define SNELLY_RNG_INV_M1 0x1.00006cp-22f  // 1 / 4194277
#define SNELLY_RNG_INV_M2 0x1.0001c4p-22f  // 1 / 4194191
#define SNELLY_RNG_INV_M3 0x1.000224p-22f  // 1 / 4194167

__device__ __forceinline__ float rand01(Rng& g) {
  g.s[0] = schrage(g.s[0], 3423, 1225u, 1112, 4194287);
  g.s[1] = schrage(g.s[1], 2646, 1585u, 367, 4194277);
  g.s[2] = schrage(g.s[2], 1707, 2457u, 92, 4194191);
  g.s[3] = schrage(g.s[3], 1999, 2098u, 265, 4194167);
  float u0 = quotient_small(small_uint_to_float(g.s[0]), 4194287.0f, SNELLY_RNG_INV_M0);
  float u1 = quotient_small(small_uint_to_float(g.s[1]), 4194277.0f, SNELLY_RNG_INV_M1);
  float u2 = quotient_small(small_uint_to_float(g.s[2]), 4194191.0f, SNELLY_RNG_INV_M2);
  float u3 = quotient_small(small_uint_to_float(g.s[3]), 4194167.0f, SNELLY_RNG_INV_M3);
  float v = __fsub_rn(__fadd_rn(__fsub_rn(u0, u1), u2), u3);
  return __fsub_rn(v, floorf(v));
}

}  // namespace sdev
