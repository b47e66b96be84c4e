// pairmath.cuh -- arithmetic helpers of the direct-N pair kernels.
//
// rsqrt_f32: the MUFU reciprocal square root (rsqrt.approx.ftz.f32).
// rsqrt_f64: FP64 has no full-precision hardware rsqrt; it is seeded with
// rsqrt.approx.ftz.f64 and refined by one third-order Householder step for
// 1/sqrt (y = y0 (1 + e/2 + 3 e^2 / 8), e = 1 - x y0^2), checked against
// 1/sqrt(x) to a few ulp by the test suite.
// f32x2: two FP32 lanes in one 64-bit register for Blackwell's packed
// add/sub/mul/fma.rn.f32x2 instructions (one instruction, two FP32 results).
#pragma once

namespace sph {

__device__ __forceinline__ float rsqrt_f32(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ double rsqrt_f64(double x) {
  double y0;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y0) : "d"(x));
  const double e = fma(-x, y0 * y0, 1.0);
  const double c = fma(0.375, e, 0.5);
  return fma(y0 * e, c, y0);
}

typedef unsigned long long f32x2;

__device__ __forceinline__ f32x2 pk2(float a, float b) {
  f32x2 r;
  asm("mov.b64 %0, {%1,%2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void upk2(f32x2 v, float &a, float &b) {
  asm("mov.b64 {%0,%1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

}  // namespace sph
