// Packed pairs of binary32 values for sm_100a's paired FP32 pipe: add, mul
// and fma on .f32x2 operands (PTX ISA 8.6, sm_100a) issue one instruction for
// two independent lanes of arithmetic, each lane rounded exactly as the scalar
// .rn operation.  A pair lives in one 64-bit register (two adjacent 32-bit
// halves: .x low, .y high), so a pair built once and used many times costs no
// moves.  There is no paired max; max is taken per half.
#pragma once

#include <stdint.h>

namespace pf {

struct f2 {
  uint64_t v;
};

__device__ __forceinline__ f2 f2_make(float x, float y) {
  f2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(x), "f"(y));
  return r;
}
__device__ __forceinline__ f2 f2_bcast(float x) { return f2_make(x, x); }
__device__ __forceinline__ float f2_x(f2 a) { return __uint_as_float((unsigned)a.v); }
__device__ __forceinline__ float f2_y(f2 a) { return __uint_as_float((unsigned)(a.v >> 32)); }
__device__ __forceinline__ void f2_split(f2 a, float& x, float& y) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(x), "=f"(y) : "l"(a.v));
}
// a + b, a * b, a * b + c, each half rounded to nearest even
__device__ __forceinline__ f2 f2_add(f2 a, f2 b) {
  f2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ f2 f2_mul(f2 a, f2 b) {
  f2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ f2 f2_fma(f2 a, f2 b, f2 c) {
  f2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
  return r;
}
// max(a, 0) per half
__device__ __forceinline__ f2 f2_relu(f2 a) {
  float x, y;
  f2_split(a, x, y);
  return f2_make(fmaxf(x, 0.f), fmaxf(y, 0.f));
}

}  // namespace pf
