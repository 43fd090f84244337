// Paired single precision: two f32 values in one 64-bit register pair, operated on by the
// sm_100 instructions add/sub/fma.rn.f32x2. Each rounds both halves to nearest exactly as
// the scalar instruction does, so a paired result is bit-identical to two scalar ones, but
// it takes one issue slot for two operations (the FMA pipe is busy for two cycles; a kernel
// bound by instruction issue rather than by that pipe gains the slot).
//
// The code generator contracts a paired mul.rn followed by a paired add.rn into one fused
// multiply-add, explicit rounding modifiers notwithstanding (measured: 20% of a*b + c
// results differ from the two-rounding value). A product written as fma(a, b, +0) is not
// contracted, and it equals the rounded product a*b except that a -0 product becomes +0
// (-0 + +0 = +0 under round-to-nearest). f2_mul is that form, so every paired expression
// keeps one rounding per operation; splat_diag_pair_exact checks it on the device.
#pragma once
#include <cstdint>

namespace splat {

struct f2 {
  unsigned long long v;
};

__device__ __forceinline__ f2 f2_make(float lo, float hi) {
  f2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ f2 f2_splat(float x) { return f2_make(x, x); }
__device__ __forceinline__ void f2_split(f2 a, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a.v));
}
__device__ __forceinline__ f2 f2_add(f2 a, f2 b) {
  f2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ f2 f2_sub(f2 a, f2 b) {
  f2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
// The rounded product, never fused into a following add (see above); -0 products give +0.
__device__ __forceinline__ f2 f2_mul(f2 a, f2 b) {
  f2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(0ull));
  return r;
}
// a * b + c with one rounding per half.
__device__ __forceinline__ f2 f2_fma(f2 a, f2 b, f2 c) {
  f2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
  return r;
}

}  // namespace splat
