// Packed FP32 pair arithmetic for sm_100a kernels.
#pragma once
#include <cuda_runtime.h>

namespace mc {

// Packed FP32 pairs (PTX add/sub/mul/fma .f32x2, sm_100): one instruction for
// both halves of a float2, each half rounded exactly as the scalar operation.
typedef unsigned long long f2reg;
__device__ __forceinline__ f2reg f2pk(float2 a) {
  f2reg r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
__device__ __forceinline__ float2 f2up(f2reg r) {
  float2 a;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
  return a;
}
__device__ __forceinline__ f2reg f2add(f2reg a, f2reg b) {
  f2reg d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2reg f2sub(f2reg a, f2reg b) {
  f2reg d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2reg f2fma(f2reg a, f2reg b, f2reg c) {  // a*b + c per half
  f2reg d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ f2reg f2splat(float c) { return f2pk(make_float2(c, c)); }
// Complex add / subtract of the butterflies.  MC_PACKED_ADD=1 makes each one
// packed instruction; measured slower inside the codelets (the register
// pairs raise the register count), so they stay scalar by default.
#ifndef MC_PACKED_ADD
#define MC_PACKED_ADD 0
#endif
__device__ __forceinline__ float2 padd(float2 a, float2 b) {
#if MC_PACKED_ADD
  return f2up(f2add(f2pk(a), f2pk(b)));
#else
  return make_float2(a.x + b.x, a.y + b.y);
#endif
}
__device__ __forceinline__ float2 psub(float2 a, float2 b) {
#if MC_PACKED_ADD
  return f2up(f2sub(f2pk(a), f2pk(b)));
#else
  return make_float2(a.x - b.x, a.y - b.y);
#endif
}

}  // namespace mc
