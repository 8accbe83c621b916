// packed2.cuh - pairs of float32 cell updates on sm_100's packed FP32 path.
//
// __fadd2_rn / __fmul2_rn / __ffma2_rn (float2, one instruction for two
// lanes) round each component exactly as __fadd_rn / __fmul_rn / __fmaf_rn
// do, so a pair of cells updated here gets the bits the scalar path gives
// each cell. Subtraction is fma(b, -1, a): one rounding of a - b, the same
// value and zero sign as __fsub_rn(a, b).
#pragma once

#include "common.cuh"

namespace pfb {

__device__ __forceinline__ float2 bc2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
  return __ffma2_rn(b, bc2(-1.f), a);
}

// qdiv_fast on two numerators with one divisor d (r = RN(1/d)): the same
// scaling, Markstein correction and sign restoration, component-wise.
__device__ __forceinline__ float2 qdiv_fast2(float2 a, float d, float r) {
  const float2 as = mul2(a, bc2(0x1p64f));
  const float2 q0 = mul2(as, bc2(r));
  const float2 rem = __ffma2_rn(q0, bc2(-d), as);
  const float2 q = mul2(__ffma2_rn(rem, bc2(r), q0), bc2(0x1p-64f));
  return make_float2(copysignf(q.x, a.x), copysignf(q.y, a.y));
}

// qdiv_fast2 with a divisor per lane (d.x for a.x, d.y for a.y).
__device__ __forceinline__ float2 qdiv_fast2v(float2 a, float2 d, float2 r) {
  const float2 as = mul2(a, bc2(0x1p64f));
  const float2 q0 = mul2(as, r);
  const float2 rem = __ffma2_rn(q0, make_float2(-d.x, -d.y), as);
  const float2 q = mul2(__ffma2_rn(rem, r, q0), bc2(0x1p-64f));
  return make_float2(copysignf(q.x, a.x), copysignf(q.y, a.y));
}

// bulk() on two cells: f + (dA - dB) * k.
__device__ __forceinline__ float2 bulk2(float2 f, float2 k, float2 dA, float2 dB) {
  return add2(f, mul2(sub2(dA, dB), k));
}

__device__ __forceinline__ float absmax2(float2 a, float2 b) {
  return fmaxf(fmaxf(fabsf(a.x), fabsf(a.y)), fmaxf(fabsf(b.x), fabsf(b.y)));
}

}  // namespace pfb
