// pt_math.cuh -- scalar/vector arithmetic of the tracer with a fixed evaluation
// order.  The library is compiled with -fmad=false, so no multiply-add is fused
// unless written as __fmaf_rn; division and sqrt are IEEE round-to-nearest.
// Every expression is evaluated left to right as in the WGSL it restates
// (src/utilities.wgsl, src/path_tracer/path_tracer.wgsl), which makes results
// reproducible bit for bit on any IEEE binary32 machine.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pt {

// ------------------------------------------------------------------ scalars
// min/max as a lattice: NaN-ignoring, -0 ordered below +0, so the result does
// not depend on the order of a reduction.
__device__ __forceinline__ float lmin(float a, float b) {
  if (a != a) return b;
  if (b != b) return a;
  if (a < b) return a;
  if (b < a) return b;
  return signbit(a) ? a : b;
}
__device__ __forceinline__ float lmax(float a, float b) {
  if (a != a) return b;
  if (b != b) return a;
  if (a > b) return a;
  if (b > a) return b;
  return signbit(a) ? b : a;
}

// sin/cos of x (|x| <= 1e5): Cody-Waite reduction by pi/2 split into three
// floats, Taylor polynomials of sin (degree 9) and cos (degree 10) on
// [-pi/4, pi/4] evaluated with fused multiply-adds.  WGSL leaves sin/cos
// precision implementation-defined; this fixed form keeps host and device
// results identical.
__device__ __forceinline__ void sincos_fixed(float x, float* s_out, float* c_out) {
  if (!(fabsf(x) <= 1.0e5f)) { *s_out = __int_as_float(0x7fc00000); *c_out = *s_out; return; }
  const float q = rintf(x * 0.636619746685028076171875f);
  float r = __fmaf_rn(-q, 1.57079637050628662109375f, x);
  r = __fmaf_rn(-q, -4.37113900018624283e-08f, r);
  r = __fmaf_rn(-q, -1.7151245100059349e-15f, r);
  const float r2 = r * r;
  float ps = __fmaf_rn(r2, 2.75573192239858906525573592e-6f, -1.98412698412698412698e-4f);
  ps = __fmaf_rn(r2, ps, 8.33333333333333333333e-3f);
  ps = __fmaf_rn(r2, ps, -1.66666666666666666667e-1f);
  const float s = __fmaf_rn(r * r2, ps, r);
  float pc = __fmaf_rn(r2, -2.75573192239858906525573592e-7f, 2.48015873015873015873e-5f);
  pc = __fmaf_rn(r2, pc, -1.38888888888888888889e-3f);
  pc = __fmaf_rn(r2, pc, 4.16666666666666666667e-2f);
  pc = __fmaf_rn(r2, pc, -0.5f);
  const float c = __fmaf_rn(r2, pc, 1.0f);
  switch (((int)q) & 3) {
    case 0: *s_out = s; *c_out = c; break;
    case 1: *s_out = c; *c_out = -s; break;
    case 2: *s_out = -s; *c_out = -c; break;
    default: *s_out = -c; *c_out = s; break;
  }
}

// pow(x, 5.0) (src/utilities.wgsl:788) as (x*x)*(x*x)*x; with quirks off the
// base is clamped at 0.
__device__ __forceinline__ float pow5(float x, bool quirks) {
  if (!quirks) x = lmax(x, 0.0f);
  const float x2 = x * x;
  return x2 * x2 * x;
}

// PCG hash, src/utilities.wgsl:67-83.
__device__ __forceinline__ uint32_t rand_u(uint32_t& st) {
  st = st * 747796405u + 2891336453u;
  const uint32_t word = ((st >> ((st >> 28u) + 4u)) ^ st) * 277803737u;
  return (word >> 22u) ^ word;
}
__device__ __forceinline__ float rand_f(uint32_t& st) {
  return __uint2float_rn(rand_u(st)) * __int_as_float(0x2f800004);
}
// Per-sample RNG state: path_tracer.wgsl:61 plus the optional seed offset.
__device__ __forceinline__ uint32_t seed_state(uint32_t pixel, uint32_t sample, uint32_t seed) {
  return pixel * 1235243u + sample * 5817321u + seed * 0x9E3779B9u;
}

// ------------------------------------------------------------------ vectors
__device__ __forceinline__ float3 v3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 add(float3 a, float3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 sub(float3 a, float3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 neg(float3 a) { return v3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 mul(float3 a, float3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float3 muls(float3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 divs(float3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float3 divv(float3 a, float3 b) { return v3(a.x / b.x, a.y / b.y, a.z / b.z); }
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float length(float3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ float3 normalize(float3 a) { return divs(a, length(a)); }
__device__ __forceinline__ float3 vmax(float3 a, float3 b) { return v3(lmax(a.x, b.x), lmax(a.y, b.y), lmax(a.z, b.z)); }
__device__ __forceinline__ float3 vmin(float3 a, float3 b) { return v3(lmin(a.x, b.x), lmin(a.y, b.y), lmin(a.z, b.z)); }
__device__ __forceinline__ float max3(float3 v) { return lmax(lmax(v.x, v.y), v.z); }
__device__ __forceinline__ float3 xyz(float4 a) { return v3(a.x, a.y, a.z); }

// Column-major 4x4 held as four float4 columns.
struct M4 { float4 c0, c1, c2, c3; };
// m * vec4(p, w) = ((c0*x + c1*y) + c2*z) + c3*w per component.
__device__ __forceinline__ float4 mul4(const M4& m, float x, float y, float z, float w) {
  return make_float4(m.c0.x * x + m.c1.x * y + m.c2.x * z + m.c3.x * w,
                     m.c0.y * x + m.c1.y * y + m.c2.y * z + m.c3.y * w,
                     m.c0.z * x + m.c1.z * y + m.c2.z * z + m.c3.z * w,
                     m.c0.w * x + m.c1.w * y + m.c2.w * z + m.c3.w * w);
}
// src/utilities.wgsl:751-759.
__device__ __forceinline__ float3 transform_position(const M4& m, float3 p) {
  const float4 h = mul4(m, p.x, p.y, p.z, 1.0f);
  return v3(h.x / h.w, h.y / h.w, h.z / h.w);
}
__device__ __forceinline__ float3 transform_direction(const M4& m, float3 p) {
  const float4 h = mul4(m, p.x, p.y, p.z, 0.0f);
  return v3(h.x, h.y, h.z);
}

}  // namespace pt
