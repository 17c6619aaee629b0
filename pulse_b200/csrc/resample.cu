// resample.cu -- the upscaling hand-off: the accumulation target resampled to
// the view's resolution as RGBA16F (half4), headless.
//
// The reference draws a fullscreen triangle whose fragment shader samples the
// path-tracer target with wgpu's default sampler (nearest filtering, clamp to
// edge; src/path_tracer/pt_upscaling/pt_upscaling.wgsl:48-50,
// src/path_tracer/pt_upscaling/node.rs:70-77) into the Rgba16Float view
// target.  Here output texel (x, y) of an out_w x out_h image takes
//   u = (x + 0.5) / out_w,  v = (y + 0.5) / out_h       (the fragment centre)
//   nearest:  source texel (min(floor(u W), W-1), min(floor(v H), H-1))
//   bilinear: the four texels around (u W - 0.5, v H - 0.5), clamped to the edge,
//             mixed as (1-fx)(1-fy) a + fx(1-fy) b + (1-fx) fy c + fx fy d
// and converts each channel to half with round-to-nearest-even.
#include <cuda_fp16.h>

#include "kernels.h"

namespace pt {

namespace {

__device__ __forceinline__ uint32_t pack_half2(float a, float b) {
  const __half ha = __float2half_rn(a), hb = __float2half_rn(b);
  return (uint32_t)__half_as_ushort(ha) | ((uint32_t)__half_as_ushort(hb) << 16);
}

__global__ void k_resample(const float4* __restrict__ src, uint32_t W, uint32_t H, uint2* __restrict__ dst,
                           uint32_t out_w, uint32_t out_h, uint32_t filter) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= out_w || y >= out_h) return;
  const float u = (__uint2float_rn(x) + 0.5f) / __uint2float_rn(out_w);
  const float v = (__uint2float_rn(y) + 0.5f) / __uint2float_rn(out_h);
  float4 c;
  if (filter == 0) {
    const uint32_t sx = min((uint32_t)floorf(u * __uint2float_rn(W)), W - 1);
    const uint32_t sy = min((uint32_t)floorf(v * __uint2float_rn(H)), H - 1);
    c = src[(size_t)sy * W + sx];
  } else {
    const float px = u * __uint2float_rn(W) - 0.5f, py = v * __uint2float_rn(H) - 0.5f;
    const float fx0 = floorf(px), fy0 = floorf(py);
    const float fx = px - fx0, fy = py - fy0;
    const int ix = (int)fx0, iy = (int)fy0;
    const uint32_t x0 = (uint32_t)max(ix, 0), x1 = (uint32_t)min(max(ix + 1, 0), (int)W - 1);
    const uint32_t y0 = (uint32_t)max(iy, 0), y1 = (uint32_t)min(max(iy + 1, 0), (int)H - 1);
    const uint32_t xa = min(x0, W - 1), ya = min(y0, H - 1);
    const float4 a = src[(size_t)ya * W + xa], b = src[(size_t)ya * W + x1];
    const float4 cc = src[(size_t)y1 * W + xa], d = src[(size_t)y1 * W + x1];
    const float w00 = (1.0f - fx) * (1.0f - fy), w10 = fx * (1.0f - fy), w01 = (1.0f - fx) * fy, w11 = fx * fy;
    c.x = ((a.x * w00 + b.x * w10) + cc.x * w01) + d.x * w11;
    c.y = ((a.y * w00 + b.y * w10) + cc.y * w01) + d.y * w11;
    c.z = ((a.z * w00 + b.z * w10) + cc.z * w01) + d.z * w11;
    c.w = ((a.w * w00 + b.w * w10) + cc.w * w01) + d.w * w11;
  }
  dst[(size_t)y * out_w + x] = make_uint2(pack_half2(c.x, c.y), pack_half2(c.z, c.w));
}

}  // namespace

cudaError_t launch_resample(const float4* src, uint32_t W, uint32_t H, void* dst, uint32_t out_w, uint32_t out_h,
                            uint32_t filter, cudaStream_t st) {
  if (out_w == 0 || out_h == 0) return cudaSuccess;
  const dim3 grid((out_w + 255) / 256, out_h);
  k_resample<<<grid, 256, 0, st>>>(src, W, H, (uint2*)dst, out_w, out_h, filter);
  return cudaGetLastError();
}

}  // namespace pt
