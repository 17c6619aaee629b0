// kernels.h -- host-callable launchers of the device kernels (internal).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "pt_path.cuh"

namespace pt {

struct FrameCfg {
  M4 ivp;
  float3 eye;
  uint32_t W, H, acc;
};

// One mesh's BVH-ordered triangle gather (see pt_trace.cuh, tri_bvh).
cudaError_t launch_gather_tri_bvh(const float4* primitives, const uint32_t* triangle_indices, float4* tri_bvh,
                                  uint32_t triangle_offset, uint32_t index_offset, uint32_t count,
                                  cudaStream_t st);

// Per-pixel megakernel: every sample of a texel traced to termination by one
// thread, then accumulated.  block = 128 threads over a 16 x 8 texel tile.
// work: nullptr, or 8 u64 tallies (rays, tlas_interior, blas_entries,
// blas_interior, tri_tests, hits, nee, cdf_reads) filled by the counting variant.
// min_blocks: register budget variant (4, 6 or 8 resident blocks per SM; else 6).
cudaError_t launch_render_mega(const DevScene& S, const TraceCfg& tc, const PathCfg& pc, const FrameCfg& fc,
                               float4* image, Counters* ctr, unsigned long long* work, uint32_t min_blocks,
                               cudaStream_t st);

cudaError_t launch_trace_rays(const DevScene& S, const TraceCfg& tc, const float* rays, uint32_t n, Hit* out,
                              Counters* ctr, cudaStream_t st);

// Resample a W x H float4 image to out_w x out_h half4 (filter 0 nearest, 1
// bilinear) into device memory dst.
cudaError_t launch_resample(const float4* src, uint32_t W, uint32_t H, void* dst, uint32_t out_w, uint32_t out_h,
                            uint32_t filter, cudaStream_t st);

}  // namespace pt
