// adjoint.h -- path-replay adjoint launcher (internal).
#pragma once
#include "wavefront.h"

namespace pt {

// Floats per material in the gradient array: base rgb, emissive rgb, roughness, unused.
constexpr uint32_t kGradStride = 8;

// Per-path adjoint record of launch_backward: kAdjRecBytes bytes per path.
constexpr size_t kAdjRecBytes = 96;

// Adds the gradients of every material (n_mat x kGradStride floats at grads,
// zeroed by the caller) for dloss/dimage dimg (float4 per texel) of the mean of
// pc.spp samples per texel (sample indices fc.acc * spp + s).  Renders the
// primal frame into primal_image with the wavefront buffers B (capacity
// W * H * spp paths), then replays every path as a wavefront with per-path
// records rec (kAdjRecBytes per path).  pc.nee_mode must be 2.
cudaError_t launch_backward(const DevScene& S, const TraceCfg& tc, const PathCfg& pc, const FrameCfg& fc,
                            const WfBuffers& B, float4* rec, float4* primal_image, uint32_t wf_segments,
                            uint32_t trace_blocks, const float4* dimg, float* grads, uint32_t n_mat, Counters* ctr,
                            uint32_t* launches, cudaStream_t st);

}  // namespace pt
