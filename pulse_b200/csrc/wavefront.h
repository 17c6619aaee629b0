// wavefront.h -- wavefront renderer buffers and launcher (internal).
#pragma once
#include "kernels.h"

namespace pt {

// Device buffers of one wavefront frame (capacity = paths per frame).
struct WfBuffers {
  float4* s;        // 4 x float4 per path: state
  float4* h0;       // per path: (t, inst, slot, u)
  float* h1;        // per path: v
  uint32_t* q[2];   // ping-pong queues of live path ids
  float4* shadow;   // 4 x float4 per shadow request
  uint32_t* counts; // [q0, q1, shadow, unused, extend cursor, shadow cursor, unused, unused]
};

// Bytes of WfBuffers for `paths` paths.
inline size_t wf_bytes(size_t paths) { return paths * (64 + 16 + 4 + 4 + 4 + 64) + 256; }

cudaError_t launch_render_wavefront(const DevScene& S, const TraceCfg& tc, const PathCfg& pc, const FrameCfg& fc,
                                    const WfBuffers& B, float4* image, Counters* ctr, unsigned long long* work,
                                    uint32_t* launches, cudaStream_t st);

}  // namespace pt
