// wavefront.h -- wavefront renderer buffers and launchers (internal).
#pragma once
#include <cstring>

#include "kernels.h"

namespace pt {

// Most scenes one batched launch takes (their table lives in shared memory).
constexpr uint32_t kMaxBatch = 64;
// wf_segments value that runs every segment in the tail kernel.
constexpr uint32_t kWfTailOnly = 0xffffffffu;
// Wavefront segments when the parameter is 0 (measured: the 1080p sphere frame
// 115.6 -> 117.2 Mpaths/s and the 512^2 x 64 spp Cornell frame 120.4 -> 97.8 ms
// from 2 to 3; the realtime GI frame is fastest at 2).
constexpr uint32_t kDefaultWfSegments = 3;
constexpr uint32_t kDefaultGiWfSegments = 2;
// Traversal blocks per SM when the parameter is 0: eight 128-thread blocks of
// a 64-register budget fill the register file (1080p sphere frame: 5 blocks
// 138.7, 6 blocks 140.9, 8 blocks 143.7 Mpaths/s; the spills of the 64-register
// build cost less than the latency the extra warps hide).
constexpr uint32_t kDefaultTraceBlocks = 8;

// One scene of a wavefront launch.  Its paths are
// [path_offset, path_offset + paths) of the launch's id space, path id =
// path_offset + texel * spp + sample.  Copied word by word into shared memory
// by every kernel, so the size is a multiple of 16 bytes.
struct alignas(16) WfScene {
  DevScene S;
  PathCfg pc;
  FrameCfg fc;
  float4* image;
  uint32_t path_offset, paths;
};
static_assert(sizeof(WfScene) % 16 == 0, "WfScene is copied as uint4 words");

// Device buffers of one wavefront launch (capacity = paths of the launch).
struct WfBuffers {
  float4* s;        // 4 x float4 per path: state
  float4* h0;       // per path: (t, inst, slot, u)
  float* h1;        // per path: v
  uint32_t* q[2];   // ping-pong queues of live path ids
  float4* shadow;   // 4 x float4 per shadow request
  uint32_t* counts; // [q0, q1, shadow, unused, extend cursor, shadow cursor, tail cursor, unused]
  WfScene* table;   // kMaxBatch entries
  uint32_t* sort_bins;  // kSortBins counters of the ray sort
};

// Bins of the ray sort: direction octant (3 bits) x origin cell (8^3).
constexpr uint32_t kSortBins = 4096;

// Launch shape of one wavefront frame.
struct WfLaunch {
  uint32_t n_scenes, total_paths;
  uint32_t segments;             // bounces of the longest path (max_depth, +1 for mode 1)
  uint32_t wf_segments;          // segments run as wavefront steps before the tail kernel
  uint32_t trace_blocks_per_sm;  // 0 = kDefaultTraceBlocks
  int sms;
  cudaEvent_t image_wait = nullptr;  // awaited before the accumulation writes the images
};

// Bytes of WfBuffers for `paths` paths (each carve rounds up to 256 bytes).
constexpr size_t wf_bytes(size_t paths) {
  return paths * (64 + 16 + 4 + 4 + 4 + 64) + 9 * 256 + (size_t)kMaxBatch * sizeof(WfScene) + kSortBins * 4;
}

// Carves WfBuffers for `paths` paths out of `base` (wf_bytes(paths) bytes,
// 256-byte aligned); every part starts on a 256-byte boundary.
inline WfBuffers wf_carve(void* base, size_t paths) {
  uintptr_t b = (uintptr_t)base;
  auto take = [&b](size_t bytes) {
    const uintptr_t at = (b + 255) & ~(uintptr_t)255;
    b = at + bytes;
    return at;
  };
  WfBuffers B;
  B.s = (float4*)take(paths * 64);
  B.h0 = (float4*)take(paths * 16);
  B.shadow = (float4*)take(paths * 64);
  B.h1 = (float*)take(paths * 4);
  B.q[0] = (uint32_t*)take(paths * 4);
  B.q[1] = (uint32_t*)take(paths * 4);
  B.counts = (uint32_t*)take(8 * sizeof(uint32_t));
  B.table = (WfScene*)take((size_t)kMaxBatch * sizeof(WfScene));
  B.sort_bins = (uint32_t*)take(kSortBins * 4);
  return B;
}

// Writes n table entries from host memory to dev with small kernels (the
// entries travel as kernel parameters: no host staging, capturable).
cudaError_t wf_upload_table(const WfScene* host, uint32_t n, WfScene* dev, cudaStream_t st);

// Enqueue one frame of the scenes already in B.table (no host synchronisation,
// so a stream capture of it is a complete frame).
cudaError_t wf_record(int mode, const TraceCfg& tc, const WfBuffers& B, const WfLaunch& L, Counters* ctr,
                      unsigned long long* work, uint32_t* launches, cudaStream_t st);

// Raises the kernels' shared-memory limits for the current device (once per
// device); call before capturing a frame into a graph.
cudaError_t wf_prepare(int mode);

// One frame of n <= kMaxBatch scenes (all estimator `mode`): assigns the
// scenes' path offsets in order, uploads the table and records the frame.
// wf_segments: segments run as wavefront steps before the tail kernel (0 = 2);
// trace_blocks: resident traversal blocks per SM (0 = kDefaultTraceBlocks).
// image_wait: an event the accumulation (the frame's only write of the
// images, its last kernel) waits for, or nullptr.
cudaError_t wf_render(int mode, const TraceCfg& tc, const WfScene* scenes, uint32_t n, uint32_t wf_segments,
                      uint32_t trace_blocks, const WfBuffers& B, Counters* ctr, unsigned long long* work,
                      uint32_t* launches, cudaStream_t st, cudaEvent_t image_wait = nullptr);

// The primary-hit G-buffer of one scene's camera (scene.fc: W x H texels of 4
// float4: position + valid flag, normal, base color, emissive): camera rays,
// the persistent closest-hit kernel, the texels.  B holds W x H paths.
cudaError_t wf_gbuffer_primary(const TraceCfg& tc, const WfScene& scene, float4* gbuf, uint32_t trace_blocks,
                               const WfBuffers& B, Counters* ctr, uint32_t* launches, cudaStream_t st);

// The realtime GI frame (src/pulse/gi.wgsl:56-135) of one scene: scene.pc.spp
// samples per texel of scene.fc's W x H image, each starting at the G-buffer
// texel (4 float4 per texel: position + valid flag, normal, base color,
// emissive; gw x gh texels), with mode 1's diffuse bounces; the image is
// overwritten with the mean.  B holds W x H paths.
cudaError_t wf_render_gi(const TraceCfg& tc, const WfScene& scene, const float4* gbuf, uint32_t gw, uint32_t gh,
                         uint32_t wf_segments, uint32_t trace_blocks, const WfBuffers& B, Counters* ctr,
                         uint32_t* launches, cudaStream_t st);

// Building blocks for other wavefront passes over the paths of the last
// wf_render with B (its one-scene table): the closest hit of every path of
// queue qi into B.h0/h1, and the reset of the counters before a segment whose
// next queue is `next`.
cudaError_t wf_extend_step(const TraceCfg& tc, const WfBuffers& B, int qi, uint32_t trace_blocks, Counters* ctr,
                           cudaStream_t st);
cudaError_t wf_reset_step(const WfBuffers& B, int next, cudaStream_t st);

// The table entry of one scene.
inline WfScene wf_scene(const DevScene& S, const PathCfg& pc, const FrameCfg& fc, float4* image) {
  WfScene w;
  std::memset(&w, 0, sizeof(w));
  w.S = S;
  w.pc = pc;
  w.fc = fc;
  w.image = image;
  w.paths = fc.W * fc.H * pc.spp;
  return w;
}

}  // namespace pt
