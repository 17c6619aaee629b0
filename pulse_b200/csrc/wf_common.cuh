// wf_common.cuh -- device helpers shared by the wavefront kernels (internal).
#pragma once
#include "wavefront.h"

namespace pt {
namespace wf {

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// The persistent kernels step until this many of a warp's 32 lanes are idle,
// then refill them (every refill costs a ballot round and a queue atomic per
// warp, so refilling after every step is slower).
constexpr uint32_t kRefillAt = 8;

// Whether a persistent warp should stop stepping and refill its idle lanes.
__device__ __forceinline__ bool time_to_refill(bool busy, bool drained) {
  const uint32_t idle = __popc(__ballot_sync(0xffffffffu, !busy));
  return idle == 32u || (!drained && idle >= kRefillAt);
}

// Warp-aggregated append: every lane of the warp calls it; lanes with pred
// get consecutive slots of *counter.
__device__ __forceinline__ uint32_t warp_append(bool pred, uint32_t* counter) {
  const uint32_t mask = __ballot_sync(0xffffffffu, pred);
  if (mask == 0u) return 0xffffffffu;
  const uint32_t leader = __ffs(mask) - 1u;
  uint32_t base = 0;
  if (lane_id() == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  return pred ? base + (uint32_t)__popc(mask & ((1u << lane_id()) - 1u)) : 0xffffffffu;
}

// Persistent-kernel refill: lanes with need=true get the next queue entries
// (one atomicAdd per warp); 0xffffffff when the queue is exhausted.
__device__ __forceinline__ uint32_t warp_fetch(bool need, uint32_t* cursor, uint32_t n) {
  const uint32_t mask = __ballot_sync(0xffffffffu, need);
  if (mask == 0u) return 0xffffffffu;
  const uint32_t leader = __ffs(mask) - 1u;
  uint32_t base = 0;
  if (lane_id() == leader) base = atomicAdd(cursor, (uint32_t)__popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  const uint32_t idx = base + (uint32_t)__popc(mask & ((1u << lane_id()) - 1u));
  return need && idx < n ? idx : 0xffffffffu;
}

__device__ __forceinline__ void load_state(const WfBuffers& B, uint32_t p, PathState& ps) {
  const float4 a = B.s[4 * (size_t)p], b = B.s[4 * (size_t)p + 1], c = B.s[4 * (size_t)p + 2],
               d = B.s[4 * (size_t)p + 3];
  ps.o = xyz(a); ps.prev_pdf = a.w;
  ps.d = xyz(b); ps.rng = __float_as_uint(b.w);
  ps.thr = xyz(c);
  const uint32_t df = __float_as_uint(c.w);
  ps.depth = df & 0xffffffu;
  ps.flags = df >> 24;
  ps.color = xyz(d);
}
__device__ __forceinline__ void store_state(const WfBuffers& B, uint32_t p, const PathState& ps) {
  B.s[4 * (size_t)p] = make_float4(ps.o.x, ps.o.y, ps.o.z, ps.prev_pdf);
  B.s[4 * (size_t)p + 1] = make_float4(ps.d.x, ps.d.y, ps.d.z, __uint_as_float(ps.rng));
  B.s[4 * (size_t)p + 2] = make_float4(ps.thr.x, ps.thr.y, ps.thr.z,
                                       __uint_as_float((ps.depth & 0xffffffu) | (ps.flags << 24)));
  B.s[4 * (size_t)p + 3] = make_float4(ps.color.x, ps.color.y, ps.color.z, 0.0f);
}

}  // namespace wf
}  // namespace pt
