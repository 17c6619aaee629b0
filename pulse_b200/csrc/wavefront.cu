// wavefront.cu -- the path tracer as a wavefront of kernels over queues of live paths.
//
// Per frame: generate -> { extend -> shade -> shadow } x segments -> accumulate.
//   extend  closest hit of every queued path's current ray (the traversal
//           kernel only: small code, all lanes traversing);
//   shade   path_on_hit of every queued path: emission, the NEE sample (queued as
//           a shadow request), BSDF sample and Russian roulette; live paths are
//           appended to the next queue;
//   shadow  closest hit of every shadow request and its contribution;
//   accumulate  the running mean of every texel over its samples.
// Queues are compacted with one warp ballot per append (one atomicAdd per warp).
// Every path runs exactly the megakernel's arithmetic in the same order, so
// images are bit-identical to it; shadow contributions of segment k land
// before segment k+1 is shaded, as in the sequential loop.
//
// Path state (64 B, four float4 per path, path id = texel * spp + sample):
//   s0 = (o.xyz, prev_pdf)  s1 = (d.xyz, rng)  s2 = (thr.xyz, depth | flags << 24)
//   s3 = (color.xyz, unused)
// Hit of the current segment: h0 = (t, inst, slot, u), h1 = v.
// Shadow request (64 B): (o.xyz, limit) (d.xyz, path) (add_vis.xyz, -) (add_occ.xyz, -).
#include "wavefront.h"

namespace pt {

namespace {

constexpr int kWfBlock = 128;

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

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
  B.s[4 * (size_t)p + 2] = make_float4(ps.thr.x, ps.thr.y, ps.thr.z, __uint_as_float((ps.depth & 0xffffffu) | (ps.flags << 24)));
  B.s[4 * (size_t)p + 3] = make_float4(ps.color.x, ps.color.y, ps.color.z, 0.0f);
}

template <int MODE>
__global__ void __launch_bounds__(kWfBlock) k_wf_generate(PathCfg pc, FrameCfg fc, WfBuffers B, uint32_t total) {
  const uint32_t warp_base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = warp_base; base < total; base += stride) {
    const uint32_t p = base + lane_id();
    bool alive = false;
    if (p < total) {
      const uint32_t texel = p / pc.spp, s = p % pc.spp;
      const uint32_t x = texel % fc.W, y = texel / fc.W;
      PathState ps;
      path_begin(ps, pc, fc.ivp, fc.eye, x, y, fc.W, fc.H, fc.acc * pc.spp + s);
      store_state(B, p, ps);
      alive = (ps.flags & kAlive) != 0u;
    }
    const uint32_t slot = warp_append(alive, B.counts + 0);
    if (alive) B.q[0][slot] = p;
  }
}

// Persistent traversal: each lane runs trace_step on its current ray; lanes
// without a ray get the next queue entries at the top of an iteration (one
// atomicAdd per warp), so the warp stays on one loop body.
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

template <bool COUNT>
__global__ void __launch_bounds__(kWfBlock) k_wf_extend(DevScene S, TraceCfg tc, WfBuffers B, int qi, Counters* ctr,
                                                        unsigned long long* work) {
  extern __shared__ uint32_t smem[];
  const uint32_t n = B.counts[qi];
  const uint32_t* q = B.q[qi];
  uint32_t* cursor = B.counts + 4;
  WorkCount wc{};
  uint32_t* stk = smem + threadIdx.x;
  TraceState T;
  uint32_t p = 0;
  bool busy = false, drained = false;
  while (true) {
    if (!drained) {
      const uint32_t i = warp_fetch(!busy, cursor, n);
      // A lane that asked and got nothing means the queue is exhausted.
      drained = __any_sync(0xffffffffu, !busy && i == 0xffffffffu);
      if (i != 0xffffffffu) {
        p = q[i];
        const float4 a = B.s[4 * (size_t)p], b = B.s[4 * (size_t)p + 1];
        if (COUNT) wc.rays++;
        busy = !trace_init(T, S, xyz(a), xyz(b));
        if (!busy) {
          B.h0[p] = make_float4(T.rec.t, __uint_as_float(T.rec.inst), __uint_as_float(T.rec.slot), T.rec.u);
          B.h1[p] = T.rec.v;
        }
      }
    }
    if (!__any_sync(0xffffffffu, busy)) {
      if (drained) break;
      continue;
    }
    if (busy && trace_step<COUNT>(T, S, stk, blockDim.x, tc, ctr, &wc)) {
      busy = false;
      B.h0[p] = make_float4(T.rec.t, __uint_as_float(T.rec.inst), __uint_as_float(T.rec.slot), T.rec.u);
      B.h1[p] = T.rec.v;
      if (COUNT && T.rec.t < 1e30f) wc.hits++;
    }
  }
  if (COUNT) {
    __syncwarp();
    unsigned long long v[6] = {wc.rays, wc.tlas_interior, wc.blas_entries, wc.blas_interior, wc.tri_tests, wc.hits};
    for (int k = 0; k < 6; ++k) {
      unsigned long long x = v[k];
      for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
      if (lane_id() == 0) atomicAdd(work + k, x);
    }
  }
}

template <int MODE, bool COUNT>
__global__ void __launch_bounds__(kWfBlock) k_wf_shade(DevScene S, PathCfg pc, WfBuffers B, int qi,
                                                       unsigned long long* work) {
  const uint32_t n = B.counts[qi];
  const uint32_t* q = B.q[qi];
  uint32_t* qn = B.q[qi ^ 1];
  const uint32_t warp_base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u;
  const uint32_t stride = gridDim.x * blockDim.x;
  uint32_t nee = 0;
  for (uint32_t base = warp_base; base < n; base += stride) {
    const uint32_t i = base + lane_id();
    bool alive = false, shadow = false;
    uint32_t p = 0;
    ShadowReq rq;
    rq.active = false;
    if (i < n) {
      p = q[i];
      PathState ps;
      load_state(B, p, ps);
      const float4 h0 = B.h0[p];
      Hit h;
      h.t = h0.x; h.inst = __float_as_uint(h0.y); h.slot = __float_as_uint(h0.z); h.u = h0.w; h.v = B.h1[p];
      path_on_hit<MODE>(S, pc, ps, h, rq);
      store_state(B, p, ps);
      alive = (ps.flags & kAlive) != 0u;
      shadow = rq.active;
    }
    const uint32_t ns = warp_append(alive, B.counts + (qi ^ 1));
    if (alive) qn[ns] = p;
    const uint32_t ss = warp_append(shadow, B.counts + 2);
    if (shadow) {
      float4* e = B.shadow + 4 * (size_t)ss;
      e[0] = make_float4(rq.o.x, rq.o.y, rq.o.z, rq.limit);
      e[1] = make_float4(rq.d.x, rq.d.y, rq.d.z, __uint_as_float(p));
      e[2] = make_float4(rq.add_vis.x, rq.add_vis.y, rq.add_vis.z, 0.0f);
      e[3] = make_float4(rq.add_occ.x, rq.add_occ.y, rq.add_occ.z, 0.0f);
      ++nee;
    }
  }
  if (COUNT) {
    unsigned long long x = nee;
    for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
    if (lane_id() == 0) atomicAdd(work + 6, x);
  }
}

template <int MODE>
__device__ __forceinline__ void finish_shadow(const WfBuffers& B, uint32_t i, float hit_t) {
  const float4* e = B.shadow + 4 * (size_t)i;
  const float4 a = e[0], b = e[1], c = e[2], d = e[3];
  const uint32_t p = __float_as_uint(b.w);
  ShadowReq rq;
  rq.limit = a.w;
  rq.add_vis = xyz(c);
  rq.add_occ = xyz(d);
  const float4 col = B.s[4 * (size_t)p + 3];
  PathState ps;
  ps.color = xyz(col);
  path_on_shadow<MODE>(ps, rq, hit_t);
  B.s[4 * (size_t)p + 3] = make_float4(ps.color.x, ps.color.y, ps.color.z, col.w);
}

template <int MODE, bool COUNT>
__global__ void __launch_bounds__(kWfBlock) k_wf_shadow(DevScene S, TraceCfg tc, WfBuffers B, Counters* ctr,
                                                        unsigned long long* work) {
  extern __shared__ uint32_t smem[];
  const uint32_t n = B.counts[2];
  uint32_t* cursor = B.counts + 5;
  WorkCount wc{};
  uint32_t* stk = smem + threadIdx.x;
  TraceState T;
  uint32_t e_idx = 0;
  bool busy = false, drained = false;
  while (true) {
    if (!drained) {
      const uint32_t i = warp_fetch(!busy, cursor, n);
      drained = __any_sync(0xffffffffu, !busy && i == 0xffffffffu);
      if (i != 0xffffffffu) {
        e_idx = i;
        const float4* e = B.shadow + 4 * (size_t)i;
        const float4 a = e[0], b = e[1];
        if (COUNT) wc.rays++;
        busy = true;
        if (trace_init(T, S, xyz(a), xyz(b))) {
          busy = false;
          finish_shadow<MODE>(B, e_idx, T.rec.t);
        }
      }
    }
    if (!__any_sync(0xffffffffu, busy)) {
      if (drained) break;
      continue;
    }
    if (busy && trace_step<COUNT>(T, S, stk, blockDim.x, tc, ctr, &wc)) {
      busy = false;
      finish_shadow<MODE>(B, e_idx, T.rec.t);
    }
  }
  if (COUNT) {
    __syncwarp();
    unsigned long long v[5] = {wc.rays, wc.tlas_interior, wc.blas_entries, wc.blas_interior, wc.tri_tests};
    for (int k = 0; k < 5; ++k) {
      unsigned long long x = v[k];
      for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
      if (lane_id() == 0) atomicAdd(work + k, x);
    }
  }
}

// The tail: one persistent kernel takes every path still alive after the
// wavefront segments and runs it to the end (segment, shading, shadow ray,
// ...), each lane fetching a new path when its own ends.  The paths' long
// traversal tails then overlap instead of adding up segment by segment.
template <int MODE>
__global__ void __launch_bounds__(kWfBlock) k_wf_tail(DevScene S, TraceCfg tc, PathCfg pc, WfBuffers B, int qi,
                                                      Counters* ctr) {
  extern __shared__ uint32_t smem[];
  const uint32_t n = B.counts[qi];
  const uint32_t* q = B.q[qi];
  uint32_t* cursor = B.counts + 6;
  uint32_t* stk = smem + threadIdx.x;
  PathState ps;
  ShadowReq rq;
  rq.active = false;
  TraceState T;
  uint32_t p = 0;
  bool busy = false, shadow = false, tracing = false, drained = false;
  while (true) {
    if (!drained) {
      const uint32_t i = warp_fetch(!busy, cursor, n);
      drained = __any_sync(0xffffffffu, !busy && i == 0xffffffffu);
      if (i != 0xffffffffu) {
        p = q[i];
        load_state(B, p, ps);
        busy = true;
        shadow = false;
        tracing = false;
      }
    }
    if (!__any_sync(0xffffffffu, busy)) {
      if (drained) break;
      continue;
    }
    if (!busy) continue;
    bool done_ray = false;
    if (!tracing) {
      const float3 o = shadow ? rq.o : ps.o, d = shadow ? rq.d : ps.d;
      if (trace_init(T, S, o, d)) done_ray = true;
      else tracing = true;
    } else if (trace_step<false>(T, S, stk, blockDim.x, tc, ctr, nullptr)) {
      tracing = false;
      done_ray = true;
    }
    if (done_ray) {
      if (shadow) {
        path_on_shadow<MODE>(ps, rq, T.rec.t);
        shadow = false;
      } else {
        path_on_hit<MODE>(S, pc, ps, T.rec, rq);
        shadow = rq.active;
      }
      if (!shadow && !(ps.flags & kAlive)) {
        store_state(B, p, ps);
        busy = false;
      }
    }
  }
}

__global__ void __launch_bounds__(kWfBlock) k_wf_accumulate(PathCfg pc, FrameCfg fc, WfBuffers B, float4* image) {
  const uint32_t texels = fc.W * fc.H;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < texels; t += gridDim.x * blockDim.x) {
    float4 px = fc.acc * pc.spp > 0 ? image[t] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    for (uint32_t s = 0; s < pc.spp; ++s) {
      const float4 c = B.s[4 * ((size_t)t * pc.spp + s) + 3];
      px = accumulate(px, xyz(c), fc.acc * pc.spp + s);
    }
    image[t] = px;
  }
}

__global__ void k_wf_reset(uint32_t* counts, int next) {
  if (threadIdx.x == 0) { counts[next] = 0; counts[2] = 0; counts[4] = 0; counts[5] = 0; counts[6] = 0; }
}

template <typename K>
cudaError_t smem_attr(K kernel) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
}

template <int MODE, bool COUNT>
cudaError_t run(const DevScene& S, const TraceCfg& tc, const PathCfg& pc, const FrameCfg& fc, const WfBuffers& B,
                uint32_t total, int sms, float4* image, Counters* ctr, unsigned long long* work, uint32_t* launches,
                cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    cudaError_t e = smem_attr(k_wf_extend<COUNT>);
    if (e == cudaSuccess) e = smem_attr(k_wf_shadow<MODE, COUNT>);
    if (e == cudaSuccess) e = smem_attr(k_wf_tail<MODE>);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const size_t smem = (size_t)2 * tc.stack_depth * kWfBlock * 4;
  const int trace_blocks = sms * 4;
  const int light_blocks = sms * 16;
  cudaError_t e = cudaMemsetAsync(B.counts, 0, 8 * sizeof(uint32_t), st);
  if (e != cudaSuccess) return e;
  uint32_t L = 0;
  k_wf_generate<MODE><<<light_blocks, kWfBlock, 0, st>>>(pc, fc, B, total);
  ++L;
  const uint32_t segments = pc.max_depth + (MODE == 1 ? 1u : 0u);
  const uint32_t wf = pc.wf_segments < segments ? pc.wf_segments : segments;
  int qi = 0;
  for (uint32_t seg = 0; seg < wf; ++seg) {
    k_wf_reset<<<1, 32, 0, st>>>(B.counts, qi ^ 1);
    k_wf_extend<COUNT><<<trace_blocks, kWfBlock, smem, st>>>(S, tc, B, qi, ctr, work);
    k_wf_shade<MODE, COUNT><<<light_blocks, kWfBlock, 0, st>>>(S, pc, B, qi, work);
    L += 3;
    if (MODE != 0) {
      k_wf_shadow<MODE, COUNT><<<trace_blocks, kWfBlock, smem, st>>>(S, tc, B, ctr, work);
      ++L;
    }
    qi ^= 1;
  }
  if (wf < segments) {
    if (COUNT) {
      // The counting instantiation keeps every segment a wavefront step.
      for (uint32_t seg = wf; seg < segments; ++seg) {
        k_wf_reset<<<1, 32, 0, st>>>(B.counts, qi ^ 1);
        k_wf_extend<COUNT><<<trace_blocks, kWfBlock, smem, st>>>(S, tc, B, qi, ctr, work);
        k_wf_shade<MODE, COUNT><<<light_blocks, kWfBlock, 0, st>>>(S, pc, B, qi, work);
        L += 3;
        if (MODE != 0) {
          k_wf_shadow<MODE, COUNT><<<trace_blocks, kWfBlock, smem, st>>>(S, tc, B, ctr, work);
          ++L;
        }
        qi ^= 1;
      }
    } else {
      k_wf_reset<<<1, 32, 0, st>>>(B.counts, qi ^ 1);
      k_wf_tail<MODE><<<trace_blocks, kWfBlock, smem, st>>>(S, tc, pc, B, qi, ctr);
      L += 2;
    }
  }
  k_wf_accumulate<<<light_blocks, kWfBlock, 0, st>>>(pc, fc, B, image);
  ++L;
  if (launches) *launches += L;
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_render_wavefront(const DevScene& S, const TraceCfg& tc, const PathCfg& pc, const FrameCfg& fc,
                                    const WfBuffers& B, float4* image, Counters* ctr, unsigned long long* work,
                                    uint32_t* launches, cudaStream_t st) {
  const uint32_t total = fc.W * fc.H * pc.spp;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  switch (pc.nee_mode) {
    case 0:
      return work ? run<0, true>(S, tc, pc, fc, B, total, sms, image, ctr, work, launches, st)
                  : run<0, false>(S, tc, pc, fc, B, total, sms, image, ctr, work, launches, st);
    case 1:
      return work ? run<1, true>(S, tc, pc, fc, B, total, sms, image, ctr, work, launches, st)
                  : run<1, false>(S, tc, pc, fc, B, total, sms, image, ctr, work, launches, st);
    default:
      return work ? run<2, true>(S, tc, pc, fc, B, total, sms, image, ctr, work, launches, st)
                  : run<2, false>(S, tc, pc, fc, B, total, sms, image, ctr, work, launches, st);
  }
}

}  // namespace pt
