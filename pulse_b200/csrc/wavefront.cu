// wavefront.cu -- the path tracer as a wavefront of kernels over queues of live
// paths, for one scene or a batch of scenes in the same launches.
//
// Per frame: generate -> { extend -> shade } x K segments -> shadow -> tail ->
// accumulate, where each extend after the first also traces the previous
// segment's shadow requests.
//   extend  closest hit of every queued path's current ray (traversal only,
//           persistent lanes refilled in-loop), plus, in one index space after
//           the paths, the previous shading's shadow rays;
//   shade   path_on_hit of every queued path: emission, the NEE sample (queued as
//           a shadow request), BSDF sample and Russian roulette; live paths are
//           appended to the next queue;
//   shadow  the last segment's shadow requests (occlusion queries) and their
//           contributions;
//   tail    after K segments, one persistent kernel runs every remaining path to
//           its end, so the paths' long traversal tails overlap;
//   accumulate  the running mean of every texel over its samples.
// Queues are compacted with one warp ballot per append (one atomicAdd per warp).
// Every path runs exactly the megakernel's arithmetic in the same order, so
// images are bit-identical to it; shadow contributions of segment k land before
// segment k+1 is shaded, as in the sequential loop.
//
// Batches: the paths of all scenes form one id space (scene s owns
// [path_offset_s, path_offset_s + paths_s)); every kernel copies the scene table
// into shared memory and finds a path's scene by binary search, so small
// scenes fill the GPU together and their tails overlap.  All scenes of a batch
// share the estimator mode and the traversal settings.
//
// Path state (64 B, four float4 per path, path id = offset + texel * spp + sample):
//   s0 = (o.xyz, prev_pdf)  s1 = (d.xyz, rng)  s2 = (thr.xyz, depth | flags << 24)
//   s3 = (color.xyz, unused)
// Hit of the current segment: h0 = (t, inst, slot, u), h1 = v.
// Shadow request (64 B): (o.xyz, limit) (d.xyz, path) (add_vis.xyz, scene) (add_occ.xyz, -).
#include <atomic>
#include <cstring>

#include "wavefront.h"
#include "wf_common.cuh"

namespace pt {

namespace {

using namespace wf;

constexpr int kWfBlock = 128;
constexpr uint32_t kTableChunk = 8;  // table entries per upload launch (kernel parameter)

// The scene table in shared memory: [n entries of WfScene][traversal stacks].
__device__ __forceinline__ const WfScene* load_table(const WfScene* g, uint32_t n, uint32_t* smem) {
  WfScene* t = reinterpret_cast<WfScene*>(smem);
  const uint4* src = reinterpret_cast<const uint4*>(g);
  uint4* dst = reinterpret_cast<uint4*>(t);
  const uint32_t words = n * (uint32_t)(sizeof(WfScene) / sizeof(uint4));
  for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
  __syncthreads();
  return t;
}
__device__ __forceinline__ uint32_t* stacks_after(uint32_t* smem, uint32_t n) {
  return smem + n * (uint32_t)(sizeof(WfScene) / 4);
}
__device__ __forceinline__ uint32_t scene_of(const WfScene* t, uint32_t n, uint32_t p) {
  uint32_t lo = 0, hi = n;  // last scene with path_offset <= p
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (t[mid].path_offset <= p) lo = mid; else hi = mid;
  }
  return lo;
}

template <int MODE>
__global__ void __launch_bounds__(kWfBlock) k_wf_generate(WfBuffers B, uint32_t n_scenes, uint32_t total) {
  extern __shared__ uint32_t smem[];
  const WfScene* tab = load_table(B.table, n_scenes, smem);
  const uint32_t warp_base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = warp_base; base < total; base += stride) {
    const uint32_t p = base + lane_id();
    bool alive = false;
    if (p < total) {
      const WfScene& sc = tab[scene_of(tab, n_scenes, p)];
      const uint32_t local = p - sc.path_offset;
      const uint32_t texel = local / sc.pc.spp, s = local % sc.pc.spp;
      const uint32_t x = texel % sc.fc.W, y = texel / sc.fc.W;
      PathState ps;
      path_begin(ps, sc.pc, sc.fc.ivp, sc.fc.eye, x, y, sc.fc.W, sc.fc.H, sc.fc.acc * sc.pc.spp + s);
      store_state(B, p, ps);
      alive = (ps.flags & kAlive) != 0u;
    }
    const uint32_t slot = warp_append(alive, B.counts + 0);
    if (alive) B.q[0][slot] = p;
  }
}

// Shadow request slot ss of path p of scene sid.
__device__ __forceinline__ void put_shadow(const WfBuffers& B, uint32_t ss, const ShadowReq& rq, uint32_t p,
                                           uint32_t sid) {
  float4* e = B.shadow + 4 * (size_t)ss;
  e[0] = make_float4(rq.o.x, rq.o.y, rq.o.z, rq.limit);
  e[1] = make_float4(rq.d.x, rq.d.y, rq.d.z, __uint_as_float(p));
  e[2] = make_float4(rq.add_vis.x, rq.add_vis.y, rq.add_vis.z, __uint_as_float(sid));
  e[3] = make_float4(rq.add_occ.x, rq.add_occ.y, rq.add_occ.z, 0.0f);
}

// Sample s of the realtime GI pass (src/pulse/gi.wgsl:56-83): one path per
// output texel, its first vertex at the G-buffer texel the reference reads
// (gi.wgsl:61-67: texel = u32(x / W * GW)); sample 0 seeds the random state,
// later samples continue the state the previous sample's path ended with.
__global__ void __launch_bounds__(kWfBlock) k_gi_generate(WfBuffers B, const float4* __restrict__ gbuf, uint32_t gw,
                                                          uint32_t gh, uint32_t s) {
  extern __shared__ uint32_t smem[];
  const WfScene* tab = load_table(B.table, 1, smem);
  const WfScene& sc = tab[0];
  const uint32_t W = sc.fc.W, H = sc.fc.H, total = W * H;
  const uint32_t warp_base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = warp_base; base < total; base += stride) {
    const uint32_t p = base + lane_id();
    bool alive = false;
    ShadowReq rq;
    rq.active = false;
    PathState ps;
    if (p < total) {
      const uint32_t x = p % W, y = p / W;
      const float ux = __uint2float_rn(x) / __uint2float_rn(W), uy = __uint2float_rn(y) / __uint2float_rn(H);
      uint32_t gx = (uint32_t)(ux * __uint2float_rn(gw)), gy = (uint32_t)(uy * __uint2float_rn(gh));
      gx = gx < gw ? gx : gw - 1;
      gy = gy < gh ? gy : gh - 1;
      const GTexel g = load_gtexel(gbuf, (size_t)gy * gw + gx);
      ps.rng = s == 0 ? gi_seed(p, sc.pc.seed) : __float_as_uint(B.s[4 * (size_t)p + 1].w);
      gi_begin(sc.S, sc.pc, g, ps, rq);
      alive = (ps.flags & kAlive) != 0u;
    }
    const uint32_t slot = warp_append(alive, B.counts + 0);
    if (alive) B.q[0][slot] = p;
    const uint32_t ss = warp_append(rq.active, B.counts + 2);
    if (p < total) store_state(B, p, ps);
    if (rq.active) put_shadow(B, ss, rq, p, 0);
  }
}

// The camera ray of every texel (path_begin), queued in texel order.
__global__ void __launch_bounds__(kWfBlock) k_gbuf_generate(WfBuffers B) {
  extern __shared__ uint32_t smem[];
  const WfScene* tab = load_table(B.table, 1, smem);
  const WfScene& sc = tab[0];
  const uint32_t total = sc.fc.W * sc.fc.H;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < total; p += gridDim.x * blockDim.x) {
    PathState ps;
    path_begin(ps, sc.pc, sc.fc.ivp, sc.fc.eye, p % sc.fc.W, p / sc.fc.W, sc.fc.W, sc.fc.H, 0);
    ps.flags = kAlive;
    store_state(B, p, ps);
    B.q[0][p] = p;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) B.counts[0] = total;
}

// G-buffer texel of every texel's closest hit (path_tracer.wgsl:89-100):
// position + valid flag, interpolated world normal, base color, emissive; a
// miss writes zeros.
__global__ void __launch_bounds__(kWfBlock) k_gbuf_write(WfBuffers B, float4* __restrict__ gbuf) {
  extern __shared__ uint32_t smem[];
  const WfScene* tab = load_table(B.table, 1, smem);
  const WfScene& sc = tab[0];
  const uint32_t total = sc.fc.W * sc.fc.H;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < total; p += gridDim.x * blockDim.x) {
    const float4 h0 = B.h0[p];
    float4* o = gbuf + 4 * (size_t)p;
    if (h0.x >= 1e30f) {
      const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      o[0] = z; o[1] = z; o[2] = z; o[3] = z;
      continue;
    }
    PathState ps;
    load_state(B, p, ps);
    Hit h;
    h.t = h0.x; h.inst = __float_as_uint(h0.y); h.slot = __float_as_uint(h0.z); h.u = h0.w; h.v = B.h1[p];
    ShadeGeom g;
    shade_geom(sc.S, ps, h, g);
    o[0] = make_float4(g.pos.x, g.pos.y, g.pos.z, __uint_as_float(1u));
    o[1] = make_float4(g.n.x, g.n.y, g.n.z, 0.0f);
    o[2] = make_float4(g.m.base.x, g.m.base.y, g.m.base.z, 0.0f);
    o[3] = make_float4(g.m.emissive.x, g.m.emissive.y, g.m.emissive.z, 0.0f);
  }
}

// color_out += color * spp_inv (src/pulse/gi.wgsl:125), stored with alpha 1
// (gi.wgsl:131) after every sample.
__global__ void __launch_bounds__(kWfBlock) k_gi_resolve(WfBuffers B, float4* image, uint32_t total, uint32_t s,
                                                         float spp_inv) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < total; p += gridDim.x * blockDim.x) {
    const float3 c = xyz(B.s[4 * (size_t)p + 3]);
    const float3 prev = s == 0 ? v3(0.0f, 0.0f, 0.0f) : xyz(image[p]);
    const float3 out = add(prev, muls(c, spp_inv));
    image[p] = make_float4(out.x, out.y, out.z, 1.0f);
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

// Closest hit of every path of queue qi into h0/h1.  SHADOW >= 0 (estimator
// mode of the frame) also resolves the shadow requests of the previous
// segment (counts[3] of them) in the same persistent launch: they only add to
// their paths' colors, which nothing reads before the next shading.
// Persistent traversal kernels take their block size BS as a template
// parameter: MINB resident 128-thread blocks per SM become MINB * 128 / BS
// blocks of BS threads (the same threads per SM and register budget).
template <bool COUNT, int MINB, int SHADOW = -1, int BS = kWfBlock>
__global__ void __launch_bounds__(BS, MINB * kWfBlock / BS) k_wf_extend(TraceCfg tc, WfBuffers B, uint32_t n_scenes,
                                                                         int qi, Counters* ctr,
                                                                         unsigned long long* work) {
  extern __shared__ uint32_t smem[];
  const WfScene* tab = load_table(B.table, n_scenes, smem);
  uint32_t* stk = stacks_after(smem, n_scenes) + threadIdx.x;
  const TraceCold C = trace_cold(stk, blockDim.x, tc);
  const uint32_t n = B.counts[qi];
  const uint32_t n_all = SHADOW >= 0 ? n + B.counts[3] : n;
  const uint32_t* q = B.q[qi];
  uint32_t* cursor = B.counts + 4;
  WorkCount wc{};
  TraceState T;
  uint32_t p = 0, sid = 0;
  bool busy = false, drained = false;
  while (true) {
    if (!drained) {
      const uint32_t i = warp_fetch(!busy, cursor, n_all);
      // A lane that asked and got nothing means the queue is exhausted.
      drained = __any_sync(0xffffffffu, !busy && i == 0xffffffffu);
      if (i != 0xffffffffu) {
        if (SHADOW >= 0 && i >= n) {
          // p holds the request index, marked by the top bit
          p = (i - n) | 0x80000000u;
          const float4* e = B.shadow + 4 * (size_t)(i - n);
          const float4 a = e[0], b = e[1];
          sid = __float_as_uint(e[2].w);
          busy = !trace_init<true>(T, C, tab[sid].S, xyz(a), xyz(b), occ_limit(tc, a.w));
          if (!busy) finish_shadow<SHADOW < 0 ? 0 : SHADOW>(B, i - n, T.rec_t);
        } else {
          p = q[i];
          sid = scene_of(tab, n_scenes, p);
          const float4 a = B.s[4 * (size_t)p], b = B.s[4 * (size_t)p + 1];
          if (COUNT) wc.rays++;
          busy = SHADOW >= 0 ? !trace_init<true>(T, C, tab[sid].S, xyz(a), xyz(b)) : !trace_init(T, C, tab[sid].S, xyz(a), xyz(b));
          if (!busy) {
            const Hit r = trace_result(T, C);
            B.h0[p] = make_float4(r.t, __uint_as_float(r.inst), __uint_as_float(r.slot), r.u);
            B.h1[p] = r.v;
          }
        }
      }
    }
    if (!__any_sync(0xffffffffu, busy)) {
      if (drained) break;
      continue;
    }
    do {
      const uint32_t act = pick_action(busy, T.next, tc.step_policy);
      if (busy && T.next == act && trace_do<COUNT>(act, T, tab[sid].S, stk, blockDim.x, tc, ctr, &wc)) {
        busy = false;
        if (SHADOW >= 0 && (p & 0x80000000u)) {
          finish_shadow<SHADOW < 0 ? 0 : SHADOW>(B, p & 0x7fffffffu, T.rec_t);
          continue;
        }
        const Hit r = trace_result(T, C);
        B.h0[p] = make_float4(r.t, __uint_as_float(r.inst), __uint_as_float(r.slot), r.u);
        B.h1[p] = r.v;
        if (COUNT && r.t < 1e30f) wc.hits++;
      }
    } while (!time_to_refill(busy, drained));
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

// Six blocks per SM (80 registers, 60 / 96 bytes of spill) rather than the
// four that 102 spill-free registers allow: the shading waits on dependent
// loads (light CDF search, triangle and material records) and gains from the
// warps.  1080p sphere frame 145.6 -> 146.2 Mpaths/s; eight blocks (64
// registers) 146.1.
constexpr int kShadeBlocks = 6;

template <int MODE, bool COUNT>
__global__ void __launch_bounds__(kWfBlock, kShadeBlocks) k_wf_shade(WfBuffers B, uint32_t n_scenes, int qi,
                                                       unsigned long long* work) {
  extern __shared__ uint32_t smem[];
  const WfScene* tab = load_table(B.table, n_scenes, smem);
  const uint32_t n = B.counts[qi];
  const uint32_t* q = B.q[qi];
  uint32_t* qn = B.q[qi ^ 1];
  const uint32_t warp_base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u;
  const uint32_t stride = gridDim.x * blockDim.x;
  uint32_t nee = 0;
  for (uint32_t base = warp_base; base < n; base += stride) {
    const uint32_t i = base + lane_id();
    bool alive = false, shadow = false;
    uint32_t p = 0, sid = 0;
    ShadowReq rq;
    rq.active = false;
    PathState ps;
    if (i < n) {
      p = q[i];
      sid = scene_of(tab, n_scenes, p);
      load_state(B, p, ps);
      const float4 h0 = B.h0[p];
      Hit h;
      h.t = h0.x; h.inst = __float_as_uint(h0.y); h.slot = __float_as_uint(h0.z); h.u = h0.w; h.v = B.h1[p];
      path_on_hit<MODE>(tab[sid].S, tab[sid].pc, ps, h, rq);
      alive = (ps.flags & kAlive) != 0u;
      shadow = rq.active;
    }
    const uint32_t ns = warp_append(alive, B.counts + (qi ^ 1));
    if (alive) qn[ns] = p;
    const uint32_t ss = warp_append(shadow, B.counts + 2);
    if (i < n) store_state(B, p, ps);
    if (shadow) {
      put_shadow(B, ss, rq, p, sid);
      ++nee;
    }
  }
  if (COUNT) {
    unsigned long long x = nee;
    for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
    if (lane_id() == 0) atomicAdd(work + 6, x);
  }
}


template <int MODE, bool COUNT, int MINB, int BS = kWfBlock>
__global__ void __launch_bounds__(BS, MINB * kWfBlock / BS) k_wf_shadow(TraceCfg tc, WfBuffers B, uint32_t n_scenes,
                                                                         Counters* ctr, unsigned long long* work) {
  extern __shared__ uint32_t smem[];
  const WfScene* tab = load_table(B.table, n_scenes, smem);
  uint32_t* stk = stacks_after(smem, n_scenes) + threadIdx.x;
  const TraceCold C = trace_cold(stk, blockDim.x, tc);
  const uint32_t n = B.counts[2];
  uint32_t* cursor = B.counts + 5;
  WorkCount wc{};
  TraceState T;
  uint32_t e_idx = 0, sid = 0;
  bool busy = false, drained = false;
  while (true) {
    if (!drained) {
      const uint32_t i = warp_fetch(!busy, cursor, n);
      drained = __any_sync(0xffffffffu, !busy && i == 0xffffffffu);
      if (i != 0xffffffffu) {
        e_idx = i;
        const float4* e = B.shadow + 4 * (size_t)i;
        const float4 a = e[0], b = e[1];
        sid = __float_as_uint(e[2].w);
        if (COUNT) wc.rays++;
        busy = true;
        if (trace_init<!COUNT>(T, C, tab[sid].S, xyz(a), xyz(b), occ_limit(tc, a.w))) {
          busy = false;
          finish_shadow<MODE>(B, e_idx, T.rec_t);
        }
      }
    }
    if (!__any_sync(0xffffffffu, busy)) {
      if (drained) break;
      continue;
    }
    do {
      const uint32_t act = pick_action(busy, T.next, tc.step_policy);
      if (busy && T.next == act && trace_do<COUNT>(act, T, tab[sid].S, stk, blockDim.x, tc, ctr, &wc)) {
        busy = false;
        finish_shadow<MODE>(B, e_idx, T.rec_t);
      }
    } while (!time_to_refill(busy, drained));
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

// The tail's shading as a call: the traversal steps around it then keep their
// own register allocation (the call's body runs once per bounce against tens
// of traversal steps).  1080p sphere frame 144.0 -> 146.9 Mpaths/s, the
// 512^2 x 64 spp Cornell frame 98.3 -> 96.4 ms.
template <int MODE>
__device__ __noinline__ void tail_shade(const DevScene& S, const PathCfg& c, PathState& ps, const Hit& h,
                                        ShadowReq& rq) {
  path_on_hit<MODE>(S, c, ps, h, rq);
}

// The tail: one persistent kernel takes every path still alive after the
// wavefront segments and runs it to the end (segment, shading, shadow ray,
// ...), each lane fetching a new path when its own ends.
template <int MODE, int MINB, int BS = kWfBlock>
__global__ void __launch_bounds__(BS, MINB * kWfBlock / BS) k_wf_tail(TraceCfg tc, WfBuffers B, uint32_t n_scenes,
                                                                       int qi, Counters* ctr) {
  extern __shared__ uint32_t smem[];
  const WfScene* tab = load_table(B.table, n_scenes, smem);
  uint32_t* stk = stacks_after(smem, n_scenes) + threadIdx.x;
  const TraceCold C = trace_cold(stk, blockDim.x, tc);
  const uint32_t n = B.counts[qi];
  const uint32_t* q = B.q[qi];
  uint32_t* cursor = B.counts + 6;
  PathState ps;
  ShadowReq rq;
  rq.active = false;
  TraceState T;
  T.next = kActDone;
  uint32_t p = 0, sid = 0;
  // A busy lane is tracing a ray (T.next says the action) or holds a finished
  // ray whose shading is pending; shading is one more action class for the
  // warp's step, so the lanes that shade do it together.
  bool busy = false, shadow = false, tracing = false, drained = false;
  while (true) {
    if (!drained) {
      const uint32_t i = warp_fetch(!busy, cursor, n);
      drained = __any_sync(0xffffffffu, !busy && i == 0xffffffffu);
      if (i != 0xffffffffu) {
        p = q[i];
        sid = scene_of(tab, n_scenes, p);
        load_state(B, p, ps);
        busy = true;
        shadow = false;
        tracing = !trace_init<true>(T, C, tab[sid].S, ps.o, ps.d);
      }
    }
    if (!__any_sync(0xffffffffu, busy)) {
      if (drained) break;
      continue;
    }
    do {
      const uint32_t cls = tracing ? T.next : kActShade;
      const uint32_t act = pick_action(busy, cls, tc.step_policy, kShadeWeight);
      if (!busy || cls != act) continue;
      const DevScene& S = tab[sid].S;
      if (act != kActShade) {
        if (trace_do<false>(act, T, S, stk, blockDim.x, tc, ctr, nullptr)) tracing = false;
        continue;
      }
      // The path state stays in memory while the lane traverses (fewer live
      // registers there); shading reloads it and writes it back.
      load_state(B, p, ps);
      if (shadow) {
        path_on_shadow<MODE>(ps, rq, T.rec_t);
        shadow = false;
      } else {
        tail_shade<MODE>(S, tab[sid].pc, ps, trace_result(T, C), rq);
        shadow = rq.active;
      }
      store_state(B, p, ps);
      if (!shadow && !(ps.flags & kAlive)) {
        busy = false;
        continue;
      }
      tracing = !trace_init<true>(T, C, S, shadow ? rq.o : ps.o, shadow ? rq.d : ps.d,
                                  shadow ? occ_limit(tc, rq.limit) : 3.0e38f);
    } while (!time_to_refill(busy, drained));
  }
}

// Texels are handled by the thread of their first sample.
__global__ void __launch_bounds__(kWfBlock) k_wf_accumulate(WfBuffers B, uint32_t n_scenes, uint32_t total) {
  extern __shared__ uint32_t smem[];
  const WfScene* tab = load_table(B.table, n_scenes, smem);
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < total; p += gridDim.x * blockDim.x) {
    const WfScene& sc = tab[scene_of(tab, n_scenes, p)];
    const uint32_t local = p - sc.path_offset;
    if (local % sc.pc.spp != 0) continue;
    const uint32_t t = local / sc.pc.spp;
    float4 px = sc.fc.acc * sc.pc.spp > 0 ? sc.image[t] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    for (uint32_t s = 0; s < sc.pc.spp; ++s) {
      const float4 c = B.s[4 * ((size_t)p + s) + 3];
      px = accumulate(px, xyz(c), sc.fc.acc * sc.pc.spp + s);
    }
    sc.image[t] = px;
  }
}

// ----------------------------------------------------------------- ray sort
// Key of a queued path's ray: direction octant (3 bits) and the cell of its
// origin in an 8^3 grid over its scene's TLAS root box (9 bits).
__device__ __forceinline__ uint32_t sort_key(const WfBuffers& B, const WfScene* tab, uint32_t n_scenes, uint32_t p) {
  const WfScene& sc = tab[scene_of(tab, n_scenes, p)];
  const float4 a = B.s[4 * (size_t)p], b = B.s[4 * (size_t)p + 1];
  const uint32_t oct = (b.x < 0.0f ? 1u : 0u) | (b.y < 0.0f ? 2u : 0u) | (b.z < 0.0f ? 4u : 0u);
  const float4 lo = __ldg(sc.S.tlas_nodes), hi = __ldg(sc.S.tlas_nodes + 1);
  auto cell = [](float o, float l, float h) -> uint32_t {
    const float c = (o - l) / (h - l) * 8.0f;
    return c >= 1.0f ? (c < 7.0f ? (uint32_t)c : 7u) : 0u;  // NaN and below the box: 0
  };
  return (oct << 9) | (cell(a.x, lo.x, hi.x) << 6) | (cell(a.y, lo.y, hi.y) << 3) | cell(a.z, lo.z, hi.z);
}

__global__ void __launch_bounds__(kWfBlock) k_sort_count(WfBuffers B, uint32_t n_scenes, int qi) {
  extern __shared__ uint32_t smem[];
  const WfScene* tab = load_table(B.table, n_scenes, smem);
  const uint32_t n = B.counts[qi];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    atomicAdd(B.sort_bins + sort_key(B, tab, n_scenes, B.q[qi][i]), 1u);
}

// Exclusive scan of the kSortBins counters in place (one block of 1024 threads).
__global__ void k_sort_scan(uint32_t* bins) {
  __shared__ uint32_t ws[32];
  constexpr uint32_t kPer = kSortBins / 1024;
  uint32_t v[kPer], sum = 0;
  for (uint32_t k = 0; k < kPer; ++k) { v[k] = bins[threadIdx.x * kPer + k]; sum += v[k]; }
  uint32_t x = sum;
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t o = __shfl_up_sync(0xffffffffu, x, off);
    if ((threadIdx.x & 31) >= (uint32_t)off) x += o;
  }
  if ((threadIdx.x & 31) == 31) ws[threadIdx.x >> 5] = x;
  __syncthreads();
  if (threadIdx.x < 32) {
    uint32_t w = ws[threadIdx.x];
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t o = __shfl_up_sync(0xffffffffu, w, off);
      if (threadIdx.x >= (uint32_t)off) w += o;
    }
    ws[threadIdx.x] = w;
  }
  __syncthreads();
  uint32_t run = x - sum + ((threadIdx.x >> 5) ? ws[(threadIdx.x >> 5) - 1] : 0u);
  for (uint32_t k = 0; k < kPer; ++k) { bins[threadIdx.x * kPer + k] = run; run += v[k]; }
}

// The paths of queue qi moved into queue qi ^ 1 in key order (any order
// within a key); the count moves with them.
__global__ void __launch_bounds__(kWfBlock) k_sort_scatter(WfBuffers B, uint32_t n_scenes, int qi) {
  extern __shared__ uint32_t smem[];
  const WfScene* tab = load_table(B.table, n_scenes, smem);
  const uint32_t n = B.counts[qi];
  uint32_t* dst = B.q[qi ^ 1];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t p = B.q[qi][i];
    const uint32_t at = atomicAdd(B.sort_bins + sort_key(B, tab, n_scenes, p), 1u);
    if (at < n) dst[at] = p;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) B.counts[qi ^ 1] = n;
}

// Counters before a segment whose next queue is `next`; with snap, the shadow
// requests of the previous segment stay listed as counts[3] for a merged
// extend (see k_wf_extend).
__global__ void k_wf_reset(uint32_t* counts, int next, int snap) {
  if (threadIdx.x == 0) {
    counts[3] = snap ? counts[2] : 0u;
    counts[next] = 0; counts[2] = 0; counts[4] = 0; counts[5] = 0; counts[6] = 0;
  }
}

struct WfTableChunk { WfScene e[kTableChunk]; };

__global__ void k_wf_set_table(WfTableChunk c, WfScene* dst, uint32_t k) {
  const uint4* src = reinterpret_cast<const uint4*>(c.e);
  uint4* d = reinterpret_cast<uint4*>(dst);
  const uint32_t words = k * (uint32_t)(sizeof(WfScene) / sizeof(uint4));
  for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) d[i] = src[i];
}

int device_sms() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

template <typename K>
cudaError_t smem_attr(K kernel) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
}

// Register budgets of the persistent traversal kernels: MINB resident blocks
// per SM (1 = no bound).  More resident warps hide more of the node-load
// latency; tighter budgets spill part of the ray state to L1.
using ExtendK = void (*)(TraceCfg, WfBuffers, uint32_t, int, Counters*, unsigned long long*);
using ShadowK = void (*)(TraceCfg, WfBuffers, uint32_t, Counters*, unsigned long long*);
using TailK = void (*)(TraceCfg, WfBuffers, uint32_t, int, Counters*);

template <int SHADOW, int BS>
ExtendK extend_by_budget(int minb) {
  return minb >= 8 ? k_wf_extend<false, 8, SHADOW, BS> : minb >= 6 ? k_wf_extend<false, 6, SHADOW, BS>
         : minb >= 5 ? k_wf_extend<false, 5, SHADOW, BS> : k_wf_extend<false, 1, SHADOW, BS>;
}
// The counting instantiation runs 128-thread blocks only.
template <bool COUNT>
ExtendK extend_kernel(int minb, uint32_t block = kWfBlock) {
  if constexpr (COUNT) return k_wf_extend<true, 1>;
  else return block == 64 ? extend_by_budget<-1, 64>(minb) : extend_by_budget<-1, kWfBlock>(minb);
}
// The extend that also resolves the previous segment's shadow requests.
template <int MODE>
ExtendK extend_shadow_kernel(int minb, uint32_t block = kWfBlock) {
  return block == 64 ? extend_by_budget<MODE, 64>(minb) : extend_by_budget<MODE, kWfBlock>(minb);
}
template <int MODE, int BS>
ShadowK shadow_by_budget(int minb) {
  return minb >= 8 ? k_wf_shadow<MODE, false, 8, BS> : minb >= 6 ? k_wf_shadow<MODE, false, 6, BS>
         : minb >= 5 ? k_wf_shadow<MODE, false, 5, BS> : k_wf_shadow<MODE, false, 1, BS>;
}
template <int MODE, bool COUNT>
ShadowK shadow_kernel(int minb, uint32_t block = kWfBlock) {
  if constexpr (COUNT) return k_wf_shadow<MODE, true, 1>;
  else return block == 64 ? shadow_by_budget<MODE, 64>(minb) : shadow_by_budget<MODE, kWfBlock>(minb);
}
template <int MODE>
TailK tail_kernel(int minb, uint32_t block = kWfBlock) {
  if (block == 64) return minb >= 4 ? k_wf_tail<MODE, 4, 64> : k_wf_tail<MODE, 1, 64>;
  return minb >= 4 ? k_wf_tail<MODE, 4> : k_wf_tail<MODE, 1>;
}

// Register budget for a traversal grid of trace_blocks blocks per SM.
int budget(uint32_t trace_blocks) {
  return trace_blocks >= 8 ? 8 : trace_blocks >= 6 ? 6 : trace_blocks == 5 ? 5 : 1;
}

template <int MODE, bool COUNT>
cudaError_t raise_limits() {
  cudaError_t e = cudaSuccess;
  for (uint32_t block : {64u, (uint32_t)kWfBlock}) {
    for (int minb : {1, 5, 6, 8}) {
      if (e == cudaSuccess) e = smem_attr(extend_kernel<COUNT>(minb, block));
      if (e == cudaSuccess) e = smem_attr(shadow_kernel<MODE, COUNT>(minb, block));
      if constexpr (MODE != 0 && !COUNT)
        if (e == cudaSuccess) e = smem_attr(extend_shadow_kernel<MODE>(minb, block));
    }
    if (e == cudaSuccess) e = smem_attr(tail_kernel<MODE>(1, block));
    if (e == cudaSuccess) e = smem_attr(tail_kernel<MODE>(4, block));
  }
  if (e == cudaSuccess) e = smem_attr(k_wf_generate<MODE>);
  if (e == cudaSuccess) e = smem_attr(k_sort_count);
  if (e == cudaSuccess) e = smem_attr(k_sort_scatter);
  if (e == cudaSuccess) e = smem_attr(k_wf_shade<MODE, COUNT>);
  if (e == cudaSuccess) e = smem_attr(k_wf_accumulate);
  return e;
}

// Launch shapes of one frame.  The persistent traversal kernels run
// trace_blocks_per_sm 128-thread blocks per SM, or twice as many 64-thread
// blocks (tc.block 64).
struct Shapes {
  size_t tab, smem_trace;
  int trace_blocks, light_blocks;
  uint32_t tbps, block;
};
Shapes shapes(const TraceCfg& tc, const WfLaunch& L) {
  Shapes g;
  g.block = tc.block == 64 ? 64u : (uint32_t)kWfBlock;
  g.tab = (size_t)L.n_scenes * sizeof(WfScene);
  g.smem_trace = g.tab + (size_t)trace_smem_words(tc) * g.block * 4;
  g.tbps = L.trace_blocks_per_sm ? L.trace_blocks_per_sm : kDefaultTraceBlocks;
  g.trace_blocks = L.sms * (int)g.tbps * (int)(kWfBlock / g.block);
  g.light_blocks = L.sms * 16;
  return g;
}

// The segments of a frame whose paths are in queue 0: wavefront steps, then
// the tail kernel.  Returns the launches.  `pending`: shadow requests (counts[2]
// of them) wait to be resolved before the paths' next shading.  Between two
// wavefront segments a segment's shadow requests are resolved by the next
// segment's extend launch (one persistent launch and one drain fewer); before
// the tail they get a launch of their own (the tail kernel, at four blocks
// per SM, traces them more slowly: +17% on a frame where every path has one).
template <int MODE, bool COUNT>
uint32_t record_segments(const TraceCfg& tc, const WfBuffers& B, const WfLaunch& L, Counters* ctr,
                         unsigned long long* work, cudaStream_t st, bool pending = false) {
  const Shapes g = shapes(tc, L);
  const uint32_t ns = L.n_scenes;
  const int minb = budget(g.tbps);
  // the counting instantiation keeps 128-thread blocks
  const uint32_t tb = COUNT ? (uint32_t)kWfBlock : g.block;
  const int grid = COUNT ? L.sms * (int)g.tbps : g.trace_blocks;
  const size_t smem_tr = COUNT ? g.tab + (size_t)trace_smem_words(tc) * kWfBlock * 4 : g.smem_trace;
  const ExtendK extend = extend_kernel<COUNT>(minb, tb);
  ExtendK extend_sh = extend;
  if constexpr (MODE != 0 && !COUNT) extend_sh = extend_shadow_kernel<MODE>(minb, tb);
  const ShadowK shadow = shadow_kernel<MODE, COUNT>(minb, tb);
  const TailK tail = tail_kernel<MODE>(g.tbps >= 4 ? 4 : 1, tb);
  const bool merge = MODE != 0 && !COUNT;
  uint32_t n = 0;
  const uint32_t wf = L.wf_segments < L.segments ? L.wf_segments : L.segments;
  int qi = 0;
  auto resolve = [&]() {
    shadow<<<grid, tb, smem_tr, st>>>(tc, B, ns, ctr, work);
    ++n;
    pending = false;
  };
  if (pending && !(merge && wf > 0)) resolve();
  for (uint32_t seg = 0; seg < L.segments; ++seg) {
    if (seg >= wf && !COUNT) break;  // the counting instantiation keeps every segment a wavefront step
    if (tc.ray_sort && seg > 0) {
      // the queue of this segment's rays, reordered into the other queue
      cudaMemsetAsync(B.sort_bins, 0, kSortBins * 4, st);
      k_sort_count<<<g.light_blocks, kWfBlock, g.tab, st>>>(B, ns, qi);
      k_sort_scan<<<1, 1024, 0, st>>>(B.sort_bins);
      k_sort_scatter<<<g.light_blocks, kWfBlock, g.tab, st>>>(B, ns, qi);
      n += 3;
      qi ^= 1;
    }
    k_wf_reset<<<1, 32, 0, st>>>(B.counts, qi ^ 1, pending ? 1 : 0);
    (pending ? extend_sh : extend)<<<grid, tb, smem_tr, st>>>(tc, B, ns, qi, ctr, work);
    pending = false;
    k_wf_shade<MODE, COUNT><<<g.light_blocks, kWfBlock, g.tab, st>>>(B, ns, qi, work);
    n += 3;
    if (MODE != 0) {
      if (merge && seg + 1 < wf) pending = true;
      else resolve();
    }
    qi ^= 1;
  }
  if (pending) resolve();  // no wavefront segment follows (no bounce, or tail only)
  if (!COUNT && wf < L.segments) {
    k_wf_reset<<<1, 32, 0, st>>>(B.counts, qi ^ 1, 0);
    tail<<<grid, tb, smem_tr, st>>>(tc, B, ns, qi, ctr);
    n += 2;
  }
  return n;
}

template <int MODE, bool COUNT>
cudaError_t record(const TraceCfg& tc, const WfBuffers& B, const WfLaunch& L, Counters* ctr, unsigned long long* work,
                   uint32_t* launches, cudaStream_t st) {
  const Shapes g = shapes(tc, L);
  const uint32_t ns = L.n_scenes;
  cudaError_t e = cudaMemsetAsync(B.counts, 0, 8 * sizeof(uint32_t), st);
  if (e != cudaSuccess) return e;
  uint32_t n = 0;
  k_wf_generate<MODE><<<g.light_blocks, kWfBlock, g.tab, st>>>(B, ns, L.total_paths);
  ++n;
  n += record_segments<MODE, COUNT>(tc, B, L, ctr, work, st);
  if (L.image_wait) {
    e = cudaStreamWaitEvent(st, L.image_wait, 0);
    if (e != cudaSuccess) return e;
  }
  k_wf_accumulate<<<g.light_blocks, kWfBlock, g.tab, st>>>(B, ns, L.total_paths);
  ++n;
  if (launches) *launches += n;
  return cudaGetLastError();
}

// The realtime GI frame: per sample, the first vertices from the G-buffer,
// their shadow rays, the diffuse bounces (mode 1), and the running sum.
cudaError_t record_gi(const TraceCfg& tc, const WfBuffers& B, const WfLaunch& L, const float4* gbuf, uint32_t gw,
                      uint32_t gh, uint32_t spp, float4* image, Counters* ctr, uint32_t* launches, cudaStream_t st) {
  const Shapes g = shapes(tc, L);
  const float spp_inv = 1.0f / (float)spp;
  uint32_t n = 0;
  for (uint32_t s = 0; s < spp; ++s) {
    cudaError_t e = cudaMemsetAsync(B.counts, 0, 8 * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    k_gi_generate<<<g.light_blocks, kWfBlock, g.tab, st>>>(B, gbuf, gw, gh, s);
    n += 1 + record_segments<1, false>(tc, B, L, ctr, nullptr, st, true);
    k_gi_resolve<<<g.light_blocks, kWfBlock, 0, st>>>(B, image, L.total_paths, s, spp_inv);
    ++n;
  }
  if (launches) *launches += n;
  return cudaGetLastError();
}

}  // namespace

cudaError_t wf_prepare(int mode) {
  static std::atomic<uint64_t> done[3];  // one bit per device: limits raised
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const int m = mode < 0 ? 0 : mode > 2 ? 2 : mode;
  const uint64_t bit = dev < 64 ? (uint64_t)1 << dev : 0;
  if (bit && (done[m].load() & bit)) return cudaSuccess;
  switch (m) {
    case 0: e = raise_limits<0, false>(); if (e == cudaSuccess) e = raise_limits<0, true>(); break;
    case 1: e = raise_limits<1, false>(); if (e == cudaSuccess) e = raise_limits<1, true>(); break;
    default: e = raise_limits<2, false>(); if (e == cudaSuccess) e = raise_limits<2, true>(); break;
  }
  if (e == cudaSuccess && bit) done[m].fetch_or(bit);
  return e;
}

cudaError_t wf_record(int mode, const TraceCfg& tc, const WfBuffers& B, const WfLaunch& L, Counters* ctr,
                      unsigned long long* work, uint32_t* launches, cudaStream_t st) {
  if (cudaError_t e = wf_prepare(mode)) return e;
  switch (mode) {
    case 0:
      return work ? record<0, true>(tc, B, L, ctr, work, launches, st)
                  : record<0, false>(tc, B, L, ctr, work, launches, st);
    case 1:
      return work ? record<1, true>(tc, B, L, ctr, work, launches, st)
                  : record<1, false>(tc, B, L, ctr, work, launches, st);
    default:
      return work ? record<2, true>(tc, B, L, ctr, work, launches, st)
                  : record<2, false>(tc, B, L, ctr, work, launches, st);
  }
}

cudaError_t wf_upload_table(const WfScene* host, uint32_t n, WfScene* dev, cudaStream_t st) {
  for (uint32_t i = 0; i < n; i += kTableChunk) {
    WfTableChunk c;
    std::memset(&c, 0, sizeof(c));
    const uint32_t k = n - i < kTableChunk ? n - i : kTableChunk;
    std::memcpy(c.e, host + i, k * sizeof(WfScene));
    k_wf_set_table<<<1, 128, 0, st>>>(c, dev + i, k);
  }
  return cudaGetLastError();
}

cudaError_t wf_extend_step(const TraceCfg& tc, const WfBuffers& B, int qi, uint32_t trace_blocks, Counters* ctr,
                           cudaStream_t st) {
  if (cudaError_t e = wf_prepare(2)) return e;
  const uint32_t tbps = trace_blocks ? trace_blocks : kDefaultTraceBlocks;
  const size_t smem = sizeof(WfScene) + (size_t)trace_smem_words(tc) * kWfBlock * 4;
  extend_kernel<false>(budget(tbps))<<<device_sms() * (int)tbps, kWfBlock, smem, st>>>(tc, B, 1, qi, ctr, nullptr);
  return cudaGetLastError();
}

cudaError_t wf_reset_step(const WfBuffers& B, int next, cudaStream_t st) {
  k_wf_reset<<<1, 32, 0, st>>>(B.counts, next, 0);
  return cudaGetLastError();
}

cudaError_t wf_gbuffer_primary(const TraceCfg& tc, const WfScene& scene, float4* gbuf, uint32_t trace_blocks,
                               const WfBuffers& B, Counters* ctr, uint32_t* launches, cudaStream_t st) {
  if (cudaError_t e = wf_prepare(1)) return e;
  WfScene one = scene;
  one.pc.spp = 1;
  one.path_offset = 0;
  one.paths = one.fc.W * one.fc.H;
  TraceCfg tcs = tc;
  trace_stacks(tcs, one.S.tlas_levels, one.S.blas_levels);
  const uint32_t tbps = trace_blocks ? trace_blocks : kDefaultTraceBlocks;
  const int sms = device_sms();
  const size_t tab = sizeof(WfScene);
  const size_t smem = tab + (size_t)trace_smem_words(tcs) * kWfBlock * 4;
  cudaError_t e = wf_upload_table(&one, 1, B.table, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(B.counts, 0, 8 * sizeof(uint32_t), st);
  if (e != cudaSuccess) return e;
  k_gbuf_generate<<<sms * 16, kWfBlock, tab, st>>>(B);
  extend_kernel<false>(budget(tbps))<<<sms * (int)tbps, kWfBlock, smem, st>>>(tcs, B, 1, 0, ctr, nullptr);
  k_gbuf_write<<<sms * 16, kWfBlock, tab, st>>>(B, gbuf);
  if (launches) *launches += 4;
  return cudaGetLastError();
}

cudaError_t wf_render_gi(const TraceCfg& tc, const WfScene& scene, const float4* gbuf, uint32_t gw, uint32_t gh,
                         uint32_t wf_segments, uint32_t trace_blocks, const WfBuffers& B, Counters* ctr,
                         uint32_t* launches, cudaStream_t st) {
  if (scene.pc.spp == 0 || gw == 0 || gh == 0) return cudaErrorInvalidValue;
  if (cudaError_t e = wf_prepare(1)) return e;
  WfScene one = scene;
  one.pc.spp = 1;  // one path per texel in each sample's pass
  one.path_offset = 0;
  one.paths = one.fc.W * one.fc.H;
  WfLaunch L;
  L.n_scenes = 1;
  L.total_paths = one.paths;
  L.segments = one.pc.max_depth;
  L.wf_segments = wf_segments == kWfTailOnly ? 0u : wf_segments ? wf_segments : kDefaultGiWfSegments;
  L.trace_blocks_per_sm = trace_blocks;
  L.sms = device_sms();
  TraceCfg tcs = tc;
  trace_stacks(tcs, one.S.tlas_levels, one.S.blas_levels);
  cudaError_t e = wf_upload_table(&one, 1, B.table, st);
  if (e != cudaSuccess) return e;
  if (launches) *launches += 1;
  return record_gi(tcs, B, L, gbuf, gw, gh, scene.pc.spp, one.image, ctr, launches, st);
}

cudaError_t wf_render(int mode, const TraceCfg& tc, const WfScene* scenes, uint32_t n, uint32_t wf_segments,
                      uint32_t trace_blocks, const WfBuffers& B, Counters* ctr, unsigned long long* work,
                      uint32_t* launches, cudaStream_t st, cudaEvent_t image_wait) {
  if (n == 0 || n > kMaxBatch) return cudaErrorInvalidValue;
  WfScene tab[kMaxBatch];
  WfLaunch L;
  L.n_scenes = n;
  L.total_paths = 0;
  L.segments = 0;
  for (uint32_t i = 0; i < n; ++i) {
    tab[i] = scenes[i];
    tab[i].path_offset = L.total_paths;
    tab[i].paths = tab[i].fc.W * tab[i].fc.H * tab[i].pc.spp;
    L.total_paths += tab[i].paths;
    const uint32_t seg = tab[i].pc.max_depth + (mode == 1 ? 1u : 0u);
    if (seg > L.segments) L.segments = seg;
  }
  L.wf_segments = wf_segments == kWfTailOnly ? 0u : wf_segments ? wf_segments : kDefaultWfSegments;
  L.trace_blocks_per_sm = trace_blocks;
  L.sms = device_sms();
  L.image_wait = image_wait;
  uint32_t tl = 1, bl = 1;  // the deepest trees of the batch size the stacks
  for (uint32_t i = 0; i < n; ++i) {
    tl = tab[i].S.tlas_levels > tl ? tab[i].S.tlas_levels : tl;
    bl = tab[i].S.blas_levels > bl ? tab[i].S.blas_levels : bl;
  }
  TraceCfg tcs = tc;
  trace_stacks(tcs, tl, bl);
  cudaError_t e = wf_upload_table(tab, n, B.table, st);
  if (e != cudaSuccess) return e;
  if (launches) *launches += (n + kTableChunk - 1) / kTableChunk;
  return wf_record(mode, tcs, B, L, ctr, work, launches, st);
}

}  // namespace pt
