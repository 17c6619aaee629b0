// adjoint.cu -- path-replay adjoint of the corrected estimator (nee_mode 2).
//
// Gradients of a loss of the image with respect to every material's base
// color, emissive color and perceptual roughness, from dloss/dimage.  The image
// is the mean of sample_count samples per texel (sample k of texel t is the
// forward's path with sample index k), so dloss/dL of one path is
// dloss/dimage[t] / sample_count.
//
// Two passes over the same paths, both recomputed from the RNG seeds; only the
// primal radiance of each path (its 16-byte color slot of the wavefront path
// state) is kept between them:
//   pass A (primal)  the forward wavefront frame itself (wf_render): L per path;
//   pass B (adjoint) the same paths again as a wavefront, one bounce per step:
//                    extend (the forward's traversal kernel), adjoint shade
//                    (the forward's vertex with its emission gradient),
//                    shadow rays (visibility only) and resolve (the NEE and
//                    BSDF-sample gradients), keeping per path
//                    L_rem = L minus the radiance already accounted for at
//                    earlier vertices (path-replay backpropagation, Vicini et
//                    al. 2021).
// Sampling is detached: directions, light samples, MIS weights, pdfs and
// Russian-roulette probabilities are the forward's constants, so the
// derivative of each path's radiance with respect to the parameters is an
// unbiased estimate of the gradient of the expected image.  Per vertex j with
// material m, throughput T (entering j) and loss weight delta:
//   emission   L += T Le(m) w             -> d/dLe(m)   += delta T w
//   NEE        L += T gv_l Le(ml) sc       -> d/dLe(ml)  += delta T gv_l sc,
//                                             d/dbase, d/drough via d gv_l
//   BSDF       T' = T gv / (pb pr)         -> dL/dgv_c = L_rem_c / gv_c (L_rem after
//                                             the terms of j), times d gv / d param
// The gradients are summed per block in shared memory (first kGradSlots
// materials; the rest straight into global memory) and added to the global
// sums once per block.
#include <atomic>

#include "adjoint.h"
#include "wf_common.cuh"

namespace pt {

namespace {

using namespace wf;

constexpr int kAdjBlock = 128;
constexpr uint32_t kGradSlots = 256;  // materials summed in shared memory per block

// Per-path adjoint record (6 float4): the vertex of the current segment and L_rem.
//   a0 = (n.xyz, sc)  a1 = (wo.xyz, mat)  a2 = (wi_l.xyz, mat_l)  a3 = (thr.xyz, flags)
//   a4 = (wi.xyz, -)  a5 = (L_rem.xyz, -)
constexpr uint32_t kRec = 6;
enum : uint32_t { kVert = 1u, kNee = 2u, kCont = 4u, kVisible = 8u };

struct GradSink {
  float* smem;
  float* global;
  uint32_t n_mat;
  __device__ __forceinline__ void add(uint32_t m, int field, float v) const {
    if (v == 0.0f || m >= n_mat) return;
    if (m < kGradSlots) atomicAdd(smem + m * kGradStride + field, v);
    else atomicAdd(global + (size_t)m * kGradStride + field, v);
  }
  // d loss / d (base, roughness) of material m through d gv (coef = delta * dL/dgv).
  __device__ __forceinline__ void bsdf(uint32_t m, float3 coef, const float3& db, const float3& dr) const {
    add(m, 0, coef.x * db.x);
    add(m, 1, coef.y * db.y);
    add(m, 2, coef.z * db.z);
    add(m, 6, coef.x * dr.x + coef.y * dr.y + coef.z * dr.z);
  }
};

__device__ __forceinline__ GradSink grad_begin(uint32_t* smem, float* grads, uint32_t n_mat) {
  const uint32_t slots = n_mat < kGradSlots ? n_mat : kGradSlots;
  float* g = reinterpret_cast<float*>(smem);
  for (uint32_t k = threadIdx.x; k < slots * kGradStride; k += blockDim.x) g[k] = 0.0f;
  __syncthreads();
  return GradSink{g, grads, n_mat};
}
__device__ __forceinline__ void grad_end(const GradSink& G) {
  __syncthreads();
  const uint32_t slots = G.n_mat < kGradSlots ? G.n_mat : kGradSlots;
  for (uint32_t k = threadIdx.x; k < slots * kGradStride; k += blockDim.x)
    if (G.smem[k] != 0.0f) atomicAdd(G.global + k, G.smem[k]);
}

__device__ __forceinline__ float3 path_delta(const float4* dimg, uint32_t p, uint32_t spp, float inv_n) {
  const float4 dg = dimg[p / spp];
  return v3(dg.x * inv_n, dg.y * inv_n, dg.z * inv_n);
}

// The replay's first segment: path state from the seed, L_rem = the primal L
// (the color slot the primal frame left), queue 0 = the paths with a nonzero
// loss weight.
__global__ void __launch_bounds__(kAdjBlock) k_adj_generate(PathCfg pc, FrameCfg fc, WfBuffers B, float4* rec,
                                                            const float4* __restrict__ dimg, uint32_t total) {
  const float inv_n = 1.0f / __uint2float_rn(pc.spp);
  const uint32_t warp_base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u;
  for (uint32_t base = warp_base; base < total; base += gridDim.x * blockDim.x) {
    const uint32_t p = base + lane_id();
    bool alive = false;
    if (p < total) {
      const float4 L = B.s[4 * (size_t)p + 3];
      rec[kRec * (size_t)p + 5] = L;
      rec[kRec * (size_t)p + 3] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      const uint32_t texel = p / pc.spp, s = p % pc.spp;
      PathState ps;
      path_begin(ps, pc, fc.ivp, fc.eye, texel % fc.W, texel / fc.W, fc.W, fc.H, fc.acc * pc.spp + s);
      store_state(B, p, ps);
      const float3 d = path_delta(dimg, p, pc.spp, inv_n);
      alive = (ps.flags & kAlive) != 0u && (d.x != 0.0f || d.y != 0.0f || d.z != 0.0f);
    }
    const uint32_t slot = warp_append(alive, B.counts + 0);
    if (alive) B.q[0][slot] = p;
  }
}

// The forward's vertex for every path of queue qi (hits from the extend step),
// recorded, with the gradient of its emission term; shadow requests and the
// next queue as in the forward.
__global__ void __launch_bounds__(kAdjBlock) k_adj_shade(DevScene S, PathCfg pc, WfBuffers B, float4* rec,
                                                         const float4* __restrict__ dimg, int qi, float* grads,
                                                         uint32_t n_mat) {
  extern __shared__ uint32_t smem[];
  const GradSink G = grad_begin(smem, grads, n_mat);
  const float inv_n = 1.0f / __uint2float_rn(pc.spp);
  const uint32_t n = B.counts[qi];
  const uint32_t* q = B.q[qi];
  uint32_t* qn = B.q[qi ^ 1];
  const uint32_t warp_base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u;
  for (uint32_t base = warp_base; base < n; base += gridDim.x * blockDim.x) {
    const uint32_t i = base + lane_id();
    bool alive = false, shadow = false;
    uint32_t p = 0;
    ShadowReq rq;
    rq.active = false;
    if (i < n) {
      p = q[i];
      float4* r = rec + kRec * (size_t)p;
      const float4 h0 = B.h0[p];
      Hit h;
      h.t = h0.x; h.inst = __float_as_uint(h0.y); h.slot = __float_as_uint(h0.z); h.u = h0.w; h.v = B.h1[p];
      if (h.t >= 1e30f) {
        r[3].w = __uint_as_float(0u);  // the path leaves the scene: no vertex
      } else {
        PathState ps;
        load_state(B, p, ps);
        VertexRec vr;
        path_on_hit<2, true>(S, pc, ps, h, rq, &vr);
        store_state(B, p, ps);
        float3 L_rem = xyz(r[5]);
        if (vr.w_le != 0.0f) {
          const float3 d = path_delta(dimg, p, pc.spp, inv_n);
          const Material m = load_material(S, vr.mat);
          G.add(vr.mat, 3, d.x * vr.thr.x * vr.w_le);
          G.add(vr.mat, 4, d.y * vr.thr.y * vr.w_le);
          G.add(vr.mat, 5, d.z * vr.thr.z * vr.w_le);
          L_rem = sub(L_rem, muls(mul(vr.thr, m.emissive), vr.w_le));
          r[5] = make_float4(L_rem.x, L_rem.y, L_rem.z, 0.0f);
        }
        const uint32_t flags = kVert | (vr.nee ? kNee : 0u) | (vr.cont ? kCont : 0u);
        r[0] = make_float4(vr.n.x, vr.n.y, vr.n.z, vr.sc);
        r[1] = make_float4(vr.wo.x, vr.wo.y, vr.wo.z, __uint_as_float(vr.mat));
        r[2] = make_float4(vr.wi_l.x, vr.wi_l.y, vr.wi_l.z, __uint_as_float(vr.mat_l));
        r[3] = make_float4(vr.thr.x, vr.thr.y, vr.thr.z, __uint_as_float(flags));
        r[4] = make_float4(vr.wi.x, vr.wi.y, vr.wi.z, 0.0f);
        alive = vr.cont;
        shadow = vr.nee;
      }
    }
    const uint32_t ns = warp_append(alive, B.counts + (qi ^ 1));
    if (alive) qn[ns] = p;
    const uint32_t ss = warp_append(shadow, B.counts + 2);
    if (shadow) {
      float4* e = B.shadow + 4 * (size_t)ss;
      e[0] = make_float4(rq.o.x, rq.o.y, rq.o.z, rq.limit);
      e[1] = make_float4(rq.d.x, rq.d.y, rq.d.z, __uint_as_float(p));
    }
  }
  grad_end(G);
}

// Visibility of every shadow request (an occlusion query), into its path's flags.
__global__ void __launch_bounds__(kAdjBlock, 8) k_adj_shadow(DevScene S, TraceCfg tc, WfBuffers B, float4* rec,
                                                          Counters* ctr) {
  extern __shared__ uint32_t smem[];
  uint32_t* stk = smem + threadIdx.x;
  const TraceCold C = trace_cold(stk, blockDim.x, tc);
  const uint32_t n = B.counts[2];
  uint32_t* cursor = B.counts + 5;
  TraceState T;
  T.next = kActDone;
  uint32_t e_idx = 0;
  float limit = 0.0f;
  bool busy = false, drained = false;
  auto finish = [&](float t) {
    const uint32_t p = __float_as_uint(B.shadow[4 * (size_t)e_idx + 1].w);
    float4* r = rec + kRec * (size_t)p;
    if (!(t < limit)) r[3].w = __uint_as_float(__float_as_uint(r[3].w) | kVisible);
  };
  while (true) {
    if (!drained) {
      const uint32_t i = warp_fetch(!busy, cursor, n);
      drained = __any_sync(0xffffffffu, !busy && i == 0xffffffffu);
      if (i != 0xffffffffu) {
        e_idx = i;
        const float4 a = B.shadow[4 * (size_t)i], b = B.shadow[4 * (size_t)i + 1];
        limit = a.w;
        busy = true;
        if (trace_init<true>(T, C, S, xyz(a), xyz(b), occ_limit(tc, limit))) {
          busy = false;
          finish(T.rec_t);
        }
      }
    }
    if (!__any_sync(0xffffffffu, busy)) {
      if (drained) break;
      continue;
    }
    do {
      const uint32_t act = pick_action(busy, T.next, tc.step_policy);
      if (busy && T.next == act && trace_do<false>(act, T, S, stk, blockDim.x, tc, ctr, nullptr)) {
        busy = false;
        finish(T.rec_t);
      }
    } while (!time_to_refill(busy, drained));
  }
}

// The NEE term (when its shadow ray reached the light) and the BSDF sample of
// every vertex recorded for queue qi.
// Eight blocks per SM (64 registers, 12 bytes of spill) rather than the seven
// that 69 registers allow: backward pass of the 512^2 x 64 spp Cornell
// workload 145.3 -> 143.1 ms.
__global__ void __launch_bounds__(kAdjBlock, 8) k_adj_resolve(DevScene S, PathCfg pc, WfBuffers B, float4* rec,
                                                           const float4* __restrict__ dimg, int qi, float* grads,
                                                           uint32_t n_mat) {
  extern __shared__ uint32_t smem[];
  const GradSink G = grad_begin(smem, grads, n_mat);
  const float inv_n = 1.0f / __uint2float_rn(pc.spp);
  const uint32_t n = B.counts[qi];
  const uint32_t* q = B.q[qi];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t p = q[i];
    float4* r = rec + kRec * (size_t)p;
    const float4 a3 = r[3];
    const uint32_t flags = __float_as_uint(a3.w);
    if (!(flags & kVert)) continue;
    const float4 a0 = r[0], a1 = r[1];
    const float3 nn = xyz(a0), wo = xyz(a1), Tv = xyz(a3);
    const uint32_t mi = __float_as_uint(a1.w);
    const Material m = load_material(S, mi);
    const float3 d = path_delta(dimg, p, pc.spp, inv_n);
    float3 L_rem = xyz(r[5]);
    if ((flags & kNee) && (flags & kVisible)) {
      const float4 a2 = r[2];
      const float3 wl = xyz(a2);
      const uint32_t ml = __float_as_uint(a2.w);
      const float sc = a0.w;
      const float3 gl = eval_g(nn, wo, wl, m);
      const float3 Le = load_material(S, ml).emissive;
      G.add(ml, 3, d.x * Tv.x * gl.x * sc);
      G.add(ml, 4, d.y * Tv.y * gl.y * sc);
      G.add(ml, 5, d.z * Tv.z * gl.z * sc);
      float3 db, dr;
      eval_g_grad(nn, wo, wl, m, db, dr);
      G.bsdf(mi, muls(mul(mul(d, Tv), Le), sc), db, dr);
      L_rem = sub(L_rem, muls(mul(mul(Tv, gl), Le), sc));
      r[5] = make_float4(L_rem.x, L_rem.y, L_rem.z, 0.0f);
    }
    if (flags & kCont) {
      const float3 wi = xyz(r[4]);
      const float3 gv = eval_g(nn, wo, wi, m);
      float3 db, dr;
      eval_g_grad(nn, wo, wi, m, db, dr);
      const float3 coef = v3(gv.x != 0.0f ? d.x * L_rem.x / gv.x : 0.0f, gv.y != 0.0f ? d.y * L_rem.y / gv.y : 0.0f,
                             gv.z != 0.0f ? d.z * L_rem.z / gv.z : 0.0f);
      G.bsdf(mi, coef, db, dr);
    }
  }
  grad_end(G);
}

template <typename K>
cudaError_t smem_limit(K kernel) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
}

}  // namespace

cudaError_t launch_backward(const DevScene& S, const TraceCfg& tc, const PathCfg& pc, const FrameCfg& fc,
                            const WfBuffers& B, float4* rec, float4* primal_image, uint32_t wf_segments,
                            uint32_t trace_blocks, const float4* dimg, float* grads, uint32_t n_mat, Counters* ctr,
                            uint32_t* launches, cudaStream_t st) {
  // Pass A: the forward frame (spp = the sample count).
  const WfScene one = wf_scene(S, pc, fc, primal_image);
  cudaError_t e = wf_render(2, tc, &one, 1, wf_segments, trace_blocks, B, ctr, nullptr, launches, st);
  if (e != cudaSuccess) return e;
  // Pass B.
  static std::atomic<uint64_t> attr_done{0};
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint64_t bit = dev < 64 ? (uint64_t)1 << dev : 0;
  if (!(attr_done.load() & bit)) {
    e = smem_limit(k_adj_shade);
    if (e == cudaSuccess) e = smem_limit(k_adj_shadow);
    if (e == cudaSuccess) e = smem_limit(k_adj_resolve);
    if (e != cudaSuccess) return e;
    attr_done.fetch_or(bit);
  }
  const uint32_t slots = n_mat < kGradSlots ? n_mat : kGradSlots;
  const size_t smem_g = (size_t)slots * kGradStride * 4;
  const size_t smem_t = (size_t)trace_smem_words(tc) * kAdjBlock * 4;
  const int light_blocks = sms * 16;
  const int trace_grid = sms * (int)(trace_blocks ? trace_blocks : kDefaultTraceBlocks);
  uint32_t n = 0;
  e = cudaMemsetAsync(B.counts, 0, 8 * sizeof(uint32_t), st);
  if (e != cudaSuccess) return e;
  k_adj_generate<<<light_blocks, kAdjBlock, 0, st>>>(pc, fc, B, rec, dimg, one.paths);
  ++n;
  int qi = 0;
  for (uint32_t seg = 0; seg < pc.max_depth; ++seg) {
    if ((e = wf_reset_step(B, qi ^ 1, st)) != cudaSuccess) return e;
    if ((e = wf_extend_step(tc, B, qi, trace_blocks, ctr, st)) != cudaSuccess) return e;
    k_adj_shade<<<light_blocks, kAdjBlock, smem_g, st>>>(S, pc, B, rec, dimg, qi, grads, n_mat);
    k_adj_shadow<<<trace_grid, kAdjBlock, smem_t, st>>>(S, tc, B, rec, ctr);
    k_adj_resolve<<<light_blocks, kAdjBlock, smem_g, st>>>(S, pc, B, rec, dimg, qi, grads, n_mat);
    n += 5;
    qi ^= 1;
  }
  if (launches) *launches += n;
  return cudaGetLastError();
}

}  // namespace pt
