// pt_trace.cuh -- closest-hit TLAS -> BLAS traversal on the device.
//
// Restates trace_ray / traverse_tlas / traverse_blas / ray_aabb_intersect /
// ray_triangle_intersect (src/utilities.wgsl:112-114, :127-188, :259-326,
// :405-426, :430-460) with the reference's arithmetic, so the closest-hit
// primitive IDs, t, u and v are bit-identical to the CPU restatement.
//
// Layout used on the device (built by the library at upload):
//   nodes       float4 pairs (min.xyz | a) (max.xyz | count) -- the 32 B std430 node
//   tri_bvh     three float4 per BVH slot of every mesh: (p0 | tri id), (p1 - p0), (p2 - p0)
//               i.e. primitives[triangle_offset + triangle_indices[index_offset + slot]]
//               pre-gathered into BVH order with the two Moller-Trumbore edges pre-subtracted
//               (same IEEE subtraction, same bits); 48 B per test instead of 4 + 48 B.
//   instances   ten float4 per instance (the 160 B std430 record).
// The two stacks (TLAS, BLAS) live in shared memory, entry i of a thread at
// stack[i * stride + lane] so a warp's pushes hit 32 different banks.
#pragma once
#include "pt_math.cuh"

namespace pt {

struct DevScene {
  const float4* __restrict__ tri_bvh;        // 3 x float4 per global slot
  const float4* __restrict__ primitives;     // 3 x float4 per triangle (mesh order)
  const float4* __restrict__ triangle_data;  // 5 x float4 per triangle
  const uint32_t* __restrict__ triangle_indices;
  const float4* __restrict__ blas_nodes;     // 2 x float4 per node
  const float4* __restrict__ tlas_nodes;     // 2 x float4 per node
  const uint32_t* __restrict__ instance_indices;
  const float4* __restrict__ instances;      // 10 x float4 per instance
  const float4* __restrict__ materials;      // 3 x float4 per material
  const float* __restrict__ strength_cdf;
  const float* __restrict__ tri_cdfs;
  const float* __restrict__ mesh_areas;
  const uint2* __restrict__ light_indices;
  const int32_t* __restrict__ inst_light;    // instance -> light index, -1 if none
  uint32_t instance_count, light_count;
};

struct TraceCfg {
  uint32_t stack_depth;  // entries per level
  uint32_t iter_cap;
  float eps_tri, eps_par;
  bool quirks;
};

struct Hit { float t; uint32_t inst, slot; float u, v; };

struct Counters { unsigned long long rays, iter_cap_hits, stack_overflows, pad; };

__device__ __forceinline__ Hit fresh_hit() { Hit h; h.t = 1e30f; h.inst = 0u; h.slot = 0u; h.u = 0.0f; h.v = 0.0f; return h; }

__device__ __forceinline__ M4 load_m4(const float4* p) { return M4{__ldg(p), __ldg(p + 1), __ldg(p + 2), __ldg(p + 3)}; }

// src/utilities.wgsl:405-426.  Only the ordering of the returned t_min is ever
// used, so fminf/fmaxf (NaN-ignoring) give the same decisions as the lattice.
__device__ __forceinline__ float ray_aabb(float3 o, float3 d, float rec_t, float4 lo, float4 hi) {
  const float tx1 = (lo.x - o.x) / d.x;
  const float tx2 = (hi.x - o.x) / d.x;
  float tmin = fminf(tx1, tx2);
  float tmax = fmaxf(tx1, tx2);
  const float ty1 = (lo.y - o.y) / d.y;
  const float ty2 = (hi.y - o.y) / d.y;
  tmin = fmaxf(tmin, fminf(ty1, ty2));
  tmax = fminf(tmax, fmaxf(ty1, ty2));
  const float tz1 = (lo.z - o.z) / d.z;
  const float tz2 = (hi.z - o.z) / d.z;
  tmin = fmaxf(tmin, fminf(tz1, tz2));
  tmax = fminf(tmax, fmaxf(tz1, tz2));
  return (tmax >= tmin && tmin < rec_t && tmax > 0.0f) ? tmin : 1e30f;
}

// src/utilities.wgsl:430-460 on a pre-gathered slot.
__device__ __forceinline__ void ray_triangle(float3 o, float3 d, Hit& rec, const float4* tri, uint32_t slot,
                                             uint32_t inst, const TraceCfg& cfg) {
  const float4 a0 = __ldg(tri), a1 = __ldg(tri + 1), a2 = __ldg(tri + 2);
  const float3 p0 = xyz(a0), e1 = xyz(a1), e2 = xyz(a2);
  const float3 h = cross(d, e2);
  const float a = dot(e1, h);
  if (fabsf(a) < cfg.eps_par) return;
  const float f = 1.0f / a;
  const float3 s = sub(o, p0);
  const float u = f * dot(s, h);
  if (u < 0.0f || u > 1.0f) return;
  const float3 q = cross(s, e1);
  const float v = f * dot(d, q);
  if (v < 0.0f || u + v > 1.0f) return;
  const float t = f * dot(e2, q);
  if (t > cfg.eps_tri && t < rec.t) {
    rec.t = t; rec.inst = inst; rec.slot = slot; rec.u = u; rec.v = v;
  }
}

// src/utilities.wgsl:259-326.
__device__ __forceinline__ void traverse_blas(const DevScene& S, float3 wo_origin, float3 wo_dir, Hit& rec,
                                              uint32_t inst_index, uint32_t* stk, uint32_t stride,
                                              const TraceCfg& cfg, Counters* ctr) {
  const float4* ip = S.instances + (size_t)inst_index * 10;
  const M4 w2o = load_m4(ip + 4);
  const float4 offs = __ldg(ip + 8);
  const uint32_t index_offset = __float_as_uint(offs.z);
  const uint32_t node_offset = __float_as_uint(offs.w);
  const float3 o = transform_position(w2o, wo_origin);
  const float3 d = normalize(transform_direction(w2o, wo_dir));
  Hit loc = fresh_hit();
  const float4* nodes = S.blas_nodes + (size_t)node_offset * 2;
  const float4* tris = S.tri_bvh + (size_t)index_offset * 3;
  uint32_t node = 0, sp = 0, it = 0;
  bool done = false;
  while (it < cfg.iter_cap) {
    ++it;
    const float4 nlo = __ldg(nodes + 2 * node), nhi = __ldg(nodes + 2 * node + 1);
    const uint32_t na = __float_as_uint(nlo.w), ncount = __float_as_uint(nhi.w);
    if (ncount > 0u) {
      for (uint32_t i = 0; i < ncount; ++i) ray_triangle(o, d, loc, tris + (size_t)(na + i) * 3, na + i, inst_index, cfg);
      if (sp == 0) { done = true; break; }
      node = stk[(--sp) * stride];
      continue;
    }
    uint32_t ca = na, cb = na + 1;
    const float4 alo = __ldg(nodes + 2 * ca), ahi = __ldg(nodes + 2 * ca + 1);
    const float4 blo = __ldg(nodes + 2 * cb), bhi = __ldg(nodes + 2 * cb + 1);
    float da = ray_aabb(o, d, loc.t, alo, ahi);
    float db = ray_aabb(o, d, loc.t, blo, bhi);
    if (da > db) { const float tf = da; da = db; db = tf; const uint32_t tc = ca; ca = cb; cb = tc; }
    if (da == 1e30f) {
      if (sp == 0) { done = true; break; }
      node = stk[(--sp) * stride];
    } else {
      node = ca;
      if (db != 1e30f) {
        if (sp < cfg.stack_depth) stk[(sp++) * stride] = cb;
        else atomicAdd(&ctr->stack_overflows, 1ull);
      }
    }
  }
  if (!done) atomicAdd(&ctr->iter_cap_hits, 1ull);
  if (!cfg.quirks && loc.t == 1e30f) return;
  const M4 o2w = load_m4(ip);
  const float3 hit_obj = add(o, muls(d, loc.t));
  const float3 hit_world = transform_position(o2w, hit_obj);
  const float new_t = length(sub(hit_world, wo_origin));
  if (new_t < rec.t) {
    rec = loc;
    rec.t = new_t;
  }
}

// src/utilities.wgsl:127-188.  stk: this thread's stack base in shared memory;
// TLAS entries at [0, depth), BLAS entries at [depth, 2*depth).
__device__ __forceinline__ void trace_closest(const DevScene& S, float3 o, float3 d, Hit& rec, uint32_t* stk,
                                              uint32_t stride, const TraceCfg& cfg, Counters* ctr) {
  rec = fresh_hit();
  const float4* tl = S.tlas_nodes;
  {
    const float4 r0 = __ldg(tl), r1 = __ldg(tl + 1);
    if (__float_as_uint(r0.w) == 0u && __float_as_uint(r1.w) == 0u) return;
  }
  uint32_t* bstk = stk + (size_t)cfg.stack_depth * stride;
  uint32_t node = 0, sp = 0, it = 0;
  bool done = false;
  while (it < cfg.iter_cap) {
    ++it;
    const float4 nlo = __ldg(tl + 2 * node), nhi = __ldg(tl + 2 * node + 1);
    const uint32_t na = __float_as_uint(nlo.w), ncount = __float_as_uint(nhi.w);
    if (ncount > 0u) {
      for (uint32_t i = 0; i < ncount; ++i) {
        const uint32_t ii = __ldg(S.instance_indices + na + i);
        traverse_blas(S, o, d, rec, ii, bstk, stride, cfg, ctr);
      }
      if (sp == 0) { done = true; break; }
      node = stk[(--sp) * stride];
      continue;
    }
    uint32_t ca = na, cb = na + 1;
    const float4 alo = __ldg(tl + 2 * ca), ahi = __ldg(tl + 2 * ca + 1);
    const float4 blo = __ldg(tl + 2 * cb), bhi = __ldg(tl + 2 * cb + 1);
    float da = ray_aabb(o, d, rec.t, alo, ahi);
    float db = ray_aabb(o, d, rec.t, blo, bhi);
    if (da > db) { const float tf = da; da = db; db = tf; const uint32_t tc = ca; ca = cb; cb = tc; }
    if (da == 1e30f) {
      if (sp == 0) { done = true; break; }
      node = stk[(--sp) * stride];
    } else {
      node = ca;
      if (db != 1e30f) {
        if (sp < cfg.stack_depth) stk[(sp++) * stride] = cb;
        else atomicAdd(&ctr->stack_overflows, 1ull);
      }
    }
  }
  if (!done) atomicAdd(&ctr->iter_cap_hits, 1ull);
}

}  // namespace pt
