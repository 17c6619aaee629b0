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

// Per-thread tallies of the reference algorithm's work (only in the counting
// instantiation): TLAS interior visits, BLAS entries, BLAS interior visits,
// triangle tests, traced rays.
struct WorkCount {
  uint32_t rays, tlas_interior, blas_entries, blas_interior, tri_tests, hits, nee, cdf_reads;
};

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

// Closest hit of a world ray: traverse_tlas (src/utilities.wgsl:127-188) with
// traverse_blas (:259-326) for every instance of every TLAS leaf reached.
//
// The reference nests the BLAS loop inside the TLAS loop; here both levels run
// in ONE loop whose state says which level the visited node belongs to, so the
// threads of a warp stay converged on the shared node-visit code whichever
// level each is in.  The arithmetic and the order of every test are the
// reference's, per level:
//   * each level keeps its own stack (32 entries in the reference, pushes past
//     the depth are dropped and counted) and its own iteration cap;
//   * entering an instance transforms the ray to object space with the
//     direction normalized and a fresh local record (t = 1e30);
//   * leaving it converts the local t back to a world distance and replaces the
//     world record if smaller (including the reference's far-hit value when the
//     instance was missed, unless quirks are off).
// Two departures that leave every result bit-identical:
//   * the visited node is carried in registers on descent (a pop reloads it);
//   * cross-BLAS culling: once the world record holds a real hit (t < 1e29),
//     BLAS boxes whose object-space entry t exceeds
//        t_cull = (rec.t * 1.0001 + 1e-3 * (1 + |o_world|_inf)) * |W d| / |d|
//     are skipped (|W d| / |d| = 1 / |M d_obj| up to rounding): such a box only
//     holds hits whose world distance cannot go below rec.t, the kept boxes are
//     visited in the same relative order, so the local closest hit below t_cull
//     and its tie-breaking are the reference's, and a local miss produces the
//     far-hit value (~1e30 |M d|), which cannot replace a real hit either.
template <bool COUNT = false>
__device__ __forceinline__ void trace_closest(const DevScene& S, float3 wo, float3 wd, Hit& rec, uint32_t* stk,
                                              uint32_t stride, const TraceCfg& cfg, Counters* ctr,
                                              WorkCount* wc = nullptr) {
  rec = fresh_hit();
  if (COUNT) wc->rays++;
  const float4* tl = S.tlas_nodes;
  float4 nlo = __ldg(tl), nhi = __ldg(tl + 1);
  if (__float_as_uint(nlo.w) == 0u && __float_as_uint(nhi.w) == 0u) return;
  uint32_t* bstk = stk + (size_t)cfg.stack_depth * stride;
  // Level state.
  bool in_blas = false;
  uint32_t sp_t = 0, sp_b = 0, it_t = 0, it_b = 0;
  uint32_t leaf_next = 0, leaf_left = 0;  // instances of the current TLAS leaf still to enter
  // BLAS state.
  float3 o = wo, d = wd;                  // current ray (world at TLAS level, object in a BLAS)
  Hit loc = fresh_hit();
  float t_cull = 3.0e38f;
  uint32_t inst = 0;
  const float4* nodes = tl;
  const float4* tris = S.tri_bvh;
  const float4* ip = S.instances;
  // Finishing a BLAS or a TLAS leaf.
  bool tlas_done = false;
  while (true) {
    bool leave_blas = false;
    if (in_blas) {
      if (it_b >= cfg.iter_cap) {
        atomicAdd(&ctr->iter_cap_hits, 1ull);
        leave_blas = true;
      } else {
        ++it_b;
      }
    } else {
      if (it_t >= cfg.iter_cap) {
        atomicAdd(&ctr->iter_cap_hits, 1ull);
        break;
      }
      ++it_t;
    }
    if (!leave_blas) {
      const uint32_t na = __float_as_uint(nlo.w), ncount = __float_as_uint(nhi.w);
      if (ncount == 0u) {
        // Interior node of either level: the shared slab test of both children.
        if (COUNT) { if (in_blas) wc->blas_interior++; else wc->tlas_interior++; }
        const float4 alo = __ldg(nodes + 2 * na), ahi = __ldg(nodes + 2 * na + 1);
        const float4 blo = __ldg(nodes + 2 * na + 2), bhi = __ldg(nodes + 2 * na + 3);
        const float rt = in_blas ? loc.t : rec.t;
        float da = ray_aabb(o, d, rt, alo, ahi);
        float db = ray_aabb(o, d, rt, blo, bhi);
        if (da > t_cull) da = 1e30f;
        if (db > t_cull) db = 1e30f;
        const bool swap = da > db;
        if (swap) { const float tf = da; da = db; db = tf; }
        if (da != 1e30f) {
          if (db != 1e30f) {
            uint32_t& sp = in_blas ? sp_b : sp_t;
            uint32_t* st = in_blas ? bstk : stk;
            if (sp < cfg.stack_depth) st[(sp++) * stride] = swap ? na : na + 1;
            else atomicAdd(&ctr->stack_overflows, 1ull);
          }
          nlo = swap ? blo : alo;
          nhi = swap ? bhi : ahi;
          continue;
        }
      } else if (in_blas) {
        if (COUNT) wc->tri_tests += ncount;
        for (uint32_t i = 0; i < ncount; ++i) ray_triangle(o, d, loc, tris + (size_t)(na + i) * 3, na + i, inst, cfg);
      } else {
        leaf_next = na;
        leaf_left = ncount;
      }
      // Pop within the current level, if anything is left there.
      if (in_blas) {
        if (sp_b > 0) {
          const uint32_t nx = bstk[(--sp_b) * stride];
          nlo = __ldg(nodes + 2 * nx);
          nhi = __ldg(nodes + 2 * nx + 1);
          continue;
        }
        leave_blas = true;
      }
    }
    if (leave_blas) {
      // End of traverse_blas: back to a world distance.
      in_blas = false;
      if (cfg.quirks || loc.t != 1e30f) {
        const M4 o2w = load_m4(ip);
        const float3 hit_world = transform_position(o2w, add(o, muls(d, loc.t)));
        const float new_t = length(sub(hit_world, wo));
        if (new_t < rec.t) {
          rec = loc;
          rec.t = new_t;
        }
      }
      o = wo;
      d = wd;
      t_cull = 3.0e38f;
      nodes = tl;
    }
    if (leaf_left > 0) {
      // Enter the next instance of the TLAS leaf.
      inst = __ldg(S.instance_indices + leaf_next);
      ++leaf_next;
      --leaf_left;
      if (COUNT) wc->blas_entries++;
      ip = S.instances + (size_t)inst * 10;
      const M4 w2o = load_m4(ip + 4);
      const float4 offs = __ldg(ip + 8);
      o = transform_position(w2o, wo);
      const float3 dw = transform_direction(w2o, wd);
      const float d_len = length(dw);
      d = divs(dw, d_len);
      if (!COUNT && rec.t < 1e29f) {
        const float om = fmaxf(fmaxf(fabsf(wo.x), fabsf(wo.y)), fabsf(wo.z));
        const float tc = (rec.t * 1.0001f + 1e-3f * (1.0f + om)) * d_len / length(wd);
        if (tc == tc && tc > 0.0f) t_cull = tc;
      }
      loc = fresh_hit();
      nodes = S.blas_nodes + (size_t)__float_as_uint(offs.w) * 2;
      tris = S.tri_bvh + (size_t)__float_as_uint(offs.z) * 3;
      nlo = __ldg(nodes);
      nhi = __ldg(nodes + 1);
      sp_b = 0;
      it_b = 0;
      in_blas = true;
      continue;
    }
    // TLAS pop.
    if (sp_t == 0) { tlas_done = true; break; }
    const uint32_t nx = stk[(--sp_t) * stride];
    nlo = __ldg(tl + 2 * nx);
    nhi = __ldg(tl + 2 * nx + 1);
  }
  (void)tlas_done;
}

}  // namespace pt
