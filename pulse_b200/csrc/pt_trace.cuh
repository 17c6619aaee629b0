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
  uint32_t fast_slabs;  // every child box lies inside its parent's: the slab guard is valid
  uint32_t tlas_levels, blas_levels;  // levels of the TLAS and of the deepest BLAS (root alone: 1)
};

struct TraceCfg {
  uint32_t stack_depth;  // entries per level (the reference's stack size)
  // Entries the traversal keeps per level: min(stack_depth, levels - 1) of the
  // launch's deepest tree.  A path from the root holds at most levels - 1
  // pushed siblings, so below stack_depth nothing can overflow and results
  // equal those of a stack_depth-entry stack; at stack_depth, pushes beyond
  // it are dropped and counted as in the reference.
  uint32_t stack_t, stack_b;
  uint32_t iter_cap;
  float eps_tri, eps_par;
  bool quirks;
  // The box-skipping shortcuts (cross-BLAS culling, the occlusion queries'
  // limit culling and early exit) visit a subset of the reference's nodes in
  // its order.  That is exact only if no push is ever dropped (a skipped push
  // would leave room for a later one the reference drops) and the iteration
  // cap does not bind at a different node.  So they are on only when the
  // stacks hold every level and the cap is at least the reference's 100000
  // (set by trace_stacks; the counting frame, which runs without them, reports
  // whether the reference's cap binds).  Encoded for branch-free use:
  // cull_margin is the culling bound's 1.0001 factor, +inf when off (every
  // bound becomes inf: nothing skipped); occ_floor is the lowest occlusion
  // limit passed to the traversal, -inf when on, 3e38 when off (the query then
  // runs as a full closest-hit query and the caller compares the hit with its
  // own limit).
  bool cull;
  float cull_margin, occ_floor;
  uint32_t step_policy;  // warp step selection: 1 = every lane its own action, else pick_action weights
  // Launch shape, read by the host only: threads per block of the persistent
  // traversal kernels (64 or 128) and whether each bounce's queue is sorted.
  uint32_t block, ray_sort;
};

// Default pick_action weights, one byte each: node | tri << 8 | enter << 16 | leave << 24.
constexpr uint32_t kStepWeights = 12u | (30u << 8) | (30u << 16) | (30u << 24);

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

// Exact slab test kept out of line: the filtered test below falls back to it.
__device__ __forceinline__ float ray_aabb_exact(float3 o, float3 d, float rec_t, float4 lo, float4 hi) {
  return ray_aabb(o, d, rec_t, lo, hi);
}

// Filtered slab test.  t' = (plane - o) * r with r = 1/d (IEEE) differs from
// the reference's t = (plane - o) / d by at most 3 u |t| (u = 2^-24, normal
// range): both round the same exact quotient num/d, one through the rounded
// reciprocal.  Every decision the traversal takes from slab values -- hit
// (t_max >= t_min, t_min < rec_t, t_max > 0) and the order of two children --
// is taken from t' only when its margin exceeds kSlabTol (5x the bound, plus
// an absolute 1e-36 for subnormal values); otherwise the box is recomputed with
// the exact division.  Signs of t' are exact (num * r has the sign and the
// zeros of num / d).  NaN (d component 0 with num 0) and values near overflow
// cannot occur on a level whose guard says so (slab_guard, checked when the
// level is entered); otherwise that level uses the exact division throughout.
// Equal t_min of two children are exactly equal when both come from the same
// slab (same axis, same numerator): the reference compares identical quotients
// there.  Results are therefore the reference's bit for bit.
constexpr float kSlabTol = 1e-6f;

__device__ __forceinline__ bool near_rel(float a, float b) {
  return fabsf(a - b) <= kSlabTol * fmaxf(fabsf(a), fabsf(b)) + 1e-36f;
}

// True when the fast slab test is valid for every box of a tree whose root box
// is (lo, hi): r finite (no zero direction component) and every
// |(plane - o) * r| < 1e29 (no overflow, no collision with the 1e30 miss value).
__device__ __forceinline__ bool slab_guard(float3 o, float3 r, float4 lo, float4 hi) {
  const float mx = fmaxf(fabsf(lo.x - o.x), fabsf(hi.x - o.x)) * fabsf(r.x);
  const float my = fmaxf(fabsf(lo.y - o.y), fabsf(hi.y - o.y)) * fabsf(r.y);
  const float mz = fmaxf(fabsf(lo.z - o.z), fabsf(hi.z - o.z)) * fabsf(r.z);
  return fmaxf(fmaxf(mx, my), mz) < 1e28f;
}

struct SlabT { float mnx, mny, mnz, tmin, tmax; };

__device__ __forceinline__ SlabT slab_t(float3 o, float3 r, float4 lo, float4 hi) {
  SlabT S;
  const float tx1 = (lo.x - o.x) * r.x, tx2 = (hi.x - o.x) * r.x;
  const float ty1 = (lo.y - o.y) * r.y, ty2 = (hi.y - o.y) * r.y;
  const float tz1 = (lo.z - o.z) * r.z, tz2 = (hi.z - o.z) * r.z;
  S.mnx = fminf(tx1, tx2);
  S.mny = fminf(ty1, ty2);
  S.mnz = fminf(tz1, tz2);
  S.tmin = fmaxf(fmaxf(S.mnx, S.mny), S.mnz);
  S.tmax = fminf(fminf(fmaxf(tx1, tx2), fmaxf(ty1, ty2)), fmaxf(tz1, tz2));
  return S;
}

// Slab (axis, numerator) giving t_min, or axis -1 when two entry values are
// within the margin of t_min (then the slab is not known exactly).
__device__ __forceinline__ int slab_key(float3 o, float4 lo, float4 hi, float3 r, const SlabT& S, float& num) {
  int axis = -1, n_near = 0;
  if (near_rel(S.mnx, S.tmin)) { ++n_near; axis = 0; num = ((lo.x - o.x) * r.x <= (hi.x - o.x) * r.x) ? lo.x - o.x : hi.x - o.x; }
  if (near_rel(S.mny, S.tmin)) { ++n_near; axis = 1; num = ((lo.y - o.y) * r.y <= (hi.y - o.y) * r.y) ? lo.y - o.y : hi.y - o.y; }
  if (near_rel(S.mnz, S.tmin)) { ++n_near; axis = 2; num = ((lo.z - o.z) * r.z <= (hi.z - o.z) * r.z) ? lo.z - o.z : hi.z - o.z; }
  return n_near == 1 ? axis : -1;
}

// Both children of an interior node: the reference's hit decisions and child
// order.  t_cull (conservative, carries its own 1e-4 margin) is applied to t'.
__device__ __forceinline__ void slab_pair(bool fast, float3 o, float3 d, float3 r, float rec_t, float t_cull,
                                          float4 alo, float4 ahi, float4 blo, float4 bhi, bool& hit_a, bool& hit_b,
                                          bool& swap) {
  float da, db;
  bool exact_a = !fast, exact_b = !fast;
  SlabT A, B;
  if (fast) {
    A = slab_t(o, r, alo, ahi);
    B = slab_t(o, r, blo, bhi);
    if (near_rel(A.tmax, A.tmin) || near_rel(A.tmin, rec_t)) exact_a = true;
    else da = (A.tmax >= A.tmin && A.tmin < rec_t && A.tmax > 0.0f) ? A.tmin : 1e30f;
    if (near_rel(B.tmax, B.tmin) || near_rel(B.tmin, rec_t)) exact_b = true;
    else db = (B.tmax >= B.tmin && B.tmin < rec_t && B.tmax > 0.0f) ? B.tmin : 1e30f;
  }
  if (exact_a) da = ray_aabb_exact(o, d, rec_t, alo, ahi);
  if (exact_b) db = ray_aabb_exact(o, d, rec_t, blo, bhi);
  if (da != 1e30f && db != 1e30f && (exact_a != exact_b || (!exact_a && near_rel(da, db)))) {
    bool same_slab = false;
    if (!exact_a && !exact_b) {
      float na = 0.0f, nb = 0.0f;
      const int ka = slab_key(o, alo, ahi, r, A, na);
      const int kb = slab_key(o, blo, bhi, r, B, nb);
      same_slab = ka >= 0 && ka == kb && __float_as_uint(na) == __float_as_uint(nb);
    }
    if (same_slab) {
      db = da;  // identical quotients in the reference: no swap
    } else if (exact_a != exact_b ? near_rel(da, db) : true) {
      if (!exact_a) da = ray_aabb_exact(o, d, rec_t, alo, ahi);
      if (!exact_b) db = ray_aabb_exact(o, d, rec_t, blo, bhi);
    }
  }
  if (da > t_cull) da = 1e30f;
  if (db > t_cull) db = 1e30f;
  hit_a = da != 1e30f;
  hit_b = db != 1e30f;
  swap = da > db;
}

// src/utilities.wgsl:430-460 on a pre-gathered slot: true when the triangle
// is hit at eps_tri < t < rec_t (t, u, v out).
__device__ __forceinline__ bool ray_triangle_v(float3 o, float3 d, float rec_t, float3 p0, float3 e1, float3 e2,
                                               const TraceCfg& cfg, float& t_out, float& u_out, float& v_out) {
  const float3 h = cross(d, e2);
  const float a = dot(e1, h);
  if (fabsf(a) < cfg.eps_par) return false;
  const float f = 1.0f / a;
  const float3 s = sub(o, p0);
  const float u = f * dot(s, h);
  if (u < 0.0f || u > 1.0f) return false;
  const float3 q = cross(s, e1);
  const float v = f * dot(d, q);
  if (v < 0.0f || u + v > 1.0f) return false;
  const float t = f * dot(e2, q);
  if (!(t > cfg.eps_tri && t < rec_t)) return false;
  t_out = t;
  u_out = u;
  v_out = v;
  return true;
}
__device__ __forceinline__ bool ray_triangle(float3 o, float3 d, float rec_t, const float4* tri, const TraceCfg& cfg,
                                             float& t_out, float& u_out, float& v_out) {
  const float4 a0 = __ldg(tri), a1 = __ldg(tri + 1), a2 = __ldg(tri + 2);
  return ray_triangle_v(o, d, rec_t, xyz(a0), xyz(a1), xyz(a2), cfg, t_out, u_out, v_out);
}

// Closest hit of a world ray: traverse_tlas (src/utilities.wgsl:127-188) with
// traverse_blas (:259-326) for every instance of every TLAS leaf reached.
//
// The reference nests the BLAS loop inside the TLAS loop; here both levels run
// in ONE loop whose state says which level the visited node belongs to.  The
// loop is written as a resumable state machine (TraceState + trace_do): each
// step performs one action -- visit a node (either level), test the next one
// or two triangles of a leaf, enter an instance, leave an instance -- and
// records the next action in
// T.next.  A warp picks one action per step for all its lanes (pick_action),
// so the lanes that execute a step run the same code; each lane still performs
// its own actions in exactly the reference's order.  The arithmetic and the
// order of every test are the reference's, per level:
//   * each level keeps its own stack (32 entries in the reference, pushes past
//     the depth are dropped and counted) and its own iteration cap;
//   * entering an instance transforms the ray to object space with the
//     direction normalized and a fresh local record (t = 1e30);
//   * leaving it converts the local t back to a world distance and replaces the
//     world record if smaller (including the reference's far-hit value when the
//     instance was missed, unless quirks are off).
// Departures that leave every result bit-identical:
//   * the visited node's a and count are carried in registers on descent,
//     and an interior node's stack entry holds them (a pop of an interior
//     node reads no memory);
//   * the filtered slab test (slab_pair);
//   * cross-BLAS culling: once the world record holds a real hit (t < 1e29),
//     BLAS boxes whose object-space entry t exceeds
//        t_cull = (rec.t * 1.0001 + 1e-3 * (1 + |o_world|_inf)) * |W d| / |d|
//     are skipped (|W d| / |d| = 1 / |M d_obj| up to rounding): such a box only
//     holds hits whose world distance cannot go below rec.t, the kept boxes are
//     visited in the same relative order, so the local closest hit below t_cull
//     and its tie-breaking are the reference's, and a local miss produces the
//     far-hit value (~1e30 |M d|), which cannot replace a real hit either.
// Occlusion queries (trace_init with a finite limit; the NEE shadow rays, whose
// only use of the closest hit is `t < limit`) add two exact shortcuts:
//   * boxes of either level whose entry distance exceeds limit (with the same
//     margins as t_cull) are skipped: every hit they hold has t >= limit;
//   * the query ends at the first triangle hit whose local t is below
//        t_exit = (limit * 0.9999 - 1e-3 * (1 + |o_world|_inf)) * |W d| / |d|,
//     i.e. whose world distance is below limit with margin: the reference's
//     closest hit can only be nearer, so `t < limit` holds; T.rec.t is then
//     set to -3e38.  A limit <= 0 (or NaN) decides `t < limit` false without a
//     traversal, as no world distance is negative.
// Both are off in the counting instantiation, whose work tallies must be the
// reference algorithm's.
enum : uint32_t { kActNode = 0, kActTri = 1, kActEnter = 2, kActLeave = 3, kActDone = 4, kActShade = 5 };
// Triangles a lane tests per triangle step, their loads in flight together
// (measured on the 1080p sphere frame: 1 -> 108, 2 -> 115.6, 3 -> 110.8,
// 4 -> 107.2 Mpaths/s; more spill registers).
constexpr int kTrisPerStep = 2;

// Weight of the shading class in kernels whose lanes also shade (the tail):
// shading costs several node visits, so it waits for more lanes.  Measured
// (weight 4 / 6 / 8 / 12): the 512^2 x 64 spp Cornell frame 87.0 / 88.7 /
// 91.3 / 98.0 ms, the 1080p sphere frame flat (116.2-116.8 Mpaths/s), the
// realtime GI frame 30.4 / 30.4 / 30.2 / 30.1 ms.
constexpr uint32_t kShadeWeight = 6;

// The ray state a step touches on every visit lives in registers (TraceState);
// the rest -- the world ray, the occlusion limit, the record's and the local
// record's ids and barycentrics, the current instance and TLAS leaf -- lives in
// shared memory after the thread's two stacks, word k at cold[k * stride]
// (TraceCold), read only when an instance is entered or left or a hit is
// recorded.  Shared memory per thread: (stack_t + stack_b + kColdWords) words.
enum ColdWord : uint32_t {
  kWoX, kWoY, kWoZ, kWdX, kWdY, kWdZ, kWiX, kWiY, kWiZ, kLimit,
  kRecInst, kRecSlot, kRecU, kRecV, kLocSlot, kLocU, kLocV, kInst, kLeafNext, kLeafLeft,
  kRecT, kSpT, kItT, kFastT,  // the TLAS level's record, stack pointer, iteration count and slab guard in a BLAS
  kColdWords
};

__host__ __device__ constexpr uint32_t trace_smem_words(const TraceCfg& tc) {
  return tc.stack_t + tc.stack_b + kColdWords;
}

// The per-level stack sizes for trees of the given levels.
__host__ __device__ inline void trace_stacks(TraceCfg& tc, uint32_t tlas_levels, uint32_t blas_levels) {
  const uint32_t t = tlas_levels > 1 ? tlas_levels - 1 : 1, b = blas_levels > 1 ? blas_levels - 1 : 1;
  tc.stack_t = t < tc.stack_depth ? t : tc.stack_depth;
  tc.stack_b = b < tc.stack_depth ? b : tc.stack_depth;
  tc.cull = tc.stack_t == t && tc.stack_b == b && tc.iter_cap >= 100000u;
  tc.cull_margin = tc.cull ? 1.0001f : INFINITY;
  tc.occ_floor = tc.cull ? -INFINITY : 3.0e38f;
}

struct TraceCold {
  uint32_t* p;
  uint32_t s;
  __device__ __forceinline__ uint32_t u(uint32_t k) const { return p[k * s]; }
  __device__ __forceinline__ float f(uint32_t k) const { return __uint_as_float(p[k * s]); }
  __device__ __forceinline__ float3 f3(uint32_t k) const { return v3(f(k), f(k + 1), f(k + 2)); }
  __device__ __forceinline__ void set(uint32_t k, uint32_t v) const { p[k * s] = v; }
  __device__ __forceinline__ void setf(uint32_t k, float v) const { p[k * s] = __float_as_uint(v); }
  __device__ __forceinline__ void setf3(uint32_t k, float3 v) const { setf(k, v.x); setf(k + 1, v.y); setf(k + 2, v.z); }
};

__device__ __forceinline__ TraceCold trace_cold(uint32_t* stk, uint32_t stride, const TraceCfg& cfg) {
  return TraceCold{stk + (cfg.stack_t + cfg.stack_b) * stride, stride};
}

// Registers hold the state of the level being traversed; while a BLAS is
// traversed, the TLAS level's record, stack pointer, iteration count and slab
// guard wait in cold words (kRecT, kSpT, kItT, kFastT) and come back when the
// instance is left.
struct TraceState {
  float3 o, d, rinv;    // current ray (world at TLAS level, object in a BLAS)
  float rec_t;          // record t of the level: the world record at the TLAS level and once the
                        // ray is finished, the local record inside a BLAS
  float t_cull;         // box entry bound of the current level
  float t_exit;         // occlusion query in a BLAS: local t below which a hit decides
  uint32_t na, ncnt;    // visited node: a (first child or first primitive) and count; in a
                        // leaf's triangle steps the next triangle and the triangles left
  const float4* nodes;
  const float4* tris;
  uint32_t sp, it;      // stack pointer and iteration count of the current level
  uint32_t next;        // action of the next step (kAct*)
  bool in_blas;
  bool fast;            // slab_guard of the current level
};

__device__ __forceinline__ float max_abs3(float3 v) { return fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fabsf(v.z)); }

// World-level box bound of an occlusion query (3e38 for a closest-hit ray).
__device__ __forceinline__ float world_cull(float limit, float3 wo) {
  return limit < 1e29f ? limit * 1.0001f + 1e-3f * (1.0f + max_abs3(wo)) : 3.0e38f;
}

// The closest hit of a finished ray (t = -3e38 when an occlusion query ended early).
__device__ __forceinline__ Hit trace_result(const TraceState& T, const TraceCold& C) {
  Hit h;
  h.t = T.rec_t;
  h.inst = C.u(kRecInst);
  h.slot = C.u(kRecSlot);
  h.u = C.f(kRecU);
  h.v = C.f(kRecV);
  return h;
}

// Returns true when the ray needs no traversal (empty scene, or an occlusion
// query whose limit is not positive).  limit < 1e29 makes it an occlusion
// query (only with OCCLUDE; the counting instantiation passes false).  Callers
// pass occ_limit(cfg, limit): without TraceCfg::cull the query runs as a full
// closest-hit query and the caller compares the hit with its own limit.
__device__ __forceinline__ float occ_limit(const TraceCfg& cfg, float limit) {
  return fmaxf(limit, cfg.occ_floor);
}

template <bool OCCLUDE = false>
__device__ __forceinline__ bool trace_init(TraceState& T, const TraceCold& C, const DevScene& S, float3 wo, float3 wd,
                                           float limit = 3.0e38f) {
  const float lim = OCCLUDE ? limit : 3.0e38f;
  const float3 winv = v3(1.0f / wd.x, 1.0f / wd.y, 1.0f / wd.z);
  C.setf3(kWoX, wo);
  C.setf3(kWdX, wd);
  C.setf3(kWiX, winv);
  C.setf(kLimit, lim);
  C.set(kRecInst, 0u);
  C.set(kRecSlot, 0u);
  C.setf(kRecU, 0.0f);
  C.setf(kRecV, 0.0f);
  C.set(kLeafLeft, 0u);
  T.rec_t = 1e30f;
  T.o = wo;
  T.d = wd;
  T.rinv = winv;
  T.t_exit = -1.0f;
  T.t_cull = OCCLUDE ? world_cull(lim, wo) : 3.0e38f;
  T.nodes = S.tlas_nodes;
  T.tris = S.tri_bvh;
  T.sp = T.it = 0;
  T.in_blas = false;
  const float4 rlo = __ldg(S.tlas_nodes), rhi = __ldg(S.tlas_nodes + 1);
  T.na = __float_as_uint(rlo.w);
  T.ncnt = __float_as_uint(rhi.w);
  T.fast = S.fast_slabs && slab_guard(wo, winv, rlo, rhi);
  const bool done = (T.na == 0u && T.ncnt == 0u) || (OCCLUDE && !(limit > 0.0f));
  T.next = done ? kActDone : kActNode;
  return done;
}

// Action picked for a warp's step: the class whose lanes give the most work
// per issued instruction (lane count x weight, the weights inversely
// proportional to each action's instruction count).  Every lane of the warp
// calls it; lanes that are not tracing pass want = false.
// step_policy 1 returns each lane's own action instead (divergent steps).
// With shade_weight > 0 the class kActShade (lanes whose ray is finished and
// whose shading is pending) takes part too.
__device__ __forceinline__ uint32_t pick_action(bool want, uint32_t next, uint32_t policy,
                                                uint32_t shade_weight = 0) {
  if (policy == 1u) return next;
  const uint32_t w = policy ? policy : kStepWeights;
  // The lane count of every class in one warp reduction: a 6-bit field per
  // class (node, tri, enter, leave, shade at bits 0, 6, 12, 18, 24); a field
  // sums at most 32 ones, so no field carries into the next.
  const uint32_t field = next < kActDone ? 6u * next : 24u;
  const bool counted = want && (next < kActDone || next == kActShade);
  const uint32_t packed = __reduce_add_sync(0xffffffffu, counted ? 1u << field : 0u);
  const uint32_t cn = (packed & 63u) * (w & 255u);
  const uint32_t ct = ((packed >> 6) & 63u) * ((w >> 8) & 255u);
  const uint32_t ce = ((packed >> 12) & 63u) * ((w >> 16) & 255u);
  const uint32_t cl = ((packed >> 18) & 63u) * (w >> 24);
  uint32_t act = kActNode, best = cn;
  if (ct > best) { act = kActTri; best = ct; }
  if (cl > best) { act = kActLeave; best = cl; }
  if (ce > best) { act = kActEnter; best = ce; }
  if (shade_weight) {
    // shade_weight is relative to the default node weight 15: scaled by the
    // policy's node weight, so custom weights keep the same balance
    const uint32_t cs = ((packed >> 24) & 63u) * shade_weight * (w & 255u);
    if (cs > best * 15u) act = kActShade;
  }
  return act;
}

// Stack entries.  A visit reads only the node's a and count (its box was
// tested by the parent), so an entry carries those where it can:
//   interior node          its first child's index a (top bit clear; count 0)
//   leaf, count < 32 and   top bits 11, count in bits 25-29, a (the first
//   a < 2^25               primitive) in bits 0-24
//   other leaves           top bits 10, the node's index (then read back)
// Popping needs no memory access except for the last kind.  Trees hold fewer
// than 2^30 nodes (meshes and TLAS of fewer than 2^29 elements, checked when a
// scene is set).
constexpr uint32_t kLeafEntry = 0x80000000u, kPackedLeaf = 0x40000000u;

__device__ __forceinline__ uint32_t stack_entry(uint32_t node, float4 lo, float4 hi) {
  const uint32_t a = __float_as_uint(lo.w), c = __float_as_uint(hi.w);
  if (c == 0u) return a;
  if (c < 32u && a < (1u << 25)) return kLeafEntry | kPackedLeaf | (c << 25) | a;
  return kLeafEntry | node;
}

// Pop the current level's stack into the visited node; false when it is empty.
__device__ __forceinline__ bool trace_pop(TraceState& T, const uint32_t* st, uint32_t& sp, uint32_t stride) {
  if (sp == 0) return false;
  const uint32_t e = st[(--sp) * stride];
  if (!(e & kLeafEntry)) {
    T.na = e;
    T.ncnt = 0u;
  } else if (e & kPackedLeaf) {
    T.na = e & ((1u << 25) - 1u);
    T.ncnt = (e >> 25) & 31u;
  } else {
    const float* w = reinterpret_cast<const float*>(T.nodes + 2 * (size_t)(e & (kPackedLeaf - 1u)));
    T.na = __float_as_uint(__ldg(w + 3));
    T.ncnt = __float_as_uint(__ldg(w + 7));
  }
  return true;
}

// Perform action `act` (== T.next) of the ray; returns true when the ray is
// finished (trace_result gives the closest hit, or decides the occlusion query).
template <bool COUNT>
__device__ __forceinline__ bool trace_do(uint32_t act, TraceState& T, const DevScene& S, uint32_t* stk,
                                         uint32_t stride, const TraceCfg& cfg, Counters* ctr, WorkCount* wc) {
  uint32_t* bstk = stk + (size_t)cfg.stack_t * stride;
  const TraceCold C = trace_cold(stk, stride, cfg);
  if (act == kActTri) {
    // Up to kTrisPerStep triangles of the leaf per step, their loads issued
    // together; the tests and record updates run in the leaf's order.
    const float4* tp = T.tris + (size_t)T.na * 3;
    float4 g[kTrisPerStep][3];
#pragma unroll
    for (int k = 0; k < kTrisPerStep; ++k)
      if (k == 0 || T.ncnt > (uint32_t)k)
#pragma unroll
        for (int j = 0; j < 3; ++j) g[k][j] = __ldg(tp + 3 * k + j);
#pragma unroll
    for (int k = 0; k < kTrisPerStep; ++k) {
      if (k > 0 && T.ncnt == 0) break;
      float t, u, v;
      if (ray_triangle_v(T.o, T.d, T.rec_t, xyz(g[k][0]), xyz(g[k][1]), xyz(g[k][2]), cfg, t, u, v)) {
        T.rec_t = t;
        C.set(kLocSlot, T.na);
        C.setf(kLocU, u);
        C.setf(kLocV, v);
      }
      ++T.na;
      if (!COUNT && T.rec_t < T.t_exit) {
        T.rec_t = -3.0e38f;
        T.next = kActDone;
        return true;
      }
      --T.ncnt;
    }
    if (T.ncnt > 0) return false;
    // Leaf done: pop within the BLAS or leave it.
    T.next = trace_pop(T, bstk, T.sp, stride) ? kActNode : kActLeave;
    return false;
  }
  if (act == kActNode) {
    if (T.it >= cfg.iter_cap) {
      atomicAdd(&ctr->iter_cap_hits, 1ull);
      T.next = T.in_blas ? kActLeave : kActDone;
      return !T.in_blas;
    }
    ++T.it;
    const uint32_t na = T.na, ncount = T.ncnt;
    if (ncount == 0u) {
      // Interior node of either level: the shared slab test of both children.
      if (COUNT) { if (T.in_blas) wc->blas_interior++; else wc->tlas_interior++; }
      const float4* nodes = T.nodes;
      const float4 alo = __ldg(nodes + 2 * na), ahi = __ldg(nodes + 2 * na + 1);
      const float4 blo = __ldg(nodes + 2 * na + 2), bhi = __ldg(nodes + 2 * na + 3);
      bool hit_a, hit_b, swap;
      slab_pair(T.fast, T.o, T.d, T.rinv, T.rec_t, T.t_cull, alo, ahi, blo, bhi, hit_a, hit_b, swap);
      if (hit_a || hit_b) {
        if (hit_a && hit_b) {
          uint32_t* st = T.in_blas ? bstk : stk;
          if (T.sp < (T.in_blas ? cfg.stack_b : cfg.stack_t))
            st[(T.sp++) * stride] = swap ? stack_entry(na, alo, ahi) : stack_entry(na + 1, blo, bhi);
          else atomicAdd(&ctr->stack_overflows, 1ull);
        }
        T.na = __float_as_uint(swap ? blo.w : alo.w);
        T.ncnt = __float_as_uint(swap ? bhi.w : ahi.w);
        return false;
      }
    } else if (T.in_blas) {
      if (COUNT) wc->tri_tests += ncount;
      T.next = kActTri;
      return false;
    } else {
      C.set(kLeafNext, na);
      C.set(kLeafLeft, ncount);
      T.next = kActEnter;
      return false;
    }
    // Neither child hit: pop within the current level.
    if (T.in_blas) {
      if (!trace_pop(T, bstk, T.sp, stride)) T.next = kActLeave;
      return false;
    }
    if (trace_pop(T, stk, T.sp, stride)) return false;
    T.next = kActDone;
    return true;
  }
  if (act == kActEnter) {
    // The next instance of the TLAS leaf.
    const uint32_t leaf_next = C.u(kLeafNext);
    const uint32_t inst = __ldg(S.instance_indices + leaf_next);
    C.set(kLeafNext, leaf_next + 1);
    C.set(kLeafLeft, C.u(kLeafLeft) - 1);
    C.set(kInst, inst);
    if (COUNT) wc->blas_entries++;
    const float4* ip = S.instances + (size_t)inst * 10;
    const M4 w2o = load_m4(ip + 4);
    const float4 offs = __ldg(ip + 8);
    const float3 wo = C.f3(kWoX), wd = C.f3(kWdX);
    T.o = transform_position(w2o, wo);
    const float3 dw = transform_direction(w2o, wd);
    const float d_len = length(dw);
    T.d = divs(dw, d_len);
    T.rinv = v3(1.0f / T.d.x, 1.0f / T.d.y, 1.0f / T.d.z);
    T.t_cull = 3.0e38f;
    const float limit = C.f(kLimit);
    const float lim = fminf(T.rec_t, limit);
    // the TLAS level waits in the cold words
    C.setf(kRecT, T.rec_t);
    C.set(kSpT, T.sp);
    C.set(kItT, T.it);
    C.set(kFastT, T.fast ? 1u : 0u);
    if (!COUNT && lim < 1e29f) {
      const float om = 1.0f + max_abs3(wo);
      const float scale = d_len / length(wd);
      const float tc = (lim * cfg.cull_margin + 1e-3f * om) * scale;
      if (tc == tc && tc > 0.0f) T.t_cull = tc;
      const float te = (limit * 0.9999f - 1e-3f * om) * scale;
      if (limit < 1e29f && te < 3.0e38f) T.t_exit = te;  // NaN and inf bounds stay off
    }
    T.rec_t = 1e30f;  // fresh local record (slot, u, v 0)
    C.set(kLocSlot, 0u);
    C.setf(kLocU, 0.0f);
    C.setf(kLocV, 0.0f);
    T.nodes = S.blas_nodes + (size_t)__float_as_uint(offs.w) * 2;
    T.tris = S.tri_bvh + (size_t)__float_as_uint(offs.z) * 3;
    const float4 rlo = __ldg(T.nodes), rhi = __ldg(T.nodes + 1);
    T.na = __float_as_uint(rlo.w);
    T.ncnt = __float_as_uint(rhi.w);
    T.fast = S.fast_slabs && slab_guard(T.o, T.rinv, rlo, rhi);
    T.sp = 0;
    T.it = 0;
    T.in_blas = true;
    T.next = kActNode;
    return false;
  }
  // kActLeave: end of traverse_blas -- back to a world distance, then the next
  // instance of the TLAS leaf or a TLAS pop.
  T.in_blas = false;
  const float3 wo = C.f3(kWoX);
  const float loc_t = T.rec_t;
  T.rec_t = C.f(kRecT);
  T.sp = C.u(kSpT);
  T.it = C.u(kItT);
  T.fast = C.u(kFastT) != 0u;
  if (cfg.quirks || loc_t != 1e30f) {
    const uint32_t inst = C.u(kInst);
    const M4 o2w = load_m4(S.instances + (size_t)inst * 10);
    const float3 hit_world = transform_position(o2w, add(T.o, muls(T.d, loc_t)));
    const float new_t = length(sub(hit_world, wo));
    if (new_t < T.rec_t) {
      // the local record: its instance is the BLAS's when it holds a hit, 0 when fresh
      T.rec_t = new_t;
      C.set(kRecInst, loc_t != 1e30f ? inst : 0u);
      C.set(kRecSlot, C.u(kLocSlot));
      C.setf(kRecU, C.f(kLocU));
      C.setf(kRecV, C.f(kLocV));
    }
  }
  T.o = wo;
  T.d = C.f3(kWdX);
  T.rinv = C.f3(kWiX);
  T.t_exit = -1.0f;
  T.t_cull = COUNT ? 3.0e38f : world_cull(C.f(kLimit), wo);
  T.nodes = S.tlas_nodes;
  if (C.u(kLeafLeft) > 0) {
    T.next = kActEnter;
    return false;
  }
  if (trace_pop(T, stk, T.sp, stride)) {
    T.next = kActNode;
    return false;
  }
  T.next = kActDone;
  return true;
}

// One lane's next action; returns true when the ray is finished.
template <bool COUNT>
__device__ __forceinline__ bool trace_step(TraceState& T, const DevScene& S, uint32_t* stk, uint32_t stride,
                                           const TraceCfg& cfg, Counters* ctr, WorkCount* wc) {
  return trace_do<COUNT>(T.next, T, S, stk, stride, cfg, ctr, wc);
}

// A whole ray on one lane (no warp cooperation).  limit < 1e29 makes it an
// occlusion query outside the counting instantiation.
template <bool COUNT = false>
__device__ __forceinline__ void trace_closest(const DevScene& S, float3 wo, float3 wd, Hit& rec, uint32_t* stk,
                                              uint32_t stride, const TraceCfg& cfg, Counters* ctr,
                                              WorkCount* wc = nullptr, float limit = 3.0e38f) {
  if (COUNT) wc->rays++;
  TraceState T;
  const TraceCold C = trace_cold(stk, stride, cfg);
  if (!trace_init<!COUNT>(T, C, S, wo, wd, occ_limit(cfg, limit)))
    while (!trace_step<COUNT>(T, S, stk, stride, cfg, ctr, wc)) {
    }
  rec = trace_result(T, C);
}

}  // namespace pt
