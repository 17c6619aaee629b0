// pt_path.cuh -- per-sample path logic on the device (shading, sampling, NEE).
//
// Restates, with the reference's arithmetic order:
//   primary ray           src/path_tracer/path_tracer.wgsl:63-75
//   path_trace loop       src/path_tracer/path_tracer.wgsl:81-114          (nee_mode 0)
//   diffuse NEE estimator src/path_tracer/path_tracer.wgsl:127-192,
//                         src/pulse/gi.wgsl:56-135, :138-196                (nee_mode 1)
//   importance_sample_ggx_d, fresnel, D_GGX, G_smith, orthonormal basis
//                         src/utilities.wgsl:719-739, :767-872
//   sample_cosine_hemisphere src/utilities.wgsl:468-476
//   sample_direct_light   src/utilities.wgsl:500-558
//   CDF search            src/utilities.wgsl:659-691 (as upper_bound; the
//                         reference's loop walks down from the right and returns
//                         the same index on a non-decreasing CDF)
//   sample_triangle_uniformly src/utilities.wgsl:695-703
// nee_mode 2 is the corrected estimator (no reference counterpart): NEE with the
// world-space area pdf and the |x - y|^2 geometry term, MIS (power heuristic)
// against BSDF sampling, the cosine factor on the specular lobe, RR clamped to 1.
//
// The path is a small state machine so the megakernel and the wavefront run
// the same arithmetic: begin -> {trace, on_hit -> [shadow trace, on_shadow]}*.
#pragma once
#include "pt_trace.cuh"

namespace pt {

constexpr float kPI = 3.14159265358f;
constexpr float kTWO_PI = 6.28318530718f;
constexpr float kINV_PI = 0.31830988618f;

struct PathCfg {
  uint32_t max_depth, spp, nee_mode, light_pick, seed, wf_segments;
  float eps_origin, eps_shadow;
  bool quirks;
  bool no_rr;  // Russian roulette off: its random number is still drawn, nothing is terminated or reweighted
};

struct Material { float3 base, emissive; float rough, refl, metal; };

__device__ __forceinline__ Material load_material(const DevScene& S, uint32_t i) {
  const float4* m = S.materials + (size_t)i * 3;
  const float4 a = __ldg(m), b = __ldg(m + 1), c = __ldg(m + 2);
  return Material{xyz(a), xyz(b), c.x, c.y, c.z};
}

__device__ __forceinline__ float3 material_f0(const Material& m) {
  const float s = 0.16f * m.refl * m.refl;
  const float om = 1.0f - m.metal;
  return v3(s * om + m.base.x * m.metal, s * om + m.base.y * m.metal, s * om + m.base.z * m.metal);
}
__device__ __forceinline__ float3 fresnel(float c, float3 f0, bool quirks) {
  const float p5 = pow5(1.0f - c, quirks);
  return v3(f0.x + (1.0f - f0.x) * p5, f0.y + (1.0f - f0.y) * p5, f0.z + (1.0f - f0.z) * p5);
}
__device__ __forceinline__ float D_GGX(float NdotM, float rough) {
  const float a = rough * rough;
  const float a2 = a * a;
  const float n2 = NdotM * NdotM;
  const float b = n2 * (a2 - 1.0f) + 1.0f;
  return a2 * kINV_PI / (b * b);
}
__device__ __forceinline__ float G1(float NdotO, float rough) {
  const float a = rough * rough;
  const float k = a / 2.0f;
  return NdotO / (NdotO * (1.0f - k) + k);
}
__device__ __forceinline__ float G_smith(float NdotO, float NdotI, float rough) {
  return G1(NdotI, rough) * G1(NdotO, rough);
}

__device__ __forceinline__ float3 sample_cosine_hemisphere(float3 n, float e0, float e1) {
  const float cos_theta = 2.0f * e0 - 1.0f;
  const float phi = 2.0f * kPI * e1;
  const float sin_theta = sqrtf(lmax(1.0f - cos_theta * cos_theta, 0.0f));
  float sp, cp;
  sincos_fixed(phi, &sp, &cp);
  const float3 unit = normalize(v3(sin_theta * cp, cos_theta, sin_theta * sp));
  return normalize(add(n, unit));
}

__device__ __forceinline__ void onb(float3 n, float3& e1, float3& e3) {
  if (!(length(sub(n, v3(1.0f, 0.0f, 0.0f))) < 0.001f)) e3 = normalize(cross(n, v3(1.0f, 0.0f, 0.0f)));
  else e3 = normalize(cross(n, v3(0.0f, 1.0f, 0.0f)));
  e1 = normalize(cross(n, e3));
}

// GGX half vector; sin(acos x), cos(acos x) by the identities sqrt(1-x^2), x.
__device__ __forceinline__ float3 ggx_half(float3 n, float rough, float e1, float e2) {
  const float a = rough * rough;
  const float a2 = a * a;
  const float x = sqrtf((1.0f - e1) / (e1 * (a2 - 1.0f) + 1.0f));
  const float cos_t = x;
  const float sin_t = sqrtf(1.0f - x * x);
  const float phi = e2 * kTWO_PI;
  float sp, cp;
  sincos_fixed(phi, &sp, &cp);
  float3 b1, b3;
  onb(n, b1, b3);
  const float3 A = muls(muls(b1, sin_t), sp);
  const float3 B = muls(n, cos_t);
  const float3 C = muls(muls(b3, sin_t), cp);
  return add(A, add(B, C));
}
__device__ __forceinline__ float3 reflect(float3 a, float3 b) { return sub(muls(b, 2.0f * dot(a, b)), a); }

// importance_sample_ggx_d (src/utilities.wgsl:816-872).
__device__ __forceinline__ void importance_sample(float3 n, float3 wo, const Material& m, uint32_t& rng, bool quirks,
                                                  float3& wi, float3& refl) {
  const float3 f0 = material_f0(m);
  const float NdotO = dot(n, wo);
  const float F0max = max3(fresnel(NdotO, f0, quirks));
  const float e0 = rand_f(rng), e1 = rand_f(rng), e2 = rand_f(rng);
  float3 brdf;
  float pdf_s = 0.0f, pdf_d = 0.0f;
  if (e0 <= F0max) {
    const float3 wm = ggx_half(n, m.rough, e1, e2);
    wi = reflect(wo, wm);
    const float NdotM = dot(n, wm), NdotI = dot(n, wi), OdotM = dot(wo, wm);
    const float3 F = fresnel(OdotM, f0, quirks);
    const float D = D_GGX(NdotM, m.rough);
    const float G = G_smith(NdotO, NdotI, m.rough);
    const float den = 4.0f * NdotO * NdotI;
    brdf = v3(F.x * D * G / den, F.y * D * G / den, F.z * D * G / den);
    pdf_s = D * NdotM / (4.0f * OdotM);
  } else {
    wi = sample_cosine_hemisphere(n, e1, e2);
    const float NdotI = dot(n, wi);
    brdf = v3(m.base.x * kPI * NdotI, m.base.y * kPI * NdotI, m.base.z * kPI * NdotI);
    pdf_d = kPI * NdotI;
  }
  float pdf = (1.0f - F0max) * pdf_d + F0max * pdf_s;
  if (pdf < 0.0001f) pdf = 1.0f;
  refl = v3(brdf.x / pdf, brdf.y / pdf, brdf.z / pdf);
}

// First index k in [offset, offset+count) with cdf[k] > e, clamped to count-1,
// minus offset (== the reference's right-to-left walk on a monotone CDF).
__device__ __forceinline__ uint32_t cdf_search(const float* cdf, uint32_t offset, uint32_t count, float e) {
  uint32_t lo = 0, hi = count;
  while (lo < hi) {
    const uint32_t mid = lo + ((hi - lo) >> 1);
    if (__ldg(cdf + offset + mid) <= e) lo = mid + 1; else hi = mid;
  }
  return lo < count - 1 ? lo : count - 1;
}

__device__ __forceinline__ float3 sample_triangle_uniformly(float e0, float e1, float3 p0, float3 p1, float3 p2) {
  const float3 a = sub(p1, p0), b = sub(p2, p0);
  if (e0 + e1 < 1.0f) return add(add(p0, muls(a, e0)), muls(b, e1));
  return add(add(p0, muls(a, 1.0f - e0)), muls(b, 1.0f - e1));
}

__device__ __forceinline__ void prim_vertices(const DevScene& S, uint32_t g, float3& q0, float3& q1, float3& q2) {
  const float4* p = S.primitives + (size_t)g * 3;
  q0 = xyz(__ldg(p)); q1 = xyz(__ldg(p + 1)); q2 = xyz(__ldg(p + 2));
}

__device__ __forceinline__ uint32_t pick_light(const DevScene& S, const PathCfg& c, uint32_t& rng, float& pdf) {
  if (c.light_pick == 0) {
    const uint32_t li = rand_u(rng) % S.light_count;
    pdf = 1.0f / __uint2float_rn(S.light_count);
    return li;
  }
  const float e = rand_f(rng);
  const uint32_t li = cdf_search(S.strength_cdf, 0, S.light_count, e);
  const float c1 = __ldg(S.strength_cdf + li);
  pdf = li == 0 ? c1 : c1 - __ldg(S.strength_cdf + li - 1);
  return li;
}
__device__ __forceinline__ float light_pick_prob(const DevScene& S, const PathCfg& c, uint32_t li) {
  if (c.light_pick == 0) return 1.0f / __uint2float_rn(S.light_count);
  const float c1 = __ldg(S.strength_cdf + li);
  return li == 0 ? c1 : c1 - __ldg(S.strength_cdf + li - 1);
}
__device__ __forceinline__ float tri_prob(const DevScene& S, uint32_t cdf_offset, uint32_t k) {
  const float c1 = __ldg(S.tri_cdfs + cdf_offset + k);
  return k == 0 ? c1 : c1 - __ldg(S.tri_cdfs + cdf_offset + k - 1);
}
__device__ __forceinline__ void world_tri(const DevScene& S, const float4* ip, uint32_t k, float3& ng, float& area) {
  const uint32_t g = __float_as_uint(__ldg(ip + 8).x) + k;
  float3 q0, q1, q2;
  prim_vertices(S, g, q0, q1, q2);
  const M4 ow = load_m4(ip);
  const float3 E1 = transform_direction(ow, sub(q1, q0)), E2 = transform_direction(ow, sub(q2, q0));
  const float3 cr = cross(E1, E2);
  const float len = length(cr);
  area = 0.5f * len;
  ng = divs(cr, len);
}

__device__ __forceinline__ float3 eval_g(float3 n, float3 wo, float3 wi, const Material& m) {
  const float NI = dot(n, wi), NO = dot(n, wo);
  if (!(NI > 0.0f) || !(NO > 0.0f)) return v3(0.0f, 0.0f, 0.0f);
  const float3 h = normalize(add(wo, wi));
  const float NM = dot(n, h), OM = dot(wo, h);
  const float3 F = fresnel(OM, material_f0(m), false);
  const float D = D_GGX(NM, m.rough);
  const float G = G_smith(NO, NI, m.rough);
  const float den = 4.0f * NO * NI;
  const float dg = D * G;
  const float3 spec = v3(F.x * dg / den, F.y * dg / den, F.z * dg / den);
  const float3 diff = muls(m.base, kINV_PI);
  return muls(add(diff, spec), NI);
}
__device__ __forceinline__ float mix_pdf(float3 n, float3 wo, float3 wi, const Material& m) {
  const float NI = dot(n, wi), NO = dot(n, wo);
  if (!(NI > 0.0f) || !(NO > 0.0f)) return 0.0f;
  const float F0max = max3(fresnel(NO, material_f0(m), false));
  const float3 h = normalize(add(wo, wi));
  const float NM = dot(n, h), OM = dot(wo, h);
  const float D = D_GGX(NM, m.rough);
  const float ps = OM > 0.0f ? D * NM / (4.0f * OM) : 0.0f;
  const float pd = NI * kINV_PI;
  return (1.0f - F0max) * pd + F0max * ps;
}
// Power-heuristic weight a^2 / (a^2 + b^2).  When a square overflows (a pdf
// above ~1.8e19: a light sampled or hit at a grazing angle, a GGX lobe of a
// near-mirror) the quotient of two infinities would be NaN and poison the
// path's color; the weight is then taken from the ratio b / a instead
// (1 / (1 + (b/a)^2): 1 for an infinite a, 0 for an infinite b, 1/2 when both
// are infinite).
__device__ __forceinline__ float mis2(float a, float b) {
  const float a2 = a * a, b2 = b * b;
  const float s = a2 + b2;
  if (!(s > 3.402823466e38f)) return a2 / s;
  const float r = b / a;
  return r == r ? 1.0f / (1.0f + r * r) : 0.5f;
}
// True when all three components are finite (not an infinity, not a NaN).
__device__ __forceinline__ bool finite3(float3 v) {
  return fabsf(v.x) <= 3.402823466e38f && fabsf(v.y) <= 3.402823466e38f && fabsf(v.z) <= 3.402823466e38f;
}

// ------------------------------------------------------------- path state
struct PathState {
  float3 o, d;          // current ray
  float3 thr, color;
  float prev_pdf;       // mode 2: mixture pdf of the last BSDF sample
  uint32_t rng;
  uint32_t depth;       // traced segments so far (mode 1: after the primary)
  uint32_t flags;       // bit0 alive, bit1 primary pending (mode 1)
};
enum : uint32_t { kAlive = 1u, kPrimary = 2u };

// A pending shadow test; on_shadow adds add_vis when the light is visible
// (closest hit t >= limit) and add_occ otherwise.
struct ShadowReq {
  float3 o, d;
  float limit;
  float3 add_vis, add_occ;
  bool active;
};

__device__ __forceinline__ void path_begin(PathState& ps, const PathCfg& c, const M4& ivp, float3 eye, uint32_t x,
                                           uint32_t y, uint32_t W, uint32_t H, uint32_t sample) {
  const float ux = __uint2float_rn(x) / __uint2float_rn(W);
  const float uy = __uint2float_rn(y) / __uint2float_rn(H);
  const float cx = ux * 2.0f - 1.0f;
  const float cy = uy * 2.0f - 1.0f;
  const float4 h = mul4(ivp, cx, -cy, 1.0f, 1.0f);
  const float3 tgt = v3(h.x / h.w, h.y / h.w, h.z / h.w);
  ps.o = eye;
  ps.d = normalize(sub(tgt, eye));
  ps.thr = v3(1.0f, 1.0f, 1.0f);
  ps.color = v3(0.0f, 0.0f, 0.0f);
  ps.prev_pdf = 0.0f;
  ps.rng = seed_state(y * W + x, sample, c.seed);
  ps.depth = 0;
  // path_trace's loop runs max_depth segments; the diffuse estimator traces its
  // primary segment before its loop.
  ps.flags = c.nee_mode == 1 ? (kAlive | kPrimary) : (c.max_depth > 0 ? kAlive : 0u);
}

struct ShadeGeom { float3 n, pos; uint32_t tidx; Material m; };

__device__ __forceinline__ void shade_geom(const DevScene& S, const PathState& ps, const Hit& h, ShadeGeom& g) {
  const float4* ip = S.instances + (size_t)h.inst * 10;
  const float4 offs = __ldg(ip + 8);
  const uint32_t tri_off = __float_as_uint(offs.x), idx_off = __float_as_uint(offs.z);
  const float4 m_idx = __ldg(ip + 9);
  g.tidx = __ldg(S.triangle_indices + idx_off + h.slot);
  const float4* td = S.triangle_data + (size_t)(tri_off + g.tidx) * 5;
  const float3 n0 = xyz(__ldg(td)), n1 = xyz(__ldg(td + 1)), n2 = xyz(__ldg(td + 2));
  const float w = 1.0f - (h.u + h.v);
  const float3 nrm = add(add(muls(n0, w), muls(n1, h.u)), muls(n2, h.v));
  g.n = normalize(transform_direction(load_m4(ip), nrm));
  g.pos = add(ps.o, muls(ps.d, h.t));
  g.m = load_material(S, __float_as_uint(m_idx.x));
}

// sample_direct_light (src/utilities.wgsl:500-558) up to the shadow trace;
// fills req with the two possible additions (mode 1 adds thr * direct).
__device__ __forceinline__ void nee_ref(const DevScene& S, const PathCfg& c, float3 p0, float3 n0, float3 base,
                                        float3 thr, bool primary, uint32_t& rng, ShadowReq& req) {
  const float3 zero = v3(0.0f, 0.0f, 0.0f);
  if (S.light_count == 0) {
    rand_u(rng); rand_u(rng); rand_u(rng); rand_u(rng);
    req.active = false;
    req.add_occ = primary ? zero : mul(thr, zero);
    req.add_vis = req.add_occ;
    return;
  }
  float light_pdf;
  const uint32_t li = pick_light(S, c, rng, light_pdf);
  const uint2 ldi = __ldg(S.light_indices + li);
  const float4* mi = S.instances + (size_t)ldi.y * 10;
  const float4 moffs = __ldg(mi + 8);
  const float e0 = rand_f(rng), e1 = rand_f(rng), e2 = rand_f(rng);
  const uint32_t k = cdf_search(S.tri_cdfs, ldi.x, __float_as_uint(moffs.y), e0);
  float3 q0, q1, q2;
  prim_vertices(S, __float_as_uint(moffs.x) + k, q0, q1, q2);
  const float3 pl_obj = sample_triangle_uniformly(e1, e2, q0, q1, q2);
  const float3 pl = transform_position(load_m4(mi), pl_obj);
  const float3 to_light = sub(pl, p0);
  req.o = add(p0, muls(n0, c.eps_origin));
  req.d = normalize(to_light);
  req.limit = length(sub(pl, req.o)) - c.eps_shadow;
  req.active = true;
  float3 nl = normalize(cross(sub(q1, q0), sub(q2, q0)));
  if (dot(nl, neg(req.d)) < 0.0f) nl = neg(nl);
  const float tri_pdf = 1.0f / __ldg(S.mesh_areas + li);
  const float pdf = light_pdf * tri_pdf;
  const float cr = dot(req.d, n0);
  const float ce = dot(neg(req.d), nl);
  const float3 brdf = muls(base, kINV_PI);
  const Material lm = load_material(S, __float_as_uint(__ldg(mi + 9).x));
  const float3 em = lm.emissive;
  const float3 dn = sub(n0, nl);
  const float dsq = dot(dn, dn);
  float3 dl = v3((((brdf.x * em.x) * cr) * ce / pdf) / dsq, (((brdf.y * em.y) * cr) * ce / pdf) / dsq,
                 (((brdf.z * em.z) * cr) * ce / pdf) / dsq);
  dl = vmax(dl, zero);
  if (primary) { req.add_vis = dl; req.add_occ = zero; }
  else { req.add_vis = mul(thr, dl); req.add_occ = mul(thr, zero); }
}

// One G-buffer texel (the PbrInput fields the realtime GI pass reads).
struct GTexel { float3 pos, n, base, emissive; bool valid; };

__device__ __forceinline__ GTexel load_gtexel(const float4* gb, size_t i) {
  const float4 a = gb[4 * i], b = gb[4 * i + 1], c = gb[4 * i + 2], d = gb[4 * i + 3];
  return GTexel{xyz(a), xyz(b), xyz(c), xyz(d), __float_as_uint(a.w) != 0u};
}

// Random state of the realtime GI pass's texel (src/pulse/gi.wgsl:58-59): the
// reference's seed for seed 0.
__device__ __forceinline__ uint32_t gi_seed(uint32_t pixel, uint32_t seed) {
  return pixel * 5817321u + seed * 0x9E3779B9u;
}

// The realtime GI pass's first vertex at a G-buffer texel
// (src/pulse/gi.wgsl:74-83): the cosine-sampled first bounce, then the direct
// light at the texel (a shadow request), emission plus direct light as the
// color and the base color as the throughput.  The bounces after it are
// path_on_hit<1>'s (gi.wgsl:85-122).  An invalid texel starts no path.
__device__ __forceinline__ void gi_begin(const DevScene& S, const PathCfg& c, const GTexel& g, PathState& ps,
                                         ShadowReq& req) {
  const float3 zero = v3(0.0f, 0.0f, 0.0f);
  ps.thr = v3(1.0f, 1.0f, 1.0f);
  ps.color = zero;
  ps.prev_pdf = 0.0f;
  ps.depth = 0;
  req.active = false;
  if (!g.valid) {
    ps.o = zero;
    ps.d = zero;
    ps.flags = 0;
    return;
  }
  const float a0 = rand_f(ps.rng), a1 = rand_f(ps.rng);
  ps.d = sample_cosine_hemisphere(g.n, a0, a1);
  ps.o = add(g.pos, muls(g.n, c.eps_origin));
  ps.color = g.emissive;
  nee_ref(S, c, g.pos, g.n, g.base, ps.thr, true, ps.rng, req);
  if (!req.active) ps.color = add(ps.color, req.add_occ);
  ps.thr = g.base;
  ps.flags = c.max_depth > 0 ? kAlive : 0u;
}

// What the path-replay adjoint needs of one mode-2 vertex (filled by
// path_on_hit<2, true>; every value is the forward's own).
struct VertexRec {
  float3 n, wo, thr;    // shading normal (facing wo), outgoing direction, throughput entering the vertex
  uint32_t mat;         // material of the hit
  float w_le;           // MIS weight of the emission term (0: no emission)
  bool nee;             // a shadow ray was requested
  float3 wi_l;          // NEE direction
  float sc;             // NEE weight (MIS / area pdf)
  uint32_t mat_l;       // material of the sampled light
  bool cont;            // the path continues past this vertex
  float3 wi;            // BSDF-sampled direction
  float pb, pr;         // its mixture pdf and the Russian-roulette probability
};

// Handle the closest hit of the current segment (h.t >= 1e30 is a miss).
// Returns with ps.flags & kAlive cleared when the path ends; req.active tells
// the caller to trace a shadow ray and call path_on_shadow before the next segment.
// REC (mode 2 only) also fills *vr for the adjoint.
template <int MODE, bool REC = false>
__device__ __forceinline__ void path_on_hit(const DevScene& S, const PathCfg& c, PathState& ps, const Hit& h,
                                            ShadowReq& req, VertexRec* vr = nullptr) {
  req.active = false;
  const float3 zero = v3(0.0f, 0.0f, 0.0f);
  if (MODE == 0) {
    if (h.t >= 1e30f) { ps.flags = 0; return; }
    ShadeGeom g;
    shade_geom(S, ps, h, g);
    ps.color = add(ps.color, mul(ps.thr, g.m.emissive));
    float3 wi, refl;
    importance_sample(g.n, neg(ps.d), g.m, ps.rng, c.quirks, wi, refl);
    ps.thr = mul(ps.thr, refl);
    const float p = max3(ps.thr);
    ps.depth += 1;
    const float u_rr = rand_f(ps.rng);
    if (!c.no_rr) {
      if (u_rr > p) { ps.flags = 0; return; }
      ps.thr = muls(ps.thr, 1.0f / p);
    }
    ps.d = normalize(wi);
    ps.o = add(g.pos, muls(g.n, c.eps_origin));
    if (ps.depth >= c.max_depth) ps.flags = 0;
    return;
  }
  if (MODE == 1) {
    if (ps.flags & kPrimary) {
      if (h.t >= 1e30f) { ps.flags = 0; return; }
      ShadeGeom g;
      shade_geom(S, ps, h, g);
      const float a0 = rand_f(ps.rng), a1 = rand_f(ps.rng);
      const float3 scatter = sample_cosine_hemisphere(g.n, a0, a1);
      ps.o = add(g.pos, muls(g.n, c.eps_origin));
      ps.d = scatter;
      ps.color = g.m.emissive;
      nee_ref(S, c, g.pos, g.n, g.m.base, ps.thr, true, ps.rng, req);
      if (!req.active) ps.color = add(ps.color, req.add_occ);
      ps.thr = g.m.base;
      ps.flags = kAlive;
      if (c.max_depth == 0) ps.flags = 0;
      return;
    }
    if (h.t >= 1e30f) { ps.flags = 0; return; }
    ShadeGeom g;
    shade_geom(S, ps, h, g);
    nee_ref(S, c, g.pos, g.n, g.m.base, ps.thr, false, ps.rng, req);
    if (!req.active) ps.color = add(ps.color, req.add_occ);
    ps.thr = mul(ps.thr, g.m.base);
    const float p = max3(ps.thr);
    ps.depth += 1;
    const float u_rr = rand_f(ps.rng);
    if (!c.no_rr) {
      if (u_rr > p) { ps.flags = 0; return; }
      ps.thr = muls(ps.thr, 1.0f / p);
    }
    const float b0 = rand_f(ps.rng), b1 = rand_f(ps.rng);
    ps.d = sample_cosine_hemisphere(g.n, b0, b1);
    ps.o = add(g.pos, muls(g.n, c.eps_origin));
    if (ps.depth >= c.max_depth) ps.flags = 0;
    return;
  }
  // ---- mode 2
  if (h.t >= 1e30f) { ps.flags = 0; return; }
  ShadeGeom g;
  shade_geom(S, ps, h, g);
  const float3 wo = neg(ps.d);
  if (dot(g.n, wo) < 0.0f) g.n = neg(g.n);
  if (REC) {
    vr->n = g.n;
    vr->wo = wo;
    vr->thr = ps.thr;
    vr->mat = __float_as_uint(__ldg(S.instances + (size_t)h.inst * 10 + 9).x);
    vr->w_le = 0.0f;
    vr->nee = false;
    vr->cont = false;
  }
  const float3 Le = g.m.emissive;
  if (Le.x > 0.0f || Le.y > 0.0f || Le.z > 0.0f) {
    const int32_t li = __ldg(S.inst_light + h.inst);
    float w = 1.0f;
    if (ps.depth > 0 && li >= 0) {
      const float4* ip = S.instances + (size_t)h.inst * 10;
      float3 ng; float area;
      world_tri(S, ip, g.tidx, ng, area);
      const uint2 ldi = __ldg(S.light_indices + li);
      const float pa = light_pick_prob(S, c, (uint32_t)li) * tri_prob(S, ldi.x, g.tidx) / area;
      const float ce = fabsf(dot(ng, ps.d));
      const float pl = pa * (h.t * h.t) / ce;
      w = mis2(ps.prev_pdf, pl);
    }
    ps.color = add(ps.color, muls(mul(ps.thr, Le), w));
    if (REC) vr->w_le = w;
  }
  if (S.light_count > 0) {
    float lpick;
    const uint32_t li = pick_light(S, c, ps.rng, lpick);
    const uint2 ldi = __ldg(S.light_indices + li);
    const float4* mi = S.instances + (size_t)ldi.y * 10;
    const float4 moffs = __ldg(mi + 8);
    const float e0 = rand_f(ps.rng), e1 = rand_f(ps.rng), e2 = rand_f(ps.rng);
    const uint32_t k = cdf_search(S.tri_cdfs, ldi.x, __float_as_uint(moffs.y), e0);
    float3 q0, q1, q2;
    prim_vertices(S, __float_as_uint(moffs.x) + k, q0, q1, q2);
    const float3 pl_obj = sample_triangle_uniformly(e1, e2, q0, q1, q2);
    const float3 pl = transform_position(load_m4(mi), pl_obj);
    float3 ng; float area;
    world_tri(S, mi, k, ng, area);
    const float pa = lpick * tri_prob(S, ldi.x, k) / area;
    const float3 to = sub(pl, g.pos);
    const float dist2 = dot(to, to);
    const float dist = sqrtf(dist2);
    const float3 wi = divs(to, dist);
    const float cr = dot(g.n, wi);
    const float ce = fabsf(dot(ng, wi));
    if (cr > 0.0f && ce > 0.0f && pa > 0.0f) {
      req.o = add(g.pos, muls(g.n, c.eps_origin));
      req.d = normalize(to);
      req.limit = length(sub(pl, req.o)) - c.eps_shadow;
      req.active = true;
      const float3 gv = eval_g(g.n, wo, wi, g.m);
      const float plw = pa * dist2 / ce;
      const float pb = mix_pdf(g.n, wo, wi, g.m);
      const float wl = mis2(plw, pb);
      const Material lm = load_material(S, __float_as_uint(__ldg(mi + 9).x));
      const float sc = wl / plw;
      req.add_vis = muls(mul(mul(ps.thr, gv), lm.emissive), sc);
      // A GGX lobe of roughness near zero evaluated at its peak overflows D
      // (the squared denominator underflows): the term is then inf * 0.
      if (!finite3(req.add_vis)) req.add_vis = zero;
      req.add_occ = zero;  // not added
      if (REC) {
        vr->nee = true;
        vr->wi_l = wi;
        vr->sc = sc;
        vr->mat_l = __float_as_uint(__ldg(mi + 9).x);
      }
    }
  }
  const float F0max = max3(fresnel(dot(g.n, wo), material_f0(g.m), false));
  const float e0 = rand_f(ps.rng), e1 = rand_f(ps.rng), e2 = rand_f(ps.rng);
  float3 wi;
  if (e0 <= F0max) wi = reflect(wo, ggx_half(g.n, g.m.rough, e1, e2));
  else wi = sample_cosine_hemisphere(g.n, e1, e2);
  wi = normalize(wi);
  const float3 gv = eval_g(g.n, wo, wi, g.m);
  const float pb = mix_pdf(g.n, wo, wi, g.m);
  ps.depth += 1;
  if (!(pb > 0.0f)) { ps.flags = 0; return; }
  // An overflowed GGX peak makes gv and pb infinite together; their ratio is
  // then NaN and the path ends, as it does for a zero pdf.
  const float3 wgt = divs(gv, pb);
  if (!finite3(wgt)) { ps.flags = 0; return; }
  ps.thr = mul(ps.thr, wgt);
  ps.prev_pdf = pb;
  const float pr = c.no_rr ? 1.0f : lmin(max3(ps.thr), 1.0f);
  const float u_rr = rand_f(ps.rng);
  if (!c.no_rr) {
    if (u_rr > pr) { ps.flags = 0; return; }
    ps.thr = muls(ps.thr, 1.0f / pr);
  }
  ps.d = wi;
  ps.o = add(g.pos, muls(g.n, c.eps_origin));
  if (ps.depth >= c.max_depth) ps.flags = 0;
  if (REC) {
    vr->cont = ps.flags != 0;
    vr->wi = wi;
    vr->pb = pb;
    vr->pr = pr;
  }
}

// Derivatives of eval_g (the BRDF times the cosine) with respect to the
// material's base color (per channel: d gv_c / d base_c; the other channels
// do not depend on base_c) and its perceptual roughness r (alpha = r^2):
//   gv_c = NI (base_c / pi + F_c D G / (4 NO NI)),  F_c = f0_c + (1 - f0_c) (1 - OM)^5,
//   f0_c = 0.16 refl^2 (1 - metal) + base_c metal,
//   D = a2 / (pi b^2),  b = NM^2 (a2 - 1) + 1,  a2 = r^4,
//   G = G1(NI) G1(NO),  G1(x) = x / (x (1 - k) + k),  k = r^2 / 2.
__device__ __forceinline__ void eval_g_grad(float3 n, float3 wo, float3 wi, const Material& m, float3& d_base,
                                            float3& d_rough) {
  const float NI = dot(n, wi), NO = dot(n, wo);
  d_base = v3(0.0f, 0.0f, 0.0f);
  d_rough = d_base;
  if (!(NI > 0.0f) || !(NO > 0.0f)) return;
  const float3 h = normalize(add(wo, wi));
  const float NM = dot(n, h), OM = dot(wo, h);
  const float p5 = pow5(1.0f - OM, false);
  const float3 f0 = material_f0(m);
  const float3 F = v3(f0.x + (1.0f - f0.x) * p5, f0.y + (1.0f - f0.y) * p5, f0.z + (1.0f - f0.z) * p5);
  const float r = m.rough;
  const float a = r * r, a2 = a * a, n2 = NM * NM;
  const float b = n2 * (a2 - 1.0f) + 1.0f;
  const float D = a2 * kINV_PI / (b * b);
  const float dD = (b - 2.0f * a2 * n2) * kINV_PI / (b * b * b) * (4.0f * a * r);
  const float k = a * 0.5f;
  const float qi = NI * (1.0f - k) + k, qo = NO * (1.0f - k) + k;
  const float gi = NI / qi, go = NO / qo;
  const float dgi = -NI * (1.0f - NI) / (qi * qi) * r, dgo = -NO * (1.0f - NO) / (qo * qo) * r;
  const float G = gi * go;
  const float dG = dgi * go + gi * dgo;
  const float den = 4.0f * NO * NI;
  const float sb = NI * m.metal * (1.0f - p5) * D * G / den;
  d_base = v3(NI * kINV_PI + sb, NI * kINV_PI + sb, NI * kINV_PI + sb);
  const float dr = NI * (dD * G + D * dG) / den;
  d_rough = v3(F.x * dr, F.y * dr, F.z * dr);
}

// Result of the shadow trace of req.
template <int MODE>
__device__ __forceinline__ void path_on_shadow(PathState& ps, const ShadowReq& req, float hit_t) {
  const bool occluded = hit_t < req.limit;
  if (MODE == 2) {
    if (!occluded) ps.color = add(ps.color, req.add_vis);
  } else {
    ps.color = add(ps.color, occluded ? req.add_occ : req.add_vis);
  }
}

// Running-mean accumulation, src/path_tracer/path_tracer.wgsl:116-123.
__device__ __forceinline__ float4 accumulate(float4 old, float3 color, uint32_t acc) {
  const float3 o = acc > 0 ? v3(old.x, old.y, old.z) : v3(0.0f, 0.0f, 0.0f);
  const float w = 1.0f / (__uint2float_rn(acc) + 1.0f);
  const float om = 1.0f - w;
  return make_float4(o.x * om + color.x * w, o.y * om + color.y * w, o.z * om + color.z * w, 1.0f);
}

}  // namespace pt
