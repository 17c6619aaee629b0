// pulse_oracle.cpp -- CPU restatement of rubengrim/pulse's path-tracing hot path.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
// calls this file; it is the checker that the CUDA library is compared with.
// Only tests/, __graft_entry__.smoke() and the cpu_baseline / reference arm of
// bench.py use it.
//
// Parity status: the reference (Rust + WGSL through wgpu) cannot be compiled or
// run on this machine, and the reference ships no tests or golden vectors.  This
// oracle is therefore "parity unpinned" against the reference's own outputs; it
// is pinned instead against hand-derived known answers (tests/test_oracle_kat.py)
// and hand-worked SAH splits.
//
// What it restates (file:line in the reference project):
//   * BLAS build      src/scene/blas.rs:21-161, :170-253, :296-314
//   * TLAS build      src/scene/tlas.rs:4-136, :168-263
//   * instance prep   src/scene/mod.rs:561-697, light CDFs :700-742
//   * host transforms src/utilities.rs:42-56
//   * RNG             src/utilities.wgsl:67-83
//   * traversal       src/utilities.wgsl:127-188 (TLAS), :259-326 (BLAS)
//   * slab test       src/utilities.wgsl:405-426
//   * ray/triangle    src/utilities.wgsl:430-460
//   * sampling / GGX  src/utilities.wgsl:468-476, :695-703, :719-739, :767-872
//   * NEE             src/utilities.wgsl:500-558 (== src/pulse/gi.wgsl:138-196)
//   * CDF search      src/utilities.wgsl:659-691
//   * path_trace      src/path_tracer/path_tracer.wgsl:58-124
//   * diffuse NEE est src/path_tracer/path_tracer.wgsl:127-202, src/pulse/gi.wgsl:56-135
//
// Floating-point convention (shared with the CUDA kernels, which follow the
// same order operation by operation): every expression is evaluated left to
// right as written in the reference, no fused multiply-add (built with
// -ffp-contract=off), IEEE division and square root.  WGSL leaves the
// precision of sin/cos/acos/pow implementation-defined; this restatement fixes:
//   * sin/cos of phi = 2*pi*e: Cody-Waite reduction by pi/2 (three-part split)
//     and Taylor polynomials to degree 9 / 10, evaluated with fmaf;
//   * sin(acos(x)), cos(acos(x)) -> sqrt(1 - x*x), x   (exact identities);
//   * pow(x, 5.0) -> (x*x)*(x*x)*x  (C powf semantics for a negative base).
// min/max are NaN-ignoring and order -0 below +0 (a lattice, so parallel
// reductions on the GPU give the same bits as these sequential loops).
//
// The scalar type is a template parameter: float is the parity oracle, double
// the converged-image oracle (run with quirks off).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>
#include <omp.h>

namespace {

// ---------------------------------------------------------------- scalars --
inline bool is_nan_f(float x) { return x != x; }
inline bool is_nan_f(double x) { return x != x; }

// Lattice min/max: NaN-ignoring, -0 < +0.
template <class T> inline T lmin(T a, T b) {
  if (a != a) return b;
  if (b != b) return a;
  if (a < b) return a;
  if (b < a) return b;
  return std::signbit(a) ? a : b;
}
template <class T> inline T lmax(T a, T b) {
  if (a != a) return b;
  if (b != b) return a;
  if (a > b) return a;
  if (b > a) return b;
  return std::signbit(a) ? b : a;
}

inline float u32_as_f32(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
inline uint32_t f32_as_u32(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }

// Own sin/cos for the f32 oracle (see header comment).  Coefficients are the
// Taylor coefficients of sin and cos; pi/2 is split into three floats.
const float kPio2Hi = 1.57079637050628662109375f;
const float kPio2Mid = -4.37113900018624283e-08f;
const float kPio2Lo = -1.7151245100059349e-15f;
inline void sincos_fixed(float x, float* s_out, float* c_out) {
  if (!(std::fabs(x) <= 1.0e5f)) { *s_out = NAN; *c_out = NAN; return; }
  float q = std::rint(x * 0.636619746685028076171875f);
  float r = std::fmaf(-q, kPio2Hi, x);
  r = std::fmaf(-q, kPio2Mid, r);
  r = std::fmaf(-q, kPio2Lo, r);
  float r2 = r * r;
  float ps = std::fmaf(r2, 2.75573192239858906525573592e-6f, -1.98412698412698412698e-4f);
  ps = std::fmaf(r2, ps, 8.33333333333333333333e-3f);
  ps = std::fmaf(r2, ps, -1.66666666666666666667e-1f);
  float s = std::fmaf(r * r2, ps, r);
  float pc = std::fmaf(r2, -2.75573192239858906525573592e-7f, 2.48015873015873015873e-5f);
  pc = std::fmaf(r2, pc, -1.38888888888888888889e-3f);
  pc = std::fmaf(r2, pc, 4.16666666666666666667e-2f);
  pc = std::fmaf(r2, pc, -0.5f);
  float c = std::fmaf(r2, pc, 1.0f);
  int qi = ((int)q) & 3;
  switch (qi) {
    case 0: *s_out = s; *c_out = c; break;
    case 1: *s_out = c; *c_out = -s; break;
    case 2: *s_out = -s; *c_out = -c; break;
    default: *s_out = -c; *c_out = s; break;
  }
}
inline void sincos_t(float x, float* s, float* c) { sincos_fixed(x, s, c); }
inline void sincos_t(double x, double* s, double* c) { *s = std::sin(x); *c = std::cos(x); }

template <class T> inline T pow5(T x, int quirks) {
  if (!quirks) x = lmax<T>(x, T(0));
  T x2 = x * x;
  return x2 * x2 * x;
}

// ---------------------------------------------------------------- vectors --
template <class T> struct V3 { T x, y, z; };
template <class T> inline V3<T> v3(T x, T y, T z) { return V3<T>{x, y, z}; }
template <class T> inline V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> inline V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> inline V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T> inline V3<T> operator*(V3<T> a, V3<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class T> inline V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> inline V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T> inline V3<T> operator/(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> inline V3<T> operator/(V3<T> a, V3<T> b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
template <class T> inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline V3<T> cross(V3<T> a, V3<T> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> inline T length(V3<T> a) { return std::sqrt(dot(a, a)); }
template <class T> inline V3<T> normalize(V3<T> a) { return a / length(a); }
template <class T> inline V3<T> vmin(V3<T> a, V3<T> b) { return {lmin(a.x, b.x), lmin(a.y, b.y), lmin(a.z, b.z)}; }
template <class T> inline V3<T> vmax(V3<T> a, V3<T> b) { return {lmax(a.x, b.x), lmax(a.y, b.y), lmax(a.z, b.z)}; }
template <class T> inline T comp(V3<T> a, int axis) { return axis == 0 ? a.x : (axis == 1 ? a.y : a.z); }

// Column-major 4x4 (m[c*4+r]), WGSL mat4x4f / glam Mat4 storage.
template <class T> struct M4 { T m[16]; };
template <class T> inline M4<T> load_m4(const float* p) { M4<T> r; for (int i = 0; i < 16; ++i) r.m[i] = T(p[i]); return r; }
// m * vec4(p, w): ((c0*x + c1*y) + c2*z) + c3*w per row (src/utilities.wgsl:751-759,
// glam Mat4::mul_vec4 column sum order).
template <class T> inline void mul4(const M4<T>& a, T x, T y, T z, T w, T out[4]) {
  for (int r = 0; r < 4; ++r) out[r] = a.m[0 * 4 + r] * x + a.m[1 * 4 + r] * y + a.m[2 * 4 + r] * z + a.m[3 * 4 + r] * w;
}
template <class T> inline V3<T> transform_position(const M4<T>& a, V3<T> p) {
  T h[4]; mul4(a, p.x, p.y, p.z, T(1), h);
  return {h[0] / h[3], h[1] / h[3], h[2] / h[3]};
}
template <class T> inline V3<T> transform_direction(const M4<T>& a, V3<T> p) {
  T h[4]; mul4(a, p.x, p.y, p.z, T(0), h);
  return {h[0], h[1], h[2]};
}

// 4x4 inverse by the adjugate built from 2x2 minors (the expansion given by
// D. Eberly, "The Laplace Expansion Theorem: Computing the Determinants and
// Inverses of Matrices", Geometric Tools).  glam's own evaluation order is not
// available offline, so this order is the convention both sides follow.
inline void inverse4(const float* src, float* dst) {
  // a[r][c] = src[c*4 + r]
  auto A = [&](int r, int c) { return src[c * 4 + r]; };
  float s0 = A(0, 0) * A(1, 1) - A(1, 0) * A(0, 1);
  float s1 = A(0, 0) * A(1, 2) - A(1, 0) * A(0, 2);
  float s2 = A(0, 0) * A(1, 3) - A(1, 0) * A(0, 3);
  float s3 = A(0, 1) * A(1, 2) - A(1, 1) * A(0, 2);
  float s4 = A(0, 1) * A(1, 3) - A(1, 1) * A(0, 3);
  float s5 = A(0, 2) * A(1, 3) - A(1, 2) * A(0, 3);
  float c5 = A(2, 2) * A(3, 3) - A(3, 2) * A(2, 3);
  float c4 = A(2, 1) * A(3, 3) - A(3, 1) * A(2, 3);
  float c3 = A(2, 1) * A(3, 2) - A(3, 1) * A(2, 2);
  float c2 = A(2, 0) * A(3, 3) - A(3, 0) * A(2, 3);
  float c1 = A(2, 0) * A(3, 2) - A(3, 0) * A(2, 2);
  float c0 = A(2, 0) * A(3, 1) - A(3, 0) * A(2, 1);
  float det = s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
  float id = 1.0f / det;
  float b[4][4];
  b[0][0] = (A(1, 1) * c5 - A(1, 2) * c4 + A(1, 3) * c3) * id;
  b[0][1] = (-A(0, 1) * c5 + A(0, 2) * c4 - A(0, 3) * c3) * id;
  b[0][2] = (A(3, 1) * s5 - A(3, 2) * s4 + A(3, 3) * s3) * id;
  b[0][3] = (-A(2, 1) * s5 + A(2, 2) * s4 - A(2, 3) * s3) * id;
  b[1][0] = (-A(1, 0) * c5 + A(1, 2) * c2 - A(1, 3) * c1) * id;
  b[1][1] = (A(0, 0) * c5 - A(0, 2) * c2 + A(0, 3) * c1) * id;
  b[1][2] = (-A(3, 0) * s5 + A(3, 2) * s2 - A(3, 3) * s1) * id;
  b[1][3] = (A(2, 0) * s5 - A(2, 2) * s2 + A(2, 3) * s1) * id;
  b[2][0] = (A(1, 0) * c4 - A(1, 1) * c2 + A(1, 3) * c0) * id;
  b[2][1] = (-A(0, 0) * c4 + A(0, 1) * c2 - A(0, 3) * c0) * id;
  b[2][2] = (A(3, 0) * s4 - A(3, 1) * s2 + A(3, 3) * s0) * id;
  b[2][3] = (-A(2, 0) * s4 + A(2, 1) * s2 - A(2, 3) * s0) * id;
  b[3][0] = (-A(1, 0) * c3 + A(1, 1) * c1 - A(1, 2) * c0) * id;
  b[3][1] = (A(0, 0) * c3 - A(0, 1) * c1 + A(0, 2) * c0) * id;
  b[3][2] = (-A(3, 0) * s3 + A(3, 1) * s1 - A(3, 2) * s0) * id;
  b[3][3] = (A(2, 0) * s3 - A(2, 1) * s1 + A(2, 2) * s0) * id;
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) dst[c * 4 + r] = b[r][c];
}

// ------------------------------------------------------------- BVH build --
// src/scene/blas.rs:21-42 -- AABB::default() is the ZERO box (0,0,0)-(0,0,0).
struct Aabb {
  V3<float> mn{0.f, 0.f, 0.f}, mx{0.f, 0.f, 0.f};
  void grow(V3<float> p) { mn = vmin(mn, p); mx = vmax(mx, p); }
  void grow(const Aabb& b) { grow(b.mn); grow(b.mx); }
  float area() const { V3<float> e = mx - mn; return e.x * e.y + e.y * e.z + e.z * e.x; }
};

const float kF32Max = 3.40282346638528859812e+38f;

struct Node { V3<float> mn, mx; uint32_t a, count; };

inline void store_node(const Node& n, uint32_t* out) {
  out[0] = f32_as_u32(n.mn.x); out[1] = f32_as_u32(n.mn.y); out[2] = f32_as_u32(n.mn.z); out[3] = n.a;
  out[4] = f32_as_u32(n.mx.x); out[5] = f32_as_u32(n.mx.y); out[6] = f32_as_u32(n.mx.z); out[7] = n.count;
}

// Rust `f32 as usize` saturates: NaN and negatives give 0.
inline uint32_t bin_index(float v, uint32_t bins) {
  if (!(v > 0.0f)) return 0;
  if (v >= (float)(bins - 1)) return bins - 1;
  uint32_t i = (uint32_t)v;
  return i < bins - 1 ? i : bins - 1;
}

// Generic restatement over "primitives" given by the three accessors the two
// reference builders use:
//   BLAS: centroid = AABB centre of the triangle, bin growth by the 3 vertices,
//         node AABB from the 3 vertices (blas.rs:47-63, :196-206, :296-314);
//   TLAS: centroid = instance `center`, bin growth by bounds_min and bounds_max,
//         node AABB min from bounds_min and max from bounds_max (tlas.rs:165-263).
struct BuildInput {
  int tlas;                   // 0 BLAS, 1 TLAS
  const float* prims;         // BLAS: n x 12 (std430 p0@0, p1@4, p2@8)
  const float* inst_bounds;   // TLAS: n x 9 (bounds_min, bounds_max, center)
  std::vector<V3<float>> centroids;
};

inline V3<float> prim_vertex(const BuildInput& in, uint32_t i, int k) {
  const float* p = in.prims + (size_t)i * 12 + k * 4;
  return {p[0], p[1], p[2]};
}
inline V3<float> inst_vec(const BuildInput& in, uint32_t i, int k) {
  const float* p = in.inst_bounds + (size_t)i * 9 + k * 3;
  return {p[0], p[1], p[2]};
}

void node_aabb(const BuildInput& in, Node& node, const std::vector<uint32_t>& idx) {
  node.mn = {kF32Max, kF32Max, kF32Max};
  node.mx = {-kF32Max, -kF32Max, -kF32Max};
  for (uint32_t i = 0; i < node.count; ++i) {
    uint32_t t = idx[node.a + i];
    if (!in.tlas) {
      for (int k = 0; k < 3; ++k) node.mn = vmin(node.mn, prim_vertex(in, t, k));
      for (int k = 0; k < 3; ++k) node.mx = vmax(node.mx, prim_vertex(in, t, k));
    } else {
      node.mn = vmin(node.mn, inst_vec(in, t, 0));
      node.mx = vmax(node.mx, inst_vec(in, t, 1));
    }
  }
}

struct Split { int axis; float pos; float cost; };

Split best_split(const BuildInput& in, const Node& node, const std::vector<uint32_t>& idx, uint32_t bins) {
  Split s{0, 0.0f, 1e30f};
  std::vector<Aabb> bb(bins);
  std::vector<uint32_t> bc(bins);
  std::vector<float> area_a(bins - 1), area_b(bins - 1);
  std::vector<uint32_t> count_a(bins - 1), count_b(bins - 1);
  for (int axis = 0; axis < 3; ++axis) {
    float bmin = 1e30f, bmax = -1e30f;
    for (uint32_t i = 0; i < node.count; ++i) {
      float c = comp(in.centroids[idx[node.a + i]], axis);
      bmin = lmin(bmin, c);
      bmax = lmax(bmax, c);
    }
    if (bmin == bmax) continue;
    std::fill(bb.begin(), bb.end(), Aabb());
    std::fill(bc.begin(), bc.end(), 0u);
    float inv = (float)bins / (bmax - bmin);
    for (uint32_t i = 0; i < node.count; ++i) {
      uint32_t t = idx[node.a + i];
      uint32_t b = bin_index((comp(in.centroids[t], axis) - bmin) * inv, bins);
      bc[b] += 1;
      if (!in.tlas) {
        for (int k = 0; k < 3; ++k) bb[b].grow(prim_vertex(in, t, k));
      } else {
        bb[b].grow(inst_vec(in, t, 0));
        bb[b].grow(inst_vec(in, t, 1));
      }
    }
    Aabb box_a, box_b;
    uint32_t sum_a = 0, sum_b = 0;
    for (uint32_t i = 0; i < bins - 1; ++i) {
      sum_a += bc[i];
      count_a[i] = sum_a;
      box_a.grow(bb[i]);
      area_a[i] = box_a.area();
      sum_b += bc[bins - 1 - i];
      count_b[bins - 2 - i] = sum_b;
      box_b.grow(bb[bins - 1 - i]);
      area_b[bins - 2 - i] = box_b.area();
    }
    float bin_size = (bmax - bmin) / (float)bins;
    for (uint32_t i = 0; i < bins - 1; ++i) {
      float cost = (float)count_a[i] * area_a[i] + (float)count_b[i] * area_b[i];
      if (cost < s.cost) {
        s.axis = axis;
        s.pos = bmin + bin_size * (float)(i + 1);
        s.cost = cost;
      }
    }
  }
  return s;
}

// Returns 0, or -7 when the reference's partition loop would underflow `j`
// (a panic in the Rust reference, blas.rs:114-121).
int build_bvh(BuildInput& in, uint32_t n, uint32_t bins, uint32_t max_leaf,
              std::vector<Node>& nodes, std::vector<uint32_t>& idx) {
  idx.resize(n);
  for (uint32_t i = 0; i < n; ++i) idx[i] = i;
  nodes.clear();
  Node root{{0, 0, 0}, {0, 0, 0}, 0, n};
  node_aabb(in, root, idx);
  nodes.push_back(root);
  // Explicit DFS stack in the recursion's order: a node, then its A subtree,
  // then its B subtree (blas.rs:147-160).
  std::vector<uint32_t> stack{0};
  while (!stack.empty()) {
    uint32_t ni = stack.back();
    stack.pop_back();
    if (nodes[ni].count <= max_leaf) continue;
    Split sp = best_split(in, nodes[ni], idx, bins);
    uint32_t i = nodes[ni].a;
    uint32_t j = i + nodes[ni].count - 1;
    while (i <= j) {
      if (comp(in.centroids[idx[i]], sp.axis) < sp.pos) {
        i += 1;
      } else {
        std::swap(idx[i], idx[j]);
        if (j == 0) return -7;
        j -= 1;
      }
    }
    uint32_t a_count = i - nodes[ni].a;
    if (a_count == 0 || a_count == nodes[ni].count) continue;
    Node ca{{0, 0, 0}, {0, 0, 0}, nodes[ni].a, a_count};
    node_aabb(in, ca, idx);
    uint32_t ca_index = (uint32_t)nodes.size();
    nodes.push_back(ca);
    Node cb{{0, 0, 0}, {0, 0, 0}, i, nodes[ni].count - a_count};
    node_aabb(in, cb, idx);
    nodes.push_back(cb);
    nodes[ni].a = ca_index;
    nodes[ni].count = 0;
    stack.push_back(ca_index + 1);
    stack.push_back(ca_index);
  }
  return 0;
}

// --------------------------------------------------------------- scene view --
struct Scene {
  uint32_t instance_count, light_count;
  const float* primitives;        // 12 f32 / tri
  const float* triangle_data;     // 20 f32 / tri
  const uint32_t* triangle_indices;
  const uint32_t* blas_nodes;     // 8 u32 / node
  const uint32_t* tlas_nodes;     // 8 u32 / node
  const uint32_t* instance_indices;
  const uint32_t* instances;      // 40 u32 / instance
  const float* materials;         // 12 f32 / material
  const float* light_emission_strength_cdf;
  const float* light_triangle_area_cdfs;
  const float* light_mesh_areas;
  const uint32_t* light_indices;  // 2 u32 / light
};

struct Inst {
  const uint32_t* w;
  const float* object_world() const { return reinterpret_cast<const float*>(w); }
  const float* world_object() const { return reinterpret_cast<const float*>(w + 16); }
  uint32_t triangle_offset() const { return w[32]; }
  uint32_t triangle_count() const { return w[33]; }
  uint32_t index_offset() const { return w[34]; }
  uint32_t node_offset() const { return w[35]; }
  uint32_t material_index() const { return w[36]; }
};
inline Inst inst_at(const Scene& s, uint32_t i) { return Inst{s.instances + (size_t)i * 40}; }

struct Params {
  uint32_t max_depth, spp, nee_mode, light_pick, seed, quirks, stack_depth, iter_cap;
  float eps_origin, eps_tri, eps_par, eps_shadow;
  uint32_t kernel, block_size, min_blocks, wf_segments, trace_blocks, step_policy, no_roulette;
};

struct RayCounters {
  uint64_t rays = 0, tlas_interior = 0, blas_entries = 0, blas_interior = 0, tri_tests = 0;
  uint64_t hits = 0, nee = 0, cdf_reads = 0, iter_cap_hits = 0, stack_overflows = 0;
  void add(const RayCounters& o) {
    rays += o.rays; tlas_interior += o.tlas_interior; blas_entries += o.blas_entries;
    blas_interior += o.blas_interior; tri_tests += o.tri_tests; hits += o.hits; nee += o.nee;
    cdf_reads += o.cdf_reads; iter_cap_hits += o.iter_cap_hits; stack_overflows += o.stack_overflows;
  }
};

template <class T> struct Record { T t; uint32_t instance_index, triangle_index; T u, v; };
template <class T> struct Ray { V3<T> origin, dir; Record<T> rec; };
template <class T> inline Record<T> fresh_record() { return Record<T>{T(1e30f), 0u, 0u, T(0), T(0)}; }

template <class T> inline V3<T> node_min(const uint32_t* nd) {
  return {T(u32_as_f32(nd[0])), T(u32_as_f32(nd[1])), T(u32_as_f32(nd[2]))};
}
template <class T> inline V3<T> node_max(const uint32_t* nd) {
  return {T(u32_as_f32(nd[4])), T(u32_as_f32(nd[5])), T(u32_as_f32(nd[6]))};
}

// src/utilities.wgsl:405-426.  fmin/fmax here: only orderings of the result
// are used, so NaN-ignoring std::fmin gives the same decisions as lmin.
template <class T> inline T ray_aabb(const Ray<T>& r, V3<T> mn, V3<T> mx) {
  T tx1 = (mn.x - r.origin.x) / r.dir.x;
  T tx2 = (mx.x - r.origin.x) / r.dir.x;
  T tmin = std::fmin(tx1, tx2);
  T tmax = std::fmax(tx1, tx2);
  T ty1 = (mn.y - r.origin.y) / r.dir.y;
  T ty2 = (mx.y - r.origin.y) / r.dir.y;
  tmin = std::fmax(tmin, std::fmin(ty1, ty2));
  tmax = std::fmin(tmax, std::fmax(ty1, ty2));
  T tz1 = (mn.z - r.origin.z) / r.dir.z;
  T tz2 = (mx.z - r.origin.z) / r.dir.z;
  tmin = std::fmax(tmin, std::fmin(tz1, tz2));
  tmax = std::fmin(tmax, std::fmax(tz1, tz2));
  if (tmax >= tmin && tmin < r.rec.t && tmax > T(0)) return tmin;
  return T(1e30f);
}

// src/utilities.wgsl:430-460.  Records the BVH slot (mesh-local), not the tri id.
template <class T> inline void ray_triangle(const Scene& s, Ray<T>& r, uint32_t slot, uint32_t inst_index,
                                           const Inst& inst, const Params& p) {
  uint32_t tri = s.triangle_indices[slot + inst.index_offset()];
  const float* pr = s.primitives + (size_t)(tri + inst.triangle_offset()) * 12;
  V3<T> p0{T(pr[0]), T(pr[1]), T(pr[2])}, p1{T(pr[4]), T(pr[5]), T(pr[6])}, p2{T(pr[8]), T(pr[9]), T(pr[10])};
  V3<T> e1 = p1 - p0;
  V3<T> e2 = p2 - p0;
  V3<T> h = cross(r.dir, e2);
  T a = dot(e1, h);
  if (std::fabs(a) < T(p.eps_par)) return;
  T f = T(1) / a;
  V3<T> sv = r.origin - p0;
  T u = f * dot(sv, h);
  if (u < T(0) || u > T(1)) return;
  V3<T> q = cross(sv, e1);
  T v = f * dot(r.dir, q);
  if (v < T(0) || u + v > T(1)) return;
  T t = f * dot(e2, q);
  if (t > T(p.eps_tri) && t < r.rec.t) {
    r.rec.t = t;
    r.rec.instance_index = inst_index;
    r.rec.triangle_index = slot;
    r.rec.u = u;
    r.rec.v = v;
  }
}

// src/utilities.wgsl:259-326.
template <class T> void traverse_blas(const Scene& s, Ray<T>& ray, uint32_t inst_index, const Params& p,
                                      RayCounters& rc, uint32_t* stack) {
  Inst inst = inst_at(s, inst_index);
  M4<T> wo = load_m4<T>(inst.world_object());
  M4<T> ow = load_m4<T>(inst.object_world());
  Ray<T> ro;
  ro.origin = transform_position(wo, ray.origin);
  ro.dir = normalize(transform_direction(wo, ray.dir));
  ro.rec = fresh_record<T>();
  rc.blas_entries++;
  const uint32_t* nodes = s.blas_nodes + (size_t)inst.node_offset() * 8;
  uint32_t node_index = 0, sp = 0, it = 0;
  bool done = false;
  while (it < p.iter_cap) {
    it++;
    const uint32_t* node = nodes + (size_t)node_index * 8;
    if (node[7] > 0) {
      for (uint32_t i = 0; i < node[7]; ++i) {
        rc.tri_tests++;
        ray_triangle(s, ro, node[3] + i, inst_index, inst, p);
      }
      if (sp == 0) { done = true; break; }
      node_index = stack[--sp];
      continue;
    }
    rc.blas_interior++;
    uint32_t ca = node[3], cb = ca + 1;
    T da = ray_aabb(ro, node_min<T>(nodes + (size_t)ca * 8), node_max<T>(nodes + (size_t)ca * 8));
    T db = ray_aabb(ro, node_min<T>(nodes + (size_t)cb * 8), node_max<T>(nodes + (size_t)cb * 8));
    if (da > db) { std::swap(da, db); std::swap(ca, cb); }
    if (da == T(1e30f)) {
      if (sp == 0) { done = true; break; }
      node_index = stack[--sp];
    } else {
      node_index = ca;
      if (db != T(1e30f)) {
        if (sp < p.stack_depth) stack[sp++] = cb; else rc.stack_overflows++;
      }
    }
  }
  if (!done) rc.iter_cap_hits++;
  if (!p.quirks && ro.rec.t == T(1e30f)) return;  // fix for the spurious far hit
  V3<T> hit_obj = ro.origin + ro.rec.t * ro.dir;
  V3<T> hit_world = transform_position(ow, hit_obj);
  T new_t = length(hit_world - ray.origin);
  if (new_t < ray.rec.t) {
    ray.rec = ro.rec;
    ray.rec.t = new_t;
  }
}

// src/utilities.wgsl:127-188.
template <class T> void traverse_tlas(const Scene& s, Ray<T>& ray, const Params& p, RayCounters& rc) {
  rc.rays++;
  const uint32_t* tl = s.tlas_nodes;
  if (tl[3] == 0 && tl[7] == 0) return;
  uint32_t stack[256];
  uint32_t bstack[256];
  uint32_t node_index = 0, sp = 0, it = 0;
  bool done = false;
  while (it < p.iter_cap) {
    it++;
    const uint32_t* node = tl + (size_t)node_index * 8;
    if (node[7] > 0) {
      for (uint32_t i = 0; i < node[7]; ++i) {
        uint32_t ii = s.instance_indices[node[3] + i];
        traverse_blas(s, ray, ii, p, rc, bstack);
      }
      if (sp == 0) { done = true; break; }
      node_index = stack[--sp];
      continue;
    }
    rc.tlas_interior++;
    uint32_t ca = node[3], cb = ca + 1;
    T da = ray_aabb(ray, node_min<T>(tl + (size_t)ca * 8), node_max<T>(tl + (size_t)ca * 8));
    T db = ray_aabb(ray, node_min<T>(tl + (size_t)cb * 8), node_max<T>(tl + (size_t)cb * 8));
    if (da > db) { std::swap(da, db); std::swap(ca, cb); }
    if (da == T(1e30f)) {
      if (sp == 0) { done = true; break; }
      node_index = stack[--sp];
    } else {
      node_index = ca;
      if (db != T(1e30f)) {
        if (sp < p.stack_depth) stack[sp++] = cb; else rc.stack_overflows++;
      }
    }
  }
  if (!done) rc.iter_cap_hits++;
}

// ------------------------------------------------------------------- RNG --
// src/utilities.wgsl:67-83 (PCG hash).
inline uint32_t rand_u(uint32_t& st) {
  st = st * 747796405u + 2891336453u;
  uint32_t word = ((st >> ((st >> 28u) + 4u)) ^ st) * 277803737u;
  return (word >> 22u) ^ word;
}
template <class T> inline T rand_f(uint32_t& st) {
  uint32_t w = rand_u(st);
  const float k = u32_as_f32(0x2f800004u);
  if (sizeof(T) == 4) return T((float)w * k);
  return T((double)w * (double)k);
}

// -------------------------------------------------------------- sampling --
const float kPI = 3.14159265358f;
const float kTWO_PI = 6.28318530718f;
const float kINV_PI = 0.31830988618f;

template <class T> inline V3<T> sample_cosine_hemisphere(V3<T> n, T e0, T e1) {
  T cos_theta = T(2) * e0 - T(1);
  T phi = T(2) * T(kPI) * e1;
  T sin_theta = std::sqrt(lmax<T>(T(1) - cos_theta * cos_theta, T(0)));
  T sp, cp;
  sincos_t(phi, &sp, &cp);
  V3<T> unit = normalize(V3<T>{sin_theta * cp, cos_theta, sin_theta * sp});
  return normalize(n + unit);
}

template <class T> inline V3<T> fresnel(T c, V3<T> f0, int quirks) {
  T p5 = pow5<T>(T(1) - c, quirks);
  return {f0.x + (T(1) - f0.x) * p5, f0.y + (T(1) - f0.y) * p5, f0.z + (T(1) - f0.z) * p5};
}
template <class T> inline T D_GGX(T NdotM, T rough) {
  T a = rough * rough;
  T a2 = a * a;
  T n2 = NdotM * NdotM;
  T b = n2 * (a2 - T(1)) + T(1);
  return a2 * T(kINV_PI) / (b * b);
}
template <class T> inline T G1(T NdotO, T rough) {
  T a = rough * rough;
  T k = a / T(2);
  return NdotO / (NdotO * (T(1) - k) + k);
}
template <class T> inline T G_smith(T NdotO, T NdotI, T rough) { return G1(NdotI, rough) * G1(NdotO, rough); }

template <class T> struct Mat {
  V3<T> base, emissive;
  T rough, refl, metal;
};
template <class T> inline Mat<T> load_mat_rows(const float* rows, uint32_t i) {
  const float* m = rows + (size_t)i * 12;
  return Mat<T>{{T(m[0]), T(m[1]), T(m[2])}, {T(m[4]), T(m[5]), T(m[6])}, T(m[8]), T(m[9]), T(m[10])};
}
template <class T> inline Mat<T> load_mat(const Scene& s, uint32_t i) { return load_mat_rows<T>(s.materials, i); }
template <class T> inline V3<T> material_f0(const Mat<T>& m) {
  T s = T(0.16f) * m.refl * m.refl;
  V3<T> f0{s, s, s};
  T om = T(1) - m.metal;
  return {f0.x * om + m.base.x * m.metal, f0.y * om + m.base.y * m.metal, f0.z * om + m.base.z * m.metal};
}
template <class T> inline T max3(V3<T> v) { return lmax(lmax(v.x, v.y), v.z); }

// src/utilities.wgsl:719-739.
template <class T> inline void onb(V3<T> n, V3<T>& e1, V3<T>& e3) {
  V3<T> x{T(1), T(0), T(0)}, y{T(0), T(1), T(0)};
  if (!(length(n - x) < T(0.001f))) e3 = normalize(cross(n, x));
  else e3 = normalize(cross(n, y));
  e1 = normalize(cross(n, e3));
}

// GGX half-vector from (e1, e2) per src/utilities.wgsl:834-842 with the
// sin/cos(acos) identities.
template <class T> inline V3<T> ggx_half(V3<T> n, T rough, T e1, T e2) {
  T a = rough * rough;
  T a2 = a * a;
  T x = std::sqrt((T(1) - e1) / (e1 * (a2 - T(1)) + T(1)));
  T cos_t = x;
  T sin_t = std::sqrt(T(1) - x * x);
  T phi = e2 * T(kTWO_PI);
  T sp, cp;
  sincos_t(phi, &sp, &cp);
  V3<T> b1, b3;
  onb(n, b1, b3);
  V3<T> A = (b1 * sin_t) * sp;
  V3<T> B = n * cos_t;
  V3<T> C = (b3 * sin_t) * cp;
  return A + (B + C);
}
template <class T> inline V3<T> reflect(V3<T> a, V3<T> b) { return (T(2) * dot(a, b)) * b - a; }

// src/utilities.wgsl:816-872 (importance_sample_ggx_d).
template <class T> inline void importance_sample(V3<T> n, V3<T> wo, const Mat<T>& m, uint32_t& rng, int quirks,
                                                 V3<T>& wi, V3<T>& refl) {
  V3<T> f0 = material_f0(m);
  T NdotO = dot(n, wo);
  V3<T> F0 = fresnel(NdotO, f0, quirks);
  T F0max = max3(F0);
  T e0 = rand_f<T>(rng), e1 = rand_f<T>(rng), e2 = rand_f<T>(rng);
  V3<T> brdf;
  T pdf_s = T(0), pdf_d = T(0);
  if (e0 <= F0max) {
    V3<T> wm = ggx_half(n, m.rough, e1, e2);
    wi = reflect(wo, wm);
    T NdotM = dot(n, wm), NdotI = dot(n, wi), OdotM = dot(wo, wm);
    V3<T> F = fresnel(OdotM, f0, quirks);
    T D = D_GGX(NdotM, m.rough);
    T G = G_smith(NdotO, NdotI, m.rough);
    T den = T(4) * NdotO * NdotI;
    brdf = V3<T>{F.x * D * G / den, F.y * D * G / den, F.z * D * G / den};
    pdf_s = D * NdotM / (T(4) * OdotM);
  } else {
    wi = sample_cosine_hemisphere(n, e1, e2);
    T NdotI = dot(n, wi);
    brdf = V3<T>{m.base.x * T(kPI) * NdotI, m.base.y * T(kPI) * NdotI, m.base.z * T(kPI) * NdotI};
    pdf_d = T(kPI) * NdotI;
  }
  T pdf = (T(1) - F0max) * pdf_d + F0max * pdf_s;
  if (pdf < T(0.0001f)) pdf = T(1);
  refl = brdf / pdf;
}

// src/utilities.wgsl:659-691: the "binary search" walks down from the right
// (mid = l + (r - l) == r); result = min(largest k with cdf[k] <= e, plus one,
// count - 1).
template <class T> inline uint32_t cdf_walk(const float* cdf, uint32_t offset, uint32_t count, T e, RayCounters& rc) {
  int64_t l = offset, r = (int64_t)offset + (int64_t)count - 1;
  while (l <= r) {
    int64_t mid = r;
    rc.cdf_reads++;
    if (T(cdf[mid]) <= e) l = mid + 1; else r = mid - 1;
  }
  uint64_t lim = (uint64_t)offset + count - 1;
  return (uint32_t)(std::min<uint64_t>((uint64_t)l, lim) - offset);
}

template <class T> inline V3<T> sample_triangle_uniformly(T e0, T e1, V3<T> p0, V3<T> p1, V3<T> p2) {
  V3<T> a = p1 - p0, b = p2 - p0;
  if (e0 + e1 < T(1)) return (p0 + e0 * a) + e1 * b;
  return (p0 + (T(1) - e0) * a) + (T(1) - e1) * b;
}

template <class T> inline V3<T> prim_v(const Scene& s, uint32_t global_tri, int k) {
  const float* pr = s.primitives + (size_t)global_tri * 12 + k * 4;
  return {T(pr[0]), T(pr[1]), T(pr[2])};
}

// Optional log of every traced ray (oracle_path_log): origin, direction and
// the closest-hit record, 11 floats per ray.
thread_local std::vector<float>* g_ray_log = nullptr;

template <class T> inline void trace(const Scene& s, Ray<T>& r, const Params& p, RayCounters& rc) {
  r.rec = fresh_record<T>();
  traverse_tlas(s, r, p, rc);
  if (g_ray_log) {
    const float row[11] = {(float)r.origin.x, (float)r.origin.y, (float)r.origin.z, (float)r.dir.x, (float)r.dir.y,
                           (float)r.dir.z, (float)r.rec.t, u32_as_f32(r.rec.instance_index),
                           u32_as_f32(r.rec.triangle_index), (float)r.rec.u, (float)r.rec.v};
    g_ray_log->insert(g_ray_log->end(), row, row + 11);
  }
}

// Light pick: uniform (reference) or by the emission-strength CDF (the
// commented-out path at src/utilities.wgsl:501, :541-545).
template <class T> inline uint32_t pick_light(const Scene& s, const Params& p, uint32_t& rng, T& pdf, RayCounters& rc) {
  if (p.light_pick == 0) {
    uint32_t li = rand_u(rng) % s.light_count;
    pdf = T(1) / T((float)s.light_count);
    return li;
  }
  T e = rand_f<T>(rng);
  uint32_t li = cdf_walk(s.light_emission_strength_cdf, 0, s.light_count, e, rc);
  T c1 = T(s.light_emission_strength_cdf[li]);
  pdf = li == 0 ? c1 : c1 - T(s.light_emission_strength_cdf[li - 1]);
  return li;
}

// src/utilities.wgsl:500-558 (reference diffuse NEE, kept with its geometry term).
template <class T> inline V3<T> sample_direct_light_ref(const Scene& s, V3<T> p0, V3<T> n0, V3<T> base, uint32_t& rng,
                                                       const Params& p, RayCounters& rc) {
  if (s.light_count == 0) {
    rand_u(rng); rand_u(rng); rand_u(rng); rand_u(rng);
    return {T(0), T(0), T(0)};
  }
  rc.nee++;
  T light_pdf;
  uint32_t li = pick_light<T>(s, p, rng, light_pdf, rc);
  const uint32_t* ldi = s.light_indices + (size_t)li * 2;
  Inst mi = inst_at(s, ldi[1]);
  T e0 = rand_f<T>(rng), e1 = rand_f<T>(rng), e2 = rand_f<T>(rng);
  uint32_t k = cdf_walk(s.light_triangle_area_cdfs, ldi[0], mi.triangle_count(), e0, rc);
  uint32_t g = mi.triangle_offset() + k;
  V3<T> q0 = prim_v<T>(s, g, 0), q1 = prim_v<T>(s, g, 1), q2 = prim_v<T>(s, g, 2);
  V3<T> pl_obj = sample_triangle_uniformly(e1, e2, q0, q1, q2);
  M4<T> ow = load_m4<T>(mi.object_world());
  V3<T> pl = transform_position(ow, pl_obj);
  V3<T> to_light = pl - p0;
  Ray<T> sh;
  sh.origin = p0 + T(p.eps_origin) * n0;
  sh.dir = normalize(to_light);
  trace(s, sh, p, rc);
  if (sh.rec.t < length(pl - sh.origin) - T(p.eps_shadow)) return {T(0), T(0), T(0)};
  V3<T> nl = normalize(cross(q1 - q0, q2 - q0));
  if (dot(nl, -sh.dir) < T(0)) nl = -nl;
  T tri_pdf = T(1) / T(s.light_mesh_areas[li]);
  T pdf = light_pdf * tri_pdf;
  T cr = dot(sh.dir, n0);
  T ce = dot(-sh.dir, nl);
  V3<T> brdf = base * T(kINV_PI);
  Mat<T> lm = load_mat<T>(s, mi.material_index());
  V3<T> em = lm.emissive;
  T dsq = dot(n0 - nl, n0 - nl);
  V3<T> d{(((brdf.x * em.x) * cr) * ce / pdf) / dsq, (((brdf.y * em.y) * cr) * ce / pdf) / dsq,
          (((brdf.z * em.z) * cr) * ce / pdf) / dsq};
  return vmax(d, V3<T>{T(0), T(0), T(0)});
}

// ------------------------------------------------ corrected estimator (mode 2)
template <class T> struct Shade { V3<T> n, pos; Mat<T> m; };

template <class T> inline V3<T> eval_g(V3<T> n, V3<T> wo, V3<T> wi, const Mat<T>& m) {
  T NI = dot(n, wi), NO = dot(n, wo);
  if (!(NI > T(0)) || !(NO > T(0))) return {T(0), T(0), T(0)};
  V3<T> h = normalize(wo + wi);
  T NM = dot(n, h), OM = dot(wo, h);
  V3<T> f0 = material_f0(m);
  V3<T> F = fresnel(OM, f0, 0);
  T D = D_GGX(NM, m.rough);
  T G = G_smith(NO, NI, m.rough);
  T den = T(4) * NO * NI;
  T dg = D * G;
  V3<T> spec{F.x * dg / den, F.y * dg / den, F.z * dg / den};
  V3<T> diff = m.base * T(kINV_PI);
  return (diff + spec) * NI;
}
template <class T> inline T mix_pdf(V3<T> n, V3<T> wo, V3<T> wi, const Mat<T>& m) {
  T NI = dot(n, wi), NO = dot(n, wo);
  if (!(NI > T(0)) || !(NO > T(0))) return T(0);
  V3<T> f0 = material_f0(m);
  T F0max = max3(fresnel(NO, f0, 0));
  V3<T> h = normalize(wo + wi);
  T NM = dot(n, h), OM = dot(wo, h);
  T D = D_GGX(NM, m.rough);
  T ps = OM > T(0) ? D * NM / (T(4) * OM) : T(0);
  T pd = NI * T(kINV_PI);
  return (T(1) - F0max) * pd + F0max * ps;
}

// Area-CDF probability of mesh-local triangle k of light li.
template <class T> inline T tri_prob(const Scene& s, uint32_t cdf_offset, uint32_t k) {
  T c1 = T(s.light_triangle_area_cdfs[cdf_offset + k]);
  return k == 0 ? c1 : c1 - T(s.light_triangle_area_cdfs[cdf_offset + k - 1]);
}
template <class T> inline T light_pick_prob(const Scene& s, const Params& p, uint32_t li) {
  if (p.light_pick == 0) return T(1) / T((float)s.light_count);
  T c1 = T(s.light_emission_strength_cdf[li]);
  return li == 0 ? c1 : c1 - T(s.light_emission_strength_cdf[li - 1]);
}
// World-space geometric normal and area of a (mesh-local) triangle of an instance.
template <class T> inline void world_tri(const Scene& s, const Inst& inst, uint32_t k, V3<T>& ng, T& area) {
  uint32_t g = inst.triangle_offset() + k;
  V3<T> q0 = prim_v<T>(s, g, 0), q1 = prim_v<T>(s, g, 1), q2 = prim_v<T>(s, g, 2);
  M4<T> ow = load_m4<T>(inst.object_world());
  V3<T> E1 = transform_direction(ow, q1 - q0), E2 = transform_direction(ow, q2 - q0);
  V3<T> cr = cross(E1, E2);
  T len = length(cr);
  area = T(0.5f) * len;
  ng = cr / len;
}

// Power-heuristic weight, with the overflow guard of the device's mis2: when
// a^2 + b^2 overflows the weight comes from the ratio b / a.
template <class T> inline bool finite3(V3<T> v) {
  return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z);
}
template <class T> inline T mis2(T a, T b) {
  T a2 = a * a, b2 = b * b;
  T s = a2 + b2;
  if (!(s > std::numeric_limits<T>::max())) return a2 / s;
  T r = b / a;
  return r == r ? T(1) / (T(1) + r * r) : T(0.5f);
}

// ---------------------------------------------------------------- shading --
template <class T> inline bool shade_hit(const Scene& s, const Ray<T>& ray, Shade<T>& sh, uint32_t& tidx) {
  Inst inst = inst_at(s, ray.rec.instance_index);
  tidx = s.triangle_indices[inst.index_offset() + ray.rec.triangle_index];
  const float* td = s.triangle_data + (size_t)(inst.triangle_offset() + tidx) * 20;
  V3<T> n0{T(td[0]), T(td[1]), T(td[2])}, n1{T(td[4]), T(td[5]), T(td[6])}, n2{T(td[8]), T(td[9]), T(td[10])};
  T w = T(1) - (ray.rec.u + ray.rec.v);
  V3<T> nrm = (w * n0 + ray.rec.u * n1) + ray.rec.v * n2;
  M4<T> ow = load_m4<T>(inst.object_world());
  sh.n = normalize(transform_direction(ow, nrm));
  sh.pos = ray.origin + ray.rec.t * ray.dir;
  sh.m = load_mat<T>(s, inst.material_index());
  return true;
}

template <class T> struct CamView { M4<T> ivp; V3<T> pos; };

template <class T> inline Ray<T> primary_ray(const CamView<T>& cv, uint32_t x, uint32_t y, uint32_t W, uint32_t H) {
  T ux = T((float)x) / T((float)W);
  T uy = T((float)y) / T((float)H);
  T cx = ux * T(2) - T(1);
  T cy = uy * T(2) - T(1);
  T h[4];
  mul4(cv.ivp, cx, -cy, T(1), T(1), h);
  V3<T> tgt{h[0] / h[3], h[1] / h[3], h[2] / h[3]};
  Ray<T> r;
  r.origin = cv.pos;
  r.dir = normalize(tgt - r.origin);
  r.rec = fresh_record<T>();
  return r;
}

// The diffuse estimator's bounces after its first vertex
// (src/path_tracer/path_tracer.wgsl:157-192 = src/pulse/gi.wgsl:85-122): NEE at
// every hit, throughput times base color, Russian roulette, cosine bounce.
template <class T> void diffuse_bounces(const Scene& s, const Params& p, Ray<T>& ray, V3<T>& color, V3<T> thr,
                                        uint32_t& rng, RayCounters& rc) {
  const T t_far = T(1e30f);
  for (uint32_t depth = 0; depth < p.max_depth; ++depth) {
    trace(s, ray, p, rc);
    if (ray.rec.t >= t_far) break;
    rc.hits++;
    Shade<T> sh; uint32_t tidx;
    shade_hit(s, ray, sh, tidx);
    V3<T> direct = sample_direct_light_ref(s, sh.pos, sh.n, sh.m.base, rng, p, rc);
    color = color + thr * direct;
    thr = thr * sh.m.base;
    T pr = max3(thr);
    const T u_rr = rand_f<T>(rng);
    if (!p.no_roulette) {
      if (u_rr > pr) break;
      thr = thr * (T(1) / pr);
    }
    T b0 = rand_f<T>(rng), b1 = rand_f<T>(rng);
    ray.dir = sample_cosine_hemisphere(sh.n, b0, b1);
    ray.origin = sh.pos + T(p.eps_origin) * sh.n;
  }
}

// One camera sample; returns radiance.  Modes:
//   0  src/path_tracer/path_tracer.wgsl:58-114 (path_trace)
//   1  the diffuse NEE estimator of path_traceBBB / gi (src/path_tracer/path_tracer.wgsl:127-192),
//      with the primary hit from a primary-ray trace instead of Bevy's G-buffer
//   2  corrected estimator: NEE with world-space pdf and |x-y|^2 geometry term,
//      MIS (power heuristic) against BSDF sampling, reference GGX/diffuse BRDF with
//      the cosine factor, RR probability clamped to 1.
// What the adjoint needs of one mode-2 vertex, recorded by radiance<float>.
struct AdjVertex {
  V3<float> n, wo;
  uint32_t mat;
  float w_le;                 // MIS weight of the emission term (0: none)
  bool nee, visible;
  V3<float> wi_l;
  float sc;
  uint32_t mat_l;
  bool cont;
  V3<float> wi;
  float pb, pr;
};

//
// eval_mats (mode 2 only, test use): a second material table whose BSDF values
// and emissions weight the path while every sampling decision -- the lobe
// choice, the GGX half vector, the mixture pdf, the MIS weights, the light pick
// and its CDFs -- still uses the scene's materials.  Central differences of
// this estimator in eval_mats are the detached-sampling derivative that the
// path-replay adjoint computes, evaluated through eval_g itself rather than
// through its derivative formulas.
template <class T> V3<T> radiance(const Scene& s, const Params& p, const CamView<T>& cv, uint32_t x, uint32_t y,
                                  uint32_t W, uint32_t H, uint32_t& rng, RayCounters& rc,
                                  const std::vector<int32_t>& inst_light, std::vector<AdjVertex>* tape = nullptr,
                                  const float* eval_mats = nullptr) {
  Ray<T> ray = primary_ray(cv, x, y, W, H);
  V3<T> thr{T(1), T(1), T(1)}, color{T(0), T(0), T(0)};
  const T t_far = T(1e30f);
  if (p.nee_mode == 0) {
    for (uint32_t depth = 0; depth < p.max_depth; ++depth) {
      trace(s, ray, p, rc);
      if (ray.rec.t >= t_far) break;
      rc.hits++;
      Shade<T> sh; uint32_t tidx;
      shade_hit(s, ray, sh, tidx);
      color = color + thr * sh.m.emissive;
      V3<T> wi, refl;
      importance_sample(sh.n, -ray.dir, sh.m, rng, (int)p.quirks, wi, refl);
      thr = thr * refl;
      T pr = max3(thr);
      const T u_rr = rand_f<T>(rng);
      if (!p.no_roulette) {
        if (u_rr > pr) break;
        thr = thr * (T(1) / pr);
      }
      ray.dir = normalize(wi);
      ray.origin = sh.pos + T(p.eps_origin) * sh.n;
      ray.rec = fresh_record<T>();
    }
    return color;
  }
  if (p.nee_mode == 1) {
    trace(s, ray, p, rc);
    if (ray.rec.t >= t_far) return color;
    rc.hits++;
    Shade<T> sh; uint32_t tidx;
    shade_hit(s, ray, sh, tidx);
    T a0 = rand_f<T>(rng), a1 = rand_f<T>(rng);
    V3<T> scatter = sample_cosine_hemisphere(sh.n, a0, a1);
    ray.origin = sh.pos + T(p.eps_origin) * sh.n;
    ray.dir = scatter;
    V3<T> direct = sample_direct_light_ref(s, sh.pos, sh.n, sh.m.base, rng, p, rc);
    color = sh.m.emissive + direct;
    diffuse_bounces(s, p, ray, color, sh.m.base, rng, rc);
    return color;
  }
  // mode 2
  T prev_pdf = T(0);
  for (uint32_t depth = 0; depth < p.max_depth; ++depth) {
    trace(s, ray, p, rc);
    if (ray.rec.t >= t_far) break;
    rc.hits++;
    Shade<T> sh; uint32_t tidx;
    shade_hit(s, ray, sh, tidx);
    V3<T> wo = -ray.dir;
    if (dot(sh.n, wo) < T(0)) sh.n = -sh.n;
    AdjVertex* av = nullptr;
    if (tape) {
      tape->push_back(AdjVertex{});
      av = &tape->back();
      av->n = {(float)sh.n.x, (float)sh.n.y, (float)sh.n.z};
      av->wo = {(float)wo.x, (float)wo.y, (float)wo.z};
      av->mat = inst_at(s, ray.rec.instance_index).material_index();
    }
    // The material that weights the path (eval_mats) and the one that samples it.
    const uint32_t mat_index = inst_at(s, ray.rec.instance_index).material_index();
    const Mat<T> me = eval_mats ? load_mat_rows<T>(eval_mats, mat_index) : sh.m;
    // Emission reached by BSDF sampling (or seen directly).
    V3<T> Le = sh.m.emissive;
    if (Le.x > T(0) || Le.y > T(0) || Le.z > T(0)) {
      Le = me.emissive;
      int32_t li = inst_light[ray.rec.instance_index];
      T w = T(1);
      if (depth > 0 && li >= 0) {
        Inst inst = inst_at(s, ray.rec.instance_index);
        V3<T> ng; T area;
        world_tri(s, inst, tidx, ng, area);
        const uint32_t* ldi = s.light_indices + (size_t)li * 2;
        T pa = light_pick_prob<T>(s, p, (uint32_t)li) * tri_prob<T>(s, ldi[0], tidx) / area;
        T ce = std::fabs(dot(ng, ray.dir));
        T pl = pa * (ray.rec.t * ray.rec.t) / ce;
        w = mis2(prev_pdf, pl);
      }
      color = color + thr * Le * w;
      if (av) av->w_le = (float)w;
    }
    // Next-event estimation.
    if (s.light_count > 0) {
      T lpick;
      uint32_t li = pick_light<T>(s, p, rng, lpick, rc);
      const uint32_t* ldi = s.light_indices + (size_t)li * 2;
      Inst mi = inst_at(s, ldi[1]);
      T e0 = rand_f<T>(rng), e1 = rand_f<T>(rng), e2 = rand_f<T>(rng);
      uint32_t k = cdf_walk(s.light_triangle_area_cdfs, ldi[0], mi.triangle_count(), e0, rc);
      uint32_t g = mi.triangle_offset() + k;
      V3<T> q0 = prim_v<T>(s, g, 0), q1 = prim_v<T>(s, g, 1), q2 = prim_v<T>(s, g, 2);
      V3<T> pl_obj = sample_triangle_uniformly(e1, e2, q0, q1, q2);
      M4<T> ow = load_m4<T>(mi.object_world());
      V3<T> pl = transform_position(ow, pl_obj);
      V3<T> ng; T area;
      world_tri(s, mi, k, ng, area);
      T pa = lpick * tri_prob<T>(s, ldi[0], k) / area;
      V3<T> to = pl - sh.pos;
      T dist2 = dot(to, to);
      T dist = std::sqrt(dist2);
      V3<T> wi = to / dist;
      T cr = dot(sh.n, wi);
      T ce = std::fabs(dot(ng, wi));
      if (cr > T(0) && ce > T(0) && pa > T(0)) {
        rc.nee++;
        Ray<T> shr;
        shr.origin = sh.pos + T(p.eps_origin) * sh.n;
        shr.dir = normalize(to);
        trace(s, shr, p, rc);
        const bool visible = !(shr.rec.t < length(pl - shr.origin) - T(p.eps_shadow));
        if (av) {
          T plw = pa * dist2 / ce;
          T pb = mix_pdf(sh.n, wo, wi, sh.m);
          av->nee = true;
          av->visible = visible;
          av->wi_l = {(float)wi.x, (float)wi.y, (float)wi.z};
          av->sc = (float)(mis2(plw, pb) / plw);
          av->mat_l = mi.material_index();
        }
        if (visible) {
          V3<T> gv = eval_g(sh.n, wo, wi, me);
          T plw = pa * dist2 / ce;
          T pb = mix_pdf(sh.n, wo, wi, sh.m);
          T wl = mis2(plw, pb);
          Mat<T> lm = eval_mats ? load_mat_rows<T>(eval_mats, mi.material_index()) : load_mat<T>(s, mi.material_index());
          T sc = wl / plw;
          const V3<T> add = ((thr * gv) * lm.emissive) * sc;
          // Device rule: a non-finite term (an overflowed GGX peak) adds nothing.
          if (finite3(add)) color = color + add;
        }
      }
    }
    // BSDF sampling.
    V3<T> f0 = material_f0(sh.m);
    T F0max = max3(fresnel(dot(sh.n, wo), f0, 0));
    T e0 = rand_f<T>(rng), e1 = rand_f<T>(rng), e2 = rand_f<T>(rng);
    V3<T> wi;
    if (e0 <= F0max) wi = reflect(wo, ggx_half(sh.n, sh.m.rough, e1, e2));
    else wi = sample_cosine_hemisphere(sh.n, e1, e2);
    wi = normalize(wi);
    V3<T> gv = eval_g(sh.n, wo, wi, me);
    T pb = mix_pdf(sh.n, wo, wi, sh.m);
    if (!(pb > T(0))) break;
    // Device rule: a non-finite sample weight (gv and pb both infinite at an
    // overflowed GGX peak) ends the path.
    const V3<T> wgt = gv / pb;
    if (!finite3(wgt)) break;
    thr = thr * wgt;
    prev_pdf = pb;
    T pr = p.no_roulette ? T(1) : lmin<T>(max3(thr), T(1));
    const T u_rr = rand_f<T>(rng);
    if (!p.no_roulette) {
      if (u_rr > pr) break;
      thr = thr * (T(1) / pr);
    }
    ray.dir = wi;
    ray.origin = sh.pos + T(p.eps_origin) * sh.n;
    if (av) {
      av->cont = depth + 1 < p.max_depth;
      av->wi = {(float)wi.x, (float)wi.y, (float)wi.z};
      av->pb = (float)pb;
      av->pr = (float)pr;
    }
  }
  return color;
}

// Derivatives of eval_g with respect to base color (per channel) and
// perceptual roughness r (alpha = r^2):
//   gv_c = NI (base_c / pi + F_c D G / (4 NO NI)),  F_c = f0_c + (1 - f0_c) (1 - OM)^5,
//   f0_c = 0.16 refl^2 (1 - metal) + base_c metal,  D = a2 / (pi b^2),
//   b = NM^2 (a2 - 1) + 1,  a2 = r^4,  G = G1(NI) G1(NO),  G1(x) = x / (x (1 - k) + k),  k = r^2 / 2.
template <class T> inline void eval_g_grad(V3<T> n, V3<T> wo, V3<T> wi, const Mat<T>& m, V3<T>& d_base,
                                           V3<T>& d_rough) {
  T NI = dot(n, wi), NO = dot(n, wo);
  d_base = {T(0), T(0), T(0)};
  d_rough = d_base;
  if (!(NI > T(0)) || !(NO > T(0))) return;
  V3<T> h = normalize(wo + wi);
  T NM = dot(n, h), OM = dot(wo, h);
  T p5 = pow5(T(1) - OM, 0);
  V3<T> f0 = material_f0(m);
  V3<T> F = fresnel(OM, f0, 0);
  T r = m.rough, a = r * r, a2 = a * a, n2 = NM * NM;
  T b = n2 * (a2 - T(1)) + T(1);
  T D = a2 / (T(kPI) * b * b);
  T dD = (b - T(2) * a2 * n2) / (T(kPI) * b * b * b) * (T(4) * a * r);
  T k = a / T(2);
  T qi = NI * (T(1) - k) + k, qo = NO * (T(1) - k) + k;
  T gi = NI / qi, go = NO / qo;
  T dgi = -NI * (T(1) - NI) / (qi * qi) * r, dgo = -NO * (T(1) - NO) / (qo * qo) * r;
  T G = gi * go, dG = dgi * go + gi * dgo;
  T den = T(4) * NO * NI;
  T sb = NI * m.metal * (T(1) - p5) * D * G / den;
  T db = NI / T(kPI) + sb;
  d_base = {db, db, db};
  T dr = NI * (dD * G + D * dG) / den;
  d_rough = {F.x * dr, F.y * dr, F.z * dr};
}

inline uint32_t seed_state(uint32_t pixel_index, uint32_t sample_index, uint32_t seed) {
  return pixel_index * 1235243u + sample_index * 5817321u + seed * 0x9E3779B9u;
}

std::vector<int32_t> instance_light_map(const Scene& s) {
  std::vector<int32_t> m(s.instance_count, -1);
  for (uint32_t l = 0; l < s.light_count; ++l) {
    uint32_t ii = s.light_indices[(size_t)l * 2 + 1];
    if (ii < s.instance_count && m[ii] < 0) m[ii] = (int32_t)l;
  }
  return m;
}

}  // namespace

extern "C" {

struct OracleScene {
  uint32_t instance_count, light_count;
  const float* primitives;
  const float* triangle_data;
  const uint32_t* triangle_indices;
  const uint32_t* blas_nodes;
  const uint32_t* tlas_nodes;
  const uint32_t* instance_indices;
  const uint32_t* instances;
  const float* materials;
  const float* light_emission_strength_cdf;
  const float* light_triangle_area_cdfs;
  const float* light_mesh_areas;
  const uint32_t* light_indices;
};

struct OracleStats {
  uint64_t rays, tlas_interior, blas_entries, blas_interior, tri_tests;
  uint64_t hits, nee, cdf_reads, iter_cap_hits, stack_overflows, paths;
};

static Scene to_scene(const OracleScene* o) {
  Scene s;
  std::memcpy(&s, o, sizeof(Scene));
  return s;
}
static void to_stats(const RayCounters& rc, uint64_t paths, OracleStats* st) {
  if (!st) return;
  st->rays = rc.rays; st->tlas_interior = rc.tlas_interior; st->blas_entries = rc.blas_entries;
  st->blas_interior = rc.blas_interior; st->tri_tests = rc.tri_tests; st->hits = rc.hits; st->nee = rc.nee;
  st->cdf_reads = rc.cdf_reads; st->iter_cap_hits = rc.iter_cap_hits; st->stack_overflows = rc.stack_overflows;
  st->paths = paths;
}

// src/scene/blas.rs:44-87.  nodes_out: (2n-1) x 8 u32; tri_indices_out: n.
int oracle_build_blas(const float* prims, uint32_t n, uint32_t bins, uint32_t max_leaf, uint32_t* nodes_out,
                      uint32_t* node_count, uint32_t* tri_indices_out) {
  if (n == 0 || bins < 2) return -1;
  BuildInput in;
  in.tlas = 0;
  in.prims = prims;
  in.inst_bounds = nullptr;
  in.centroids.resize(n);
  for (uint32_t i = 0; i < n; ++i) {
    V3<float> bmin{kF32Max, kF32Max, kF32Max}, bmax{-kF32Max, -kF32Max, -kF32Max};
    for (int k = 0; k < 3; ++k) bmin = vmin(bmin, prim_vertex(in, i, k));
    for (int k = 0; k < 3; ++k) bmax = vmax(bmax, prim_vertex(in, i, k));
    in.centroids[i] = bmin + 0.5f * (bmax - bmin);
  }
  std::vector<Node> nodes;
  std::vector<uint32_t> idx;
  int rc = build_bvh(in, n, bins, max_leaf, nodes, idx);
  if (rc) return rc;
  for (size_t i = 0; i < nodes.size(); ++i) store_node(nodes[i], nodes_out + i * 8);
  *node_count = (uint32_t)nodes.size();
  std::memcpy(tri_indices_out, idx.data(), n * 4);
  return 0;
}

// src/scene/tlas.rs:29-65.  bounds: n x 9 (bounds_min, bounds_max, center).
int oracle_build_tlas(const float* bounds, uint32_t n, uint32_t bins, uint32_t max_leaf, uint32_t* nodes_out,
                      uint32_t* node_count, uint32_t* idx_out) {
  if (n == 0) {
    Node inv{{0, 0, 0}, {0, 0, 0}, 0, 0};
    store_node(inv, nodes_out);
    *node_count = 1;
    return 0;
  }
  if (bins < 2) return -1;
  BuildInput in;
  in.tlas = 1;
  in.prims = nullptr;
  in.inst_bounds = bounds;
  in.centroids.resize(n);
  for (uint32_t i = 0; i < n; ++i) in.centroids[i] = inst_vec(in, i, 2);
  std::vector<Node> nodes;
  std::vector<uint32_t> idx;
  int rc = build_bvh(in, n, bins, max_leaf, nodes, idx);
  if (rc) return rc;
  for (size_t i = 0; i < nodes.size(); ++i) store_node(nodes[i], nodes_out + i * 8);
  *node_count = (uint32_t)nodes.size();
  std::memcpy(idx_out, idx.data(), n * 4);
  return 0;
}

void oracle_inverse4(const float* src, float* dst) { inverse4(src, dst); }

// src/scene/mod.rs:561-697 + :700-742.  Inputs per instance: object_world (16 f32),
// mesh index {triangle_offset, triangle_count, index_offset, node_offset}, material.
// Outputs (caller sized): instances_out k x 40 u32, bounds_out k x 9 f32,
// light_indices_out k x 2, strength_cdf_out k, mesh_areas_out k,
// tri_cdfs_out (sum of tri counts), counts_out[0]=light_count, [1]=cdf length.
int oracle_prepare_instances(uint32_t k, const float* object_world, const uint32_t* mesh_index,
                             const uint32_t* material_index, const float* materials, uint32_t n_materials,
                             const float* primitives, const uint32_t* blas_nodes, uint32_t* instances_out,
                             float* bounds_out, uint32_t* light_indices_out, float* strength_cdf_out,
                             float* mesh_areas_out, float* tri_cdfs_out, uint32_t* counts_out) {
  std::vector<float> strengths;
  uint32_t n_lights = 0, cdf_len = 0;
  for (uint32_t i = 0; i < k; ++i) {
    const float* M = object_world + (size_t)i * 16;
    const uint32_t* mi = mesh_index + (size_t)i * 4;
    uint32_t mat = material_index[i];
    if (mat >= n_materials) return -1;
    uint32_t* out = instances_out + (size_t)i * 40;
    std::memset(out, 0, 160);
    std::memcpy(out, M, 64);
    float inv[16];
    inverse4(M, inv);
    std::memcpy(out + 16, inv, 64);
    out[32] = mi[0]; out[33] = mi[1]; out[34] = mi[2]; out[35] = mi[3]; out[36] = mat;
    const float* m = materials + (size_t)mat * 12;
    V3<float> em{m[4], m[5], m[6]};
    if (length(em) > 0.0001f) {
      strengths.push_back(dot(em, em));
      // create_triangle_area_cdf over this mesh's primitives (object space).
      std::vector<float> areas(mi[1]);
      for (uint32_t t = 0; t < mi[1]; ++t) {
        const float* pr = primitives + (size_t)(mi[0] + t) * 12;
        V3<float> p0{pr[0], pr[1], pr[2]}, p1{pr[4], pr[5], pr[6]}, p2{pr[8], pr[9], pr[10]};
        float a = length(p1 - p0);
        float b = length(p2 - p0);
        float c = length(p2 - p1);
        float s = 0.5f * (a + b + c);
        areas[t] = std::sqrt(s * (s - a) * (s - b) * (s - c));
      }
      float total = 0.0f;
      for (float a : areas) total = total + a;
      float prev = 0.0f;
      light_indices_out[n_lights * 2 + 0] = cdf_len;
      light_indices_out[n_lights * 2 + 1] = i;
      for (uint32_t t = 0; t < mi[1]; ++t) {
        float cur = prev + areas[t] / total;
        tri_cdfs_out[cdf_len++] = cur;
        prev = cur;
      }
      mesh_areas_out[n_lights] = total;
      n_lights++;
    }
    // World bounds from the 8 transformed root-AABB corners (mod.rs:625-658).
    const uint32_t* root = blas_nodes + (size_t)mi[3] * 8;
    V3<float> bmin{u32_as_f32(root[0]), u32_as_f32(root[1]), u32_as_f32(root[2])};
    V3<float> bmax{u32_as_f32(root[4]), u32_as_f32(root[5]), u32_as_f32(root[6])};
    M4<float> mm = load_m4<float>(M);
    V3<float> corners[8] = {
        {bmin.x, bmin.y, bmin.z}, {bmax.x, bmin.y, bmin.z}, {bmin.x, bmax.y, bmin.z}, {bmin.x, bmin.y, bmax.z},
        {bmax.x, bmax.y, bmin.z}, {bmin.x, bmax.y, bmax.z}, {bmax.x, bmin.y, bmax.z}, {bmax.x, bmax.y, bmax.z}};
    V3<float> wmin{kF32Max, kF32Max, kF32Max}, wmax{-kF32Max, -kF32Max, -kF32Max};
    V3<float> tc[8];
    for (int c = 0; c < 8; ++c) tc[c] = transform_position(mm, corners[c]);
    for (int c = 0; c < 8; ++c) wmin = vmin(wmin, tc[c]);
    for (int c = 0; c < 8; ++c) wmax = vmax(wmax, tc[c]);
    V3<float> center = wmin + 0.5f * (wmax - wmin);
    float* bo = bounds_out + (size_t)i * 9;
    bo[0] = wmin.x; bo[1] = wmin.y; bo[2] = wmin.z;
    bo[3] = wmax.x; bo[4] = wmax.y; bo[5] = wmax.z;
    bo[6] = center.x; bo[7] = center.y; bo[8] = center.z;
  }
  float total = 0.0f;
  for (float s : strengths) total = total + s;
  float prev = 0.0f;
  for (size_t i = 0; i < strengths.size(); ++i) {
    float cur = prev + strengths[i] / total;
    strength_cdf_out[i] = cur;
    prev = cur;
  }
  counts_out[0] = n_lights;
  counts_out[1] = cdf_len;
  return 0;
}

// Closest-hit trace of world rays (n x 6: origin, dir).
int oracle_trace(const OracleScene* os, const float* rays, uint32_t n, const Params* p, float* t_out,
                 uint32_t* inst_out, uint32_t* tri_out, float* u_out, float* v_out, OracleStats* st, int nthreads) {
  Scene s = to_scene(os);
  RayCounters total;
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
  {
    RayCounters rc;
#pragma omp for schedule(dynamic, 256)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
      Ray<float> r;
      const float* q = rays + i * 6;
      r.origin = {q[0], q[1], q[2]};
      r.dir = {q[3], q[4], q[5]};
      trace(s, r, *p, rc);
      t_out[i] = r.rec.t; inst_out[i] = r.rec.instance_index; tri_out[i] = r.rec.triangle_index;
      u_out[i] = r.rec.u; v_out[i] = r.rec.v;
    }
#pragma omp critical
    total.add(rc);
  }
  to_stats(total, 0, st);
  return 0;
}

// One frame of the running-mean accumulation (path_tracer.wgsl:116-123) for a
// list of pixels (or all pixels if pixels == NULL).  image: W*H*4 f32, read if
// accumulation_count > 0 and written.  precision 32 or 64.
int oracle_render(const OracleScene* os, const float* inv_view_proj, const float* world_pos, uint32_t W, uint32_t H,
                  uint32_t accumulation_count, const Params* p, int precision, const uint32_t* pixels,
                  uint32_t n_pixels, float* image, OracleStats* st, int nthreads) {
  Scene s = to_scene(os);
  std::vector<int32_t> il = instance_light_map(s);
  uint64_t n = pixels ? n_pixels : (uint64_t)W * H;
  RayCounters total;
  CamView<float> cf{load_m4<float>(inv_view_proj), {world_pos[0], world_pos[1], world_pos[2]}};
  CamView<double> cd{load_m4<double>(inv_view_proj), {world_pos[0], world_pos[1], world_pos[2]}};
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
  {
    RayCounters rc;
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
      uint32_t pix = pixels ? pixels[i] : (uint32_t)i;
      uint32_t x = pix % W, y = pix / W;
      float* px = image + (size_t)pix * 4;
      for (uint32_t sidx = 0; sidx < p->spp; ++sidx) {
        uint32_t acc = accumulation_count * p->spp + sidx;
        uint32_t rng = seed_state(pix, acc, p->seed);
        V3<float> c;
        if (precision == 64) {
          V3<double> cdv = radiance<double>(s, *p, cd, x, y, W, H, rng, rc, il);
          c = {(float)cdv.x, (float)cdv.y, (float)cdv.z};
        } else {
          c = radiance<float>(s, *p, cf, x, y, W, H, rng, rc, il);
        }
        V3<float> old{0.f, 0.f, 0.f};
        if (acc > 0) old = {px[0], px[1], px[2]};
        float w = 1.0f / ((float)acc + 1.0f);
        float om = 1.0f - w;
        px[0] = old.x * om + c.x * w;
        px[1] = old.y * om + c.y * w;
        px[2] = old.z * om + c.z * w;
        px[3] = 1.0f;
      }
    }
#pragma omp critical
    total.add(rc);
  }
  to_stats(total, n * p->spp, st);
  return 0;
}

// Primary-hit G-buffer (16 floats per texel: position + valid bits, normal,
// base color, emissive): the camera ray of src/path_tracer/path_tracer.wgsl:63-75
// and the hit shading of :89-100.
int oracle_gbuffer_primary(const OracleScene* os, const float* inv_view_proj, const float* world_pos, uint32_t W,
                           uint32_t H, const Params* p, float* gbuf, int nthreads) {
  Scene s = to_scene(os);
  CamView<float> cv{load_m4<float>(inv_view_proj), {world_pos[0], world_pos[1], world_pos[2]}};
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
  {
    RayCounters rc;
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < (int64_t)W * H; ++i) {
      float* o = gbuf + (size_t)i * 16;
      std::memset(o, 0, 64);
      Ray<float> ray = primary_ray(cv, (uint32_t)(i % W), (uint32_t)(i / W), W, H);
      trace(s, ray, *p, rc);
      if (ray.rec.t >= 1e30f) continue;
      Shade<float> sh; uint32_t tidx;
      shade_hit(s, ray, sh, tidx);
      const float v[16] = {sh.pos.x, sh.pos.y, sh.pos.z, u32_as_f32(1u), sh.n.x, sh.n.y, sh.n.z, 0.f,
                           sh.m.base.x, sh.m.base.y, sh.m.base.z, 0.f, sh.m.emissive.x, sh.m.emissive.y,
                           sh.m.emissive.z, 0.f};
      std::memcpy(o, v, 64);
    }
  }
  return 0;
}

// The realtime GI pass, src/pulse/gi.wgsl:56-135, over a decoded G-buffer
// (gw x gh texels of 16 floats as above) into a W x H image: the texel
// read at gi.wgsl:61-67, the seed of :58-59, spp samples sharing one random
// state (:69-126), each a cosine bounce from the texel with the direct light
// there (:74-83) and the diffuse bounces (:85-122), the image overwritten with
// (mean, 1) (:125, :131).  A texel whose valid word is 0 gives (0, 0, 0, 1).
int oracle_render_gi(const OracleScene* os, const float* gbuf, uint32_t gw, uint32_t gh, uint32_t W, uint32_t H,
                     const Params* p, const uint32_t* pixels, uint32_t n_pixels, float* image, OracleStats* st,
                     int nthreads) {
  Scene s = to_scene(os);
  uint64_t n = pixels ? n_pixels : (uint64_t)W * H;
  RayCounters total;
  const float spp_inv = 1.0f / (float)p->spp;
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
  {
    RayCounters rc;
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
      const uint32_t pix = pixels ? pixels[i] : (uint32_t)i;
      const uint32_t x = pix % W, y = pix / W;
      float* px = image + (size_t)pix * 4;
      const float ux = (float)x / (float)W, uy = (float)y / (float)H;
      uint32_t gx = (uint32_t)(ux * (float)gw), gy = (uint32_t)(uy * (float)gh);
      gx = gx < gw ? gx : gw - 1;
      gy = gy < gh ? gy : gh - 1;
      const float* t = gbuf + ((size_t)gy * gw + gx) * 16;
      V3<float> out{0.f, 0.f, 0.f};
      if (f32_as_u32(t[3]) != 0u) {
        const V3<float> pos{t[0], t[1], t[2]}, nrm{t[4], t[5], t[6]}, base{t[8], t[9], t[10]},
            em{t[12], t[13], t[14]};
        uint32_t rng = pix * 5817321u + p->seed * 0x9E3779B9u;
        for (uint32_t k = 0; k < p->spp; ++k) {
          Ray<float> ray;
          float a0 = rand_f<float>(rng), a1 = rand_f<float>(rng);
          ray.dir = sample_cosine_hemisphere(nrm, a0, a1);
          ray.origin = pos + p->eps_origin * nrm;
          V3<float> direct = sample_direct_light_ref(s, pos, nrm, base, rng, *p, rc);
          V3<float> color = em + direct;
          diffuse_bounces(s, *p, ray, color, base, rng, rc);
          out = out + color * spp_inv;
        }
      }
      px[0] = out.x; px[1] = out.y; px[2] = out.z; px[3] = 1.0f;
    }
#pragma omp critical
    total.add(rc);
  }
  to_stats(total, n * p->spp, st);
  return 0;
}

// One FP32 sample of texel (x, y) (sample index `sample`) with every ray it
// traces -- camera, bounce and shadow rays in order -- logged as 11 floats
// (origin, direction, t, instance and triangle bits, u, v) into out, at most
// max_rays rays; *n_rays receives the count, rgb the sample's radiance.  A
// debugging aid for locating the first ray on which two tracers disagree.
int oracle_path_log(const OracleScene* os, const float* inv_view_proj, const float* world_pos, uint32_t W, uint32_t H,
                    uint32_t x, uint32_t y, uint32_t sample, const Params* p, float* out, uint32_t max_rays,
                    uint32_t* n_rays, float* rgb) {
  Scene s = to_scene(os);
  std::vector<int32_t> il = instance_light_map(s);
  CamView<float> cf{load_m4<float>(inv_view_proj), {world_pos[0], world_pos[1], world_pos[2]}};
  std::vector<float> log;
  g_ray_log = &log;
  RayCounters rc;
  uint32_t rng = seed_state(y * W + x, sample, p->seed);
  const V3<float> c = radiance<float>(s, *p, cf, x, y, W, H, rng, rc, il);
  g_ray_log = nullptr;
  const uint32_t n = (uint32_t)(log.size() / 11);
  *n_rays = n;
  std::memcpy(out, log.data(), (size_t)std::min(n, max_rays) * 11 * sizeof(float));
  rgb[0] = c.x; rgb[1] = c.y; rgb[2] = c.z;
  return 0;
}

// Mean over spp_total samples (sample indices 0..spp_total-1) of every texel,
// each path in double precision (precision 64, quirks forced off: the
// converged-image oracle) or in float (precision 32, the parity arithmetic),
// summed in double.  out: n_pixels x 3 f64 means.
// eval_mats: NULL, or (mode 2) the material table that weights the paths
// while the scene's materials sample them (see radiance).
int oracle_render_mean64(const OracleScene* os, const float* inv_view_proj, const float* world_pos, uint32_t W,
                         uint32_t H, uint32_t spp_total, const Params* p_in, const uint32_t* pixels,
                         uint32_t n_pixels, double* out, int nthreads, const float* eval_mats, int precision) {
  Scene s = to_scene(os);
  std::vector<int32_t> il = instance_light_map(s);
  Params p = *p_in;
  if (precision != 32) p.quirks = 0;
  uint64_t n = pixels ? n_pixels : (uint64_t)W * H;
  CamView<double> cd{load_m4<double>(inv_view_proj), {world_pos[0], world_pos[1], world_pos[2]}};
  CamView<float> cf{load_m4<float>(inv_view_proj), {world_pos[0], world_pos[1], world_pos[2]}};
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
  {
    RayCounters rc;
#pragma omp for schedule(dynamic, 16)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
      uint32_t pix = pixels ? pixels[i] : (uint32_t)i;
      uint32_t x = pix % W, y = pix / W;
      double sx = 0, sy = 0, sz = 0;
      for (uint32_t sidx = 0; sidx < spp_total; ++sidx) {
        uint32_t rng = seed_state(pix, sidx, p.seed);
        if (precision == 32) {
          V3<float> c = radiance<float>(s, p, cf, x, y, W, H, rng, rc, il, nullptr, eval_mats);
          sx += c.x; sy += c.y; sz += c.z;
        } else {
          V3<double> c = radiance<double>(s, p, cd, x, y, W, H, rng, rc, il, nullptr, eval_mats);
          sx += c.x; sy += c.y; sz += c.z;
        }
      }
      out[i * 3 + 0] = sx / spp_total;
      out[i * 3 + 1] = sy / spp_total;
      out[i * 3 + 2] = sz / spp_total;
    }
  }
  return 0;
}

// FP64 path-replay adjoint of the corrected estimator (mode 2): every path is
// the FP32 forward's own (recorded by radiance<float>), the gradient algebra is
// done in double with exact suffix sums (no L - prefix subtraction).  Sampling
// is detached as on the device: directions, MIS weights, pdfs and
// Russian-roulette probabilities are the forward's constants.  dimg: W*H*4 f32
// dloss/dimage of the mean of n_samples samples per texel; grads: n_mat x 8
// doubles (base rgb, emissive rgb, roughness, unused), accumulated.
int oracle_backward(const OracleScene* os, const float* inv_view_proj, const float* world_pos, uint32_t W,
                    uint32_t H, uint32_t n_samples, const Params* p, const float* dimg, uint32_t n_mat,
                    double* grads, int nthreads) {
  if (p->nee_mode != 2) return -1;
  Scene s = to_scene(os);
  std::vector<int32_t> il = instance_light_map(s);
  CamView<float> cf{load_m4<float>(inv_view_proj), {world_pos[0], world_pos[1], world_pos[2]}};
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
  {
    std::vector<double> g((size_t)n_mat * 8, 0.0);
    std::vector<AdjVertex> tape;
    std::vector<V3<double>> Tj, term;
    RayCounters rc;
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < (int64_t)W * H; ++i) {
      const uint32_t pix = (uint32_t)i, x = pix % W, y = pix / W;
      const V3<double> delta{double(dimg[4 * i]) / n_samples, double(dimg[4 * i + 1]) / n_samples,
                             double(dimg[4 * i + 2]) / n_samples};
      if (delta.x == 0 && delta.y == 0 && delta.z == 0) continue;
      for (uint32_t k = 0; k < n_samples; ++k) {
        uint32_t rng = seed_state(pix, k, p->seed);
        tape.clear();
        radiance<float>(s, *p, cf, x, y, W, H, rng, rc, il, &tape);
        const size_t nv = tape.size();
        Tj.assign(nv, V3<double>{0, 0, 0});
        term.assign(nv, V3<double>{0, 0, 0});
        V3<double> T{1, 1, 1};
        for (size_t j = 0; j < nv; ++j) {
          const AdjVertex& v = tape[j];
          const Mat<double> m = load_mat<double>(s, v.mat);
          const V3<double> n{v.n.x, v.n.y, v.n.z}, wo{v.wo.x, v.wo.y, v.wo.z};
          Tj[j] = T;
          V3<double> e{0, 0, 0};
          if (v.w_le != 0.0f) e = e + m.emissive * double(v.w_le);
          if (v.nee && v.visible) {
            const V3<double> wl{v.wi_l.x, v.wi_l.y, v.wi_l.z};
            e = e + (eval_g(n, wo, wl, m) * load_mat<double>(s, v.mat_l).emissive) * double(v.sc);
          }
          term[j] = T * e;
          if (!v.cont) break;
          const V3<double> wi{v.wi.x, v.wi.y, v.wi.z};
          T = T * (eval_g(n, wo, wi, m) / (double(v.pb) * double(v.pr)));
        }
        V3<double> rem{0, 0, 0};  // radiance of the vertices after j
        for (size_t jj = nv; jj-- > 0;) {
          const AdjVertex& v = tape[jj];
          const Mat<double> m = load_mat<double>(s, v.mat);
          const V3<double> n{v.n.x, v.n.y, v.n.z}, wo{v.wo.x, v.wo.y, v.wo.z};
          double* gm = g.data() + (size_t)v.mat * 8;
          const V3<double> Tv = Tj[jj];
          if (v.cont) {
            const V3<double> wi{v.wi.x, v.wi.y, v.wi.z};
            const V3<double> gv = eval_g(n, wo, wi, m);
            V3<double> db, dr;
            eval_g_grad(n, wo, wi, m, db, dr);
            const V3<double> coef{gv.x != 0 ? delta.x * rem.x / gv.x : 0.0, gv.y != 0 ? delta.y * rem.y / gv.y : 0.0,
                                  gv.z != 0 ? delta.z * rem.z / gv.z : 0.0};
            gm[0] += coef.x * db.x; gm[1] += coef.y * db.y; gm[2] += coef.z * db.z;
            gm[6] += coef.x * dr.x + coef.y * dr.y + coef.z * dr.z;
          }
          if (v.w_le != 0.0f) {
            gm[3] += delta.x * Tv.x * v.w_le; gm[4] += delta.y * Tv.y * v.w_le; gm[5] += delta.z * Tv.z * v.w_le;
          }
          if (v.nee && v.visible) {
            const V3<double> wl{v.wi_l.x, v.wi_l.y, v.wi_l.z};
            const V3<double> gl = eval_g(n, wo, wl, m);
            const V3<double> Le = load_mat<double>(s, v.mat_l).emissive;
            double* gl_m = g.data() + (size_t)v.mat_l * 8;
            gl_m[3] += delta.x * Tv.x * gl.x * v.sc; gl_m[4] += delta.y * Tv.y * gl.y * v.sc;
            gl_m[5] += delta.z * Tv.z * gl.z * v.sc;
            V3<double> db, dr;
            eval_g_grad(n, wo, wl, m, db, dr);
            const V3<double> coef = ((delta * Tv) * Le) * double(v.sc);
            gm[0] += coef.x * db.x; gm[1] += coef.y * db.y; gm[2] += coef.z * db.z;
            gm[6] += coef.x * dr.x + coef.y * dr.y + coef.z * dr.z;
          }
          rem = rem + term[jj];
        }
      }
    }
#pragma omp critical
    for (size_t k = 0; k < g.size(); ++k) grads[k] += g[k];
  }
  return 0;
}

// eval_g and its derivatives in double for one (n, wo, wi, material) -- the
// material as its 12-word std430 row.  out: gv rgb, d/dbase rgb, d/drough rgb.
void oracle_eval_g_grad(const double* n, const double* wo, const double* wi, const float* mat12, double* out) {
  Mat<double> m{{mat12[0], mat12[1], mat12[2]}, {mat12[4], mat12[5], mat12[6]}, mat12[8], mat12[9], mat12[10]};
  V3<double> N{n[0], n[1], n[2]}, O{wo[0], wo[1], wo[2]}, I{wi[0], wi[1], wi[2]};
  V3<double> g = eval_g(N, O, I, m), db, dr;
  eval_g_grad(N, O, I, m, db, dr);
  double v[9] = {g.x, g.y, g.z, db.x, db.y, db.z, dr.x, dr.y, dr.z};
  for (int i = 0; i < 9; ++i) out[i] = v[i];
}

// Known-answer hooks for the primitives (tests/test_oracle_kat.py).
uint32_t oracle_rand_u(uint32_t* state) { return rand_u(*state); }
float oracle_rand_f(uint32_t* state) { return rand_f<float>(*state); }
void oracle_sincos(float x, float* s, float* c) { sincos_fixed(x, s, c); }
uint32_t oracle_cdf_walk(const float* cdf, uint32_t offset, uint32_t count, float e) {
  RayCounters rc;
  return cdf_walk<float>(cdf, offset, count, e, rc);
}
float oracle_ray_aabb(const float* o, const float* d, const float* mn, const float* mx, float rec_t) {
  Ray<float> r;
  r.origin = {o[0], o[1], o[2]};
  r.dir = {d[0], d[1], d[2]};
  r.rec = fresh_record<float>();
  r.rec.t = rec_t;
  return ray_aabb(r, V3<float>{mn[0], mn[1], mn[2]}, V3<float>{mx[0], mx[1], mx[2]});
}
// Single triangle test; returns 1 on hit with t,u,v.
int oracle_ray_triangle(const float* o, const float* d, const float* tri9, float* tuv) {
  float prim[12] = {tri9[0], tri9[1], tri9[2], 0, tri9[3], tri9[4], tri9[5], 0, tri9[6], tri9[7], tri9[8], 0};
  uint32_t ti = 0;
  uint32_t inst_words[40] = {0};
  Scene s{};
  s.primitives = prim;
  s.triangle_indices = &ti;
  Params p{};
  p.eps_par = 1e-4f;
  p.eps_tri = 0.001f;
  Ray<float> r;
  r.origin = {o[0], o[1], o[2]};
  r.dir = {d[0], d[1], d[2]};
  r.rec = fresh_record<float>();
  ray_triangle(s, r, 0, 0, Inst{inst_words}, p);
  if (r.rec.t == 1e30f) return 0;
  tuv[0] = r.rec.t; tuv[1] = r.rec.u; tuv[2] = r.rec.v;
  return 1;
}
// importance_sample_ggx_d for one shading point (n, wo, material 12 f32).
void oracle_importance_sample(const float* n, const float* wo, const float* mat12, uint32_t* rng, int quirks,
                              float* wi_out, float* refl_out) {
  Scene s{};
  s.materials = mat12;
  Mat<float> m = load_mat<float>(s, 0);
  V3<float> wi, refl;
  importance_sample(V3<float>{n[0], n[1], n[2]}, V3<float>{wo[0], wo[1], wo[2]}, m, *rng, quirks, wi, refl);
  wi_out[0] = wi.x; wi_out[1] = wi.y; wi_out[2] = wi.z;
  refl_out[0] = refl.x; refl_out[1] = refl.y; refl_out[2] = refl.z;
}

}  // extern "C"
