// bvh.cu -- device binned-SAH build; see bvh.cuh for the parity argument.
//
// Two phases, one result:
//   phase 1  nodes with more than kSmall elements, level by level with
//            multi-block kernels (tiles of at least kTile elements, atomics on
//            order-preserving integer keys for min/max);
//   phase 2  each remaining subtree (<= kSmall elements) built by one block
//            in shared memory, a warp per node of a level, node records in
//            the reference's depth-first, subtree-local numbering;
// then the host assigns final indices from subtree sizes and one kernel
// writes every record to its place.
#include "bvh.cuh"

#include <algorithm>
#include <atomic>
#include <array>
#include <cfloat>
#include <cstring>
#include <vector>

#include "dev_alloc.h"
#include "pt_math.cuh"

namespace bvh {

using pt::lmax;
using pt::lmin;

namespace {

constexpr uint32_t kSmall = 512;  // subtree size handed to one block (k_subtree_block)
constexpr uint32_t kTile = 1024;   // fewest elements per block in phase 1
constexpr uint64_t kTilesPerLevel = 1184;  // phase-1 blocks per level: 8 per SM of a B200
constexpr int kMaxBins = 32;

// Order-preserving key of a (non-NaN) float: -0 below +0.
__device__ __forceinline__ uint32_t okey(float f) {
  const uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ofloat(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}
__device__ __forceinline__ void amin_key(uint32_t* a, float v) { if (v == v) atomicMin(a, okey(v)); }
__device__ __forceinline__ void amax_key(uint32_t* a, float v) { if (v == v) atomicMax(a, okey(v)); }

__device__ __forceinline__ float comp(const float4& v, int axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }

// Rust `f32 as usize` saturation then min(bins - 1) (blas.rs:198-201).
__device__ __forceinline__ uint32_t bin_index(float v, uint32_t bins) {
  if (!(v > 0.0f)) return 0;
  if (v >= __uint2float_rn(bins - 1)) return bins - 1;
  const uint32_t i = __float2uint_rz(v);
  return i < bins - 1 ? i : bins - 1;
}

// Box grown into a bin: the three vertices (BLAS, == their lattice box) or
// bounds_min and bounds_max (TLAS).
__device__ __forceinline__ void grow_box(const float4& a, const float4& b, bool tlas, float* mn, float* mx) {
  if (!tlas) {
    mn[0] = a.x; mn[1] = a.y; mn[2] = a.z;
    mx[0] = b.x; mx[1] = b.y; mx[2] = b.z;
  } else {
    mn[0] = lmin(a.x, b.x); mn[1] = lmin(a.y, b.y); mn[2] = lmin(a.z, b.z);
    mx[0] = lmax(a.x, b.x); mx[1] = lmax(a.y, b.y); mx[2] = lmax(a.z, b.z);
  }
}

__device__ __forceinline__ float box_area(float mnx, float mny, float mnz, float mxx, float mxy, float mxz) {
  const float ex = mxx - mnx, ey = mxy - mny, ez = mxz - mnz;
  return ex * ey + ey * ez + ez * ex;
}

struct Best { int axis; float pos, cost; };

// One axis of find_best_split_plane (blas.rs:208-237) by a full warp; lane i
// holds bin i (i < bins).  Prefix/suffix boxes are lattice scans (exact), the
// first minimum of the plane costs wins as with the reference's strict `<`.
__device__ __forceinline__ void sweep_axis(uint32_t bins, int axis, float bmin, float bmax, uint32_t cnt,
                                           float mnx, float mny, float mnz, float mxx, float mxy, float mxz,
                                           Best& best) {
  const int lane = threadIdx.x & 31;
  const bool in = lane < (int)bins;
  if (!in) { cnt = 0; mnx = mny = mnz = mxx = mxy = mxz = 0.0f; }
  uint32_t ca = cnt;
  float a0 = mnx, a1 = mny, a2 = mnz, a3 = mxx, a4 = mxy, a5 = mxz;
  uint32_t cb = cnt;
  float b0 = mnx, b1 = mny, b2 = mnz, b3 = mxx, b4 = mxy, b5 = mxz;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t oc = __shfl_up_sync(0xffffffffu, ca, off);
    const float o0 = __shfl_up_sync(0xffffffffu, a0, off), o1 = __shfl_up_sync(0xffffffffu, a1, off);
    const float o2 = __shfl_up_sync(0xffffffffu, a2, off), o3 = __shfl_up_sync(0xffffffffu, a3, off);
    const float o4 = __shfl_up_sync(0xffffffffu, a4, off), o5 = __shfl_up_sync(0xffffffffu, a5, off);
    if (lane >= off) {
      ca += oc;
      a0 = lmin(o0, a0); a1 = lmin(o1, a1); a2 = lmin(o2, a2);
      a3 = lmax(o3, a3); a4 = lmax(o4, a4); a5 = lmax(o5, a5);
    }
    const uint32_t pc = __shfl_down_sync(0xffffffffu, cb, off);
    const float p0 = __shfl_down_sync(0xffffffffu, b0, off), p1 = __shfl_down_sync(0xffffffffu, b1, off);
    const float p2 = __shfl_down_sync(0xffffffffu, b2, off), p3 = __shfl_down_sync(0xffffffffu, b3, off);
    const float p4 = __shfl_down_sync(0xffffffffu, b4, off), p5 = __shfl_down_sync(0xffffffffu, b5, off);
    if (lane + off < (int)bins) {
      cb += pc;
      b0 = lmin(b0, p0); b1 = lmin(b1, p1); b2 = lmin(b2, p2);
      b3 = lmax(b3, p3); b4 = lmax(b4, p4); b5 = lmax(b5, p5);
    }
  }
  // Plane i separates bins [0, i] from [i+1, bins).
  const uint32_t cbn = __shfl_down_sync(0xffffffffu, cb, 1);
  const float q0 = __shfl_down_sync(0xffffffffu, b0, 1), q1 = __shfl_down_sync(0xffffffffu, b1, 1);
  const float q2 = __shfl_down_sync(0xffffffffu, b2, 1), q3 = __shfl_down_sync(0xffffffffu, b3, 1);
  const float q4 = __shfl_down_sync(0xffffffffu, b4, 1), q5 = __shfl_down_sync(0xffffffffu, b5, 1);
  float cost = 0.0f;
  bool valid = false;
  if (lane < (int)bins - 1) {
    const float area_a = box_area(a0, a1, a2, a3, a4, a5);
    const float area_b = box_area(q0, q1, q2, q3, q4, q5);
    cost = __uint2float_rn(ca) * area_a + __uint2float_rn(cbn) * area_b;
    valid = cost < 1e30f;
  }
  // First minimum over the valid planes.
  float bc = valid ? cost : 0.0f;
  int bl = valid ? lane : 64;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const float oc = __shfl_xor_sync(0xffffffffu, bc, off);
    const int ol = __shfl_xor_sync(0xffffffffu, bl, off);
    const bool take = (ol < 64) && (bl >= 64 || oc < bc || (oc == bc && ol < bl));
    if (take) { bc = oc; bl = ol; }
  }
  if (bl < 64 && bc < best.cost) {
    const float bin_size = (bmax - bmin) / __uint2float_rn(bins);
    best.axis = axis;
    best.pos = bmin + bin_size * __uint2float_rn((uint32_t)bl + 1u);
    best.cost = bc;
  }
}

__device__ __forceinline__ float warp_lmin(float v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = lmin(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}
__device__ __forceinline__ float warp_lmax(float v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = lmax(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}

struct Rec { float4 lo, hi; };  // (min.xyz | a) (max.xyz | count), the 32 B node

// ------------------------------------------------------------ input prep
__global__ void k_prep_triangles(const float4* __restrict__ prims, uint32_t n, float4* pmin, float4* pmax,
                                 float4* cent) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 p0 = prims[3 * i], p1 = prims[3 * i + 1], p2 = prims[3 * i + 2];
  float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  const float4 v[3] = {p0, p1, p2};
  for (int k = 0; k < 3; ++k) { mn[0] = lmin(mn[0], v[k].x); mn[1] = lmin(mn[1], v[k].y); mn[2] = lmin(mn[2], v[k].z); }
  for (int k = 0; k < 3; ++k) { mx[0] = lmax(mx[0], v[k].x); mx[1] = lmax(mx[1], v[k].y); mx[2] = lmax(mx[2], v[k].z); }
  pmin[i] = make_float4(mn[0], mn[1], mn[2], 0.0f);
  pmax[i] = make_float4(mx[0], mx[1], mx[2], 0.0f);
  cent[i] = make_float4(mn[0] + 0.5f * (mx[0] - mn[0]), mn[1] + 0.5f * (mx[1] - mn[1]), mn[2] + 0.5f * (mx[2] - mn[2]), 0.0f);
}

__global__ void k_prep_instances(const float* __restrict__ b, uint32_t n, float4* pmin, float4* pmax, float4* cent) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* q = b + (size_t)i * 9;
  pmin[i] = make_float4(q[0], q[1], q[2], 0.0f);
  pmax[i] = make_float4(q[3], q[4], q[5], 0.0f);
  cent[i] = make_float4(q[6], q[7], q[8], 0.0f);
}

// ------------------------------------------------------------ root box
// Box of [first, first+count) of idx over pmin/pmax into keys[6] (min xyz, max xyz).
__global__ void k_range_box(const uint32_t* __restrict__ idx, const float4* __restrict__ pmin,
                            const float4* __restrict__ pmax, uint32_t first, uint32_t count, uint32_t* keys) {
  float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
    const uint32_t id = idx[first + k];
    const float4 a = pmin[id], b = pmax[id];
    mn[0] = lmin(mn[0], a.x); mn[1] = lmin(mn[1], a.y); mn[2] = lmin(mn[2], a.z);
    mx[0] = lmax(mx[0], b.x); mx[1] = lmax(mx[1], b.y); mx[2] = lmax(mx[2], b.z);
  }
  for (int c = 0; c < 3; ++c) { mn[c] = warp_lmin(mn[c]); mx[c] = warp_lmax(mx[c]); }
  if ((threadIdx.x & 31) == 0)
    for (int c = 0; c < 3; ++c) { amin_key(keys + c, mn[c]); amax_key(keys + 3 + c, mx[c]); }
}

// ------------------------------------------------------------ phase 1
struct Tile { uint32_t node, start, len, pad; };
struct LNode { uint32_t first, count; };  // active node of a level

// Per-node accumulators of a level (all keys):
//   cb[6]          centroid bounds  (min xyz, max xyz)
//   bins[3][B][7]  count, min xyz, max xyz
//   split          (axis, pos bits)
//   m              left count
//   child[12]      A box, B box
struct LevelAcc {
  uint32_t* cb;
  uint32_t* bins;
  uint32_t* split;
  uint32_t* child;
};

__global__ void k_level_init(LevelAcc acc, uint32_t n_nodes) {
  const uint32_t j = blockIdx.x;
  if (j >= n_nodes) return;
  const uint32_t k1e30 = okey(1e30f), km1e30 = okey(-1e30f), kzero = okey(0.0f);
  const uint32_t kmax = okey(FLT_MAX), kmin = okey(-FLT_MAX);
  for (uint32_t t = threadIdx.x; t < 6; t += blockDim.x) acc.cb[j * 6 + t] = t < 3 ? k1e30 : km1e30;
  for (uint32_t t = threadIdx.x; t < 3 * kMaxBins * 7; t += blockDim.x)
    acc.bins[(size_t)j * 3 * kMaxBins * 7 + t] = (t % 7) == 0 ? 0u : kzero;
  for (uint32_t t = threadIdx.x; t < 12; t += blockDim.x) acc.child[j * 12 + t] = (t % 6) < 3 ? kmax : kmin;
}

__device__ __forceinline__ void block_reduce_minmax6(float* v, float* red) {
  // v[0..2] lattice-min, v[3..5] lattice-max; result valid in thread 0.
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int c = 0; c < 3; ++c) { v[c] = warp_lmin(v[c]); v[3 + c] = warp_lmax(v[3 + c]); }
  if (lane == 0) for (int c = 0; c < 6; ++c) red[warp * 6 + c] = v[c];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < nw; ++w)
      for (int c = 0; c < 6; ++c) v[c] = c < 3 ? lmin(v[c], red[w * 6 + c]) : lmax(v[c], red[w * 6 + c]);
  }
}

__global__ void k_level_cbounds(const Tile* __restrict__ tiles, const uint32_t* __restrict__ idx,
                                const float4* __restrict__ cent, LevelAcc acc) {
  __shared__ float red[32 * 6];
  const Tile t = tiles[blockIdx.x];
  float v[6] = {1e30f, 1e30f, 1e30f, -1e30f, -1e30f, -1e30f};
  for (uint32_t k = threadIdx.x; k < t.len; k += blockDim.x) {
    const float4 c = cent[idx[t.start + k]];
    v[0] = lmin(v[0], c.x); v[1] = lmin(v[1], c.y); v[2] = lmin(v[2], c.z);
    v[3] = lmax(v[3], c.x); v[4] = lmax(v[4], c.y); v[5] = lmax(v[5], c.z);
  }
  block_reduce_minmax6(v, red);
  if (threadIdx.x == 0) {
    uint32_t* cb = acc.cb + t.node * 6;
    for (int c = 0; c < 3; ++c) { amin_key(cb + c, v[c]); amax_key(cb + 3 + c, v[3 + c]); }
  }
}

__global__ void k_level_bins(const Tile* __restrict__ tiles, const uint32_t* __restrict__ idx,
                             const float4* __restrict__ pmin, const float4* __restrict__ pmax,
                             const float4* __restrict__ cent, LevelAcc acc, uint32_t bins, uint32_t tlas) {
  __shared__ uint32_t sb[3 * kMaxBins * 7];
  __shared__ float bmn[3], bmx[3], binv[3];
  const Tile t = tiles[blockIdx.x];
  const uint32_t kzero = okey(0.0f);
  for (uint32_t i = threadIdx.x; i < 3 * kMaxBins * 7; i += blockDim.x) sb[i] = (i % 7) == 0 ? 0u : kzero;
  if (threadIdx.x < 3) {
    const uint32_t* cb = acc.cb + t.node * 6;
    bmn[threadIdx.x] = ofloat(cb[threadIdx.x]);
    bmx[threadIdx.x] = ofloat(cb[3 + threadIdx.x]);
    binv[threadIdx.x] = __uint2float_rn(bins) / (bmx[threadIdx.x] - bmn[threadIdx.x]);
  }
  __syncthreads();
  for (uint32_t k = threadIdx.x; k < t.len; k += blockDim.x) {
    const uint32_t id = idx[t.start + k];
    const float4 c = cent[id];
    float gmn[3], gmx[3];
    grow_box(pmin[id], pmax[id], tlas != 0, gmn, gmx);
    for (int axis = 0; axis < 3; ++axis) {
      if (bmn[axis] == bmx[axis]) continue;
      const uint32_t b = bin_index((comp(c, axis) - bmn[axis]) * binv[axis], bins);
      uint32_t* s = sb + (axis * kMaxBins + b) * 7;
      atomicAdd(s, 1u);
      for (int q = 0; q < 3; ++q) {
        if (gmn[q] == gmn[q]) atomicMin(s + 1 + q, okey(gmn[q]));
        if (gmx[q] == gmx[q]) atomicMax(s + 4 + q, okey(gmx[q]));
      }
    }
  }
  __syncthreads();
  uint32_t* g = acc.bins + (size_t)t.node * 3 * kMaxBins * 7;
  for (uint32_t i = threadIdx.x; i < 3 * kMaxBins; i += blockDim.x) {
    const uint32_t* s = sb + i * 7;
    if (s[0] == 0) continue;
    uint32_t* d = g + i * 7;
    atomicAdd(d, s[0]);
    for (int q = 0; q < 3; ++q) { atomicMin(d + 1 + q, s[1 + q]); atomicMax(d + 4 + q, s[4 + q]); }
  }
}

// One warp per node: the sweep of find_best_split_plane over the three axes.
__global__ void k_level_sweep(LevelAcc acc, uint32_t n_nodes, uint32_t bins) {
  const uint32_t j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (j >= n_nodes) return;
  const int lane = threadIdx.x & 31;
  const uint32_t* cb = acc.cb + j * 6;
  Best best{0, 0.0f, 1e30f};
  for (int axis = 0; axis < 3; ++axis) {
    const float bmin = ofloat(cb[axis]), bmax = ofloat(cb[3 + axis]);
    if (bmin == bmax) continue;
    const uint32_t* g = acc.bins + ((size_t)j * 3 * kMaxBins + axis * kMaxBins) * 7;
    uint32_t cnt = 0;
    float m[6] = {0, 0, 0, 0, 0, 0};
    if (lane < (int)bins) {
      const uint32_t* s = g + lane * 7;
      cnt = s[0];
      for (int q = 0; q < 6; ++q) m[q] = ofloat(s[1 + q]);
    }
    sweep_axis(bins, axis, bmin, bmax, cnt, m[0], m[1], m[2], m[3], m[4], m[5], best);
  }
  if (lane == 0) {
    acc.split[j * 2] = (uint32_t)best.axis;
    acc.split[j * 2 + 1] = __float_as_uint(best.pos);
  }
}

__global__ void k_level_flags(const Tile* __restrict__ tiles, const uint32_t* __restrict__ idx,
                              const float4* __restrict__ cent, LevelAcc acc, uint32_t* flags) {
  const Tile t = tiles[blockIdx.x];
  const int axis = (int)acc.split[t.node * 2];
  const float pos = __uint_as_float(acc.split[t.node * 2 + 1]);
  for (uint32_t k = threadIdx.x; k < t.len; k += blockDim.x)
    flags[t.start + k] = comp(cent[idx[t.start + k]], axis) < pos ? 1u : 0u;
}

// Exclusive scan of flags[0, n) into P[0, n] (3 kernels).
constexpr int kScanBlock = 1024;
constexpr int kScanItems = 4;
__global__ void k_scan_reduce(const uint32_t* __restrict__ in, uint32_t n, uint32_t* sums) {
  __shared__ uint32_t s[kScanBlock / 32];
  const uint64_t base = (uint64_t)blockIdx.x * kScanBlock * kScanItems;
  uint32_t acc = 0;
  for (int i = 0; i < kScanItems; ++i) {
    const uint64_t g = base + (uint64_t)i * kScanBlock + threadIdx.x;
    if (g < n) acc += in[g];
  }
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    uint32_t v = s[threadIdx.x];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if (threadIdx.x == 0) sums[blockIdx.x] = v;
  }
}
__global__ void k_scan_sums(uint32_t* sums, uint32_t nb) {
  // single block: exclusive scan in place
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < nb; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    uint32_t v = i < nb ? sums[i] : 0u;
    // block inclusive scan
    __shared__ uint32_t ws[32];
    uint32_t x = v;
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t o = __shfl_up_sync(0xffffffffu, x, off);
      if ((threadIdx.x & 31) >= (unsigned)off) x += o;
    }
    if ((threadIdx.x & 31) == 31) ws[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x < 32) {
      uint32_t w = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0u;
      for (int off = 1; off < 32; off <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, w, off);
        if (threadIdx.x >= (unsigned)off) w += o;
      }
      ws[threadIdx.x] = w;
    }
    __syncthreads();
    const uint32_t warp_prefix = (threadIdx.x >> 5) ? ws[(threadIdx.x >> 5) - 1] : 0u;
    const uint32_t incl = x + warp_prefix;
    if (i < nb) sums[i] = carry + incl - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry += incl;
    __syncthreads();
  }
}
__global__ void k_scan_apply(const uint32_t* __restrict__ in, uint32_t n, const uint32_t* __restrict__ sums,
                             uint32_t* out) {
  __shared__ uint32_t ws[kScanBlock / 32];
  __shared__ uint32_t carry;
  const uint64_t base = (uint64_t)blockIdx.x * kScanBlock * kScanItems;
  if (threadIdx.x == 0) carry = sums[blockIdx.x];
  __syncthreads();
  for (int it = 0; it < kScanItems; ++it) {
    const uint64_t g = base + (uint64_t)it * kScanBlock + threadIdx.x;
    const uint32_t v = g < n ? in[g] : 0u;
    uint32_t x = v;
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t o = __shfl_up_sync(0xffffffffu, x, off);
      if ((threadIdx.x & 31) >= (unsigned)off) x += o;
    }
    if ((threadIdx.x & 31) == 31) ws[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x < 32) {
      uint32_t w = ws[threadIdx.x];
      for (int off = 1; off < 32; off <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, w, off);
        if (threadIdx.x >= (unsigned)off) w += o;
      }
      ws[threadIdx.x] = w;
    }
    __syncthreads();
    const uint32_t incl = x + ((threadIdx.x >> 5) ? ws[(threadIdx.x >> 5) - 1] : 0u);
    if (g < n) out[g] = carry + incl - v;
    if (g == n) out[g] = carry + incl - v;  // total at P[n]
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry += incl;
    __syncthreads();
  }
}

__device__ __forceinline__ void node_counts(const uint32_t* P, uint32_t f, uint32_t n, uint32_t& m, uint32_t& LF,
                                            uint32_t& r) {
  const uint32_t p0 = P[f];
  m = P[f + n] - p0;
  LF = P[f + m] - p0;
  r = m - LF;
}

__global__ void k_level_frbl(const Tile* __restrict__ tiles, const LNode* __restrict__ nodes,
                             const uint32_t* __restrict__ flags, const uint32_t* __restrict__ P, uint32_t* FR,
                             uint32_t* BL) {
  const Tile t = tiles[blockIdx.x];
  const LNode nd = nodes[t.node];
  uint32_t m, LF, r;
  node_counts(P, nd.first, nd.count, m, LF, r);
  for (uint32_t q = threadIdx.x; q < t.len; q += blockDim.x) {
    const uint32_t g = t.start + q, k = g - nd.first;
    const uint32_t lb = P[g] - P[nd.first];
    const bool left = flags[g] != 0;
    if (k < m && !left) FR[nd.first + (k - lb)] = k;  // rank t = k - lb + 1 (< r)
    else if (k >= m && left && r - lb + LF - 1 < nd.count) BL[nd.first + (r - lb + LF) - 1] = k;  // top rank
  }
}

__device__ __forceinline__ uint32_t dest_of(uint32_t k, bool left, uint32_t n, uint32_t m, uint32_t LF, uint32_t r,
                                            uint32_t lb, const uint32_t* FR, const uint32_t* BL) {
  if (k < m) {
    if (left) return k;
    const uint32_t t = k - lb + 1;
    return t == 1 ? n - 1 : BL[t - 2] - 1;
  }
  if (left) return FR[(r - lb + LF) - 1];
  if (k == m) return r == 0 ? n - 1 : BL[r - 1] - 1;
  return k - 1;
}

__global__ void k_level_scatter(const Tile* __restrict__ tiles, const LNode* __restrict__ nodes,
                                const uint32_t* __restrict__ flags, const uint32_t* __restrict__ P,
                                const uint32_t* __restrict__ FR, const uint32_t* __restrict__ BL,
                                const uint32_t* __restrict__ idx, uint32_t* tmp, int* error) {
  const Tile t = tiles[blockIdx.x];
  const LNode nd = nodes[t.node];
  uint32_t m, LF, r;
  node_counts(P, nd.first, nd.count, m, LF, r);
  for (uint32_t q = threadIdx.x; q < t.len; q += blockDim.x) {
    const uint32_t g = t.start + q, k = g - nd.first;
    const uint32_t lb = P[g] - P[nd.first];
    const uint32_t d = dest_of(k, flags[g] != 0, nd.count, m, LF, r, lb, FR + nd.first, BL + nd.first);
    if (d < nd.count) tmp[nd.first + d] = idx[g];
    else atomicExch(error, -9);
  }
}

__global__ void k_level_copy_child(const Tile* __restrict__ tiles, const LNode* __restrict__ nodes,
                                   const uint32_t* __restrict__ P, const uint32_t* __restrict__ tmp, uint32_t* idx,
                                   const float4* __restrict__ pmin, const float4* __restrict__ pmax, LevelAcc acc) {
  __shared__ float red[32 * 6];
  const Tile t = tiles[blockIdx.x];
  const LNode nd = nodes[t.node];
  const uint32_t m = P[nd.first + nd.count] - P[nd.first];
  float va[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
  float vb[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (uint32_t q = threadIdx.x; q < t.len; q += blockDim.x) {
    const uint32_t g = t.start + q, k = g - nd.first;
    const uint32_t id = tmp[g];
    idx[g] = id;
    const float4 a = pmin[id], b = pmax[id];
    float* v = k < m ? va : vb;
    v[0] = lmin(v[0], a.x); v[1] = lmin(v[1], a.y); v[2] = lmin(v[2], a.z);
    v[3] = lmax(v[3], b.x); v[4] = lmax(v[4], b.y); v[5] = lmax(v[5], b.z);
  }
  block_reduce_minmax6(va, red);
  __syncthreads();
  block_reduce_minmax6(vb, red);
  if (threadIdx.x == 0) {
    uint32_t* c = acc.child + t.node * 12;
    for (int q = 0; q < 3; ++q) {
      amin_key(c + q, va[q]); amax_key(c + 3 + q, va[3 + q]);
      amin_key(c + 6 + q, vb[q]); amax_key(c + 9 + q, vb[3 + q]);
    }
  }
}

// ------------------------------------------------------------ phase 2
struct SmallRoot {
  uint32_t first, count, base, pad;  // base: first slot of this subtree in the local record buffer
  float4 lo, hi;                     // root box (a/count fields unused)
};

// Bin counts up to which a warp bins by reductions rather than shared atomics.
constexpr uint32_t kReduceBins = 8;

// Centroid bounds of node [f, f+n) of idx (lattice min / max, every lane
// gets them): v[0..2] min, v[3..5] max.
__device__ __forceinline__ void warp_cbounds(const uint32_t* idx, const float4* cent, uint32_t f, uint32_t n,
                                             float* v) {
  const int lane = threadIdx.x & 31;
  v[0] = v[1] = v[2] = 1e30f;
  v[3] = v[4] = v[5] = -1e30f;
  for (uint32_t k = lane; k < n; k += 32) {
    const float4 c = cent[idx[f + k]];
    v[0] = lmin(v[0], c.x); v[1] = lmin(v[1], c.y); v[2] = lmin(v[2], c.z);
    v[3] = lmax(v[3], c.x); v[4] = lmax(v[4], c.y); v[5] = lmax(v[5], c.z);
  }
  for (int c = 0; c < 3; ++c) { v[c] = warp_lmin(v[c]); v[3 + c] = warp_lmax(v[3 + c]); }
}

// One axis of find_best_split_plane (blas.rs:208-237) for node [f, f+n):
// bins over the centroid range [bmin, bmax] of that axis (bmin < bmax), then
// the sweep; updates best when a plane beats it (strict <, as the reference).
__device__ void warp_split_axis(const uint32_t* idx, const float4* pmin, const float4* pmax, const float4* cent,
                                uint32_t f, uint32_t n, uint32_t bins, bool tlas, uint32_t* sb, int axis,
                                float bmin, float bmax, Best& best) {
  const int lane = threadIdx.x & 31;
  const uint32_t kzero = okey(0.0f);
  const float inv = __uint2float_rn(bins) / (bmax - bmin);
  for (int i = lane; i < kMaxBins * 7; i += 32) sb[i] = (i % 7) == 0 ? 0u : kzero;
  __syncwarp();
  if (bins <= kReduceBins) {
    // Few bins (the TLAS's 2): per-bin warp reductions of the same ordered
    // keys instead of shared atomics that all lanes would aim at 2 words.
    for (uint32_t base = 0; base < n; base += 32) {
      const uint32_t k = base + lane;
      uint32_t b = 0xffffffffu;
      float gmn[3] = {0, 0, 0}, gmx[3] = {0, 0, 0};
      if (k < n) {
        const uint32_t id = idx[f + k];
        grow_box(pmin[id], pmax[id], tlas, gmn, gmx);
        b = bin_index((comp(cent[id], axis) - bmin) * inv, bins);
      }
      for (uint32_t j = 0; j < bins; ++j) {
        const bool in = b == j;
        const uint32_t cnt = __popc(__ballot_sync(0xffffffffu, in));
        if (cnt == 0) continue;
        uint32_t r[6];
        for (int q = 0; q < 3; ++q) {
          r[q] = __reduce_min_sync(0xffffffffu, in && gmn[q] == gmn[q] ? okey(gmn[q]) : 0xffffffffu);
          r[3 + q] = __reduce_max_sync(0xffffffffu, in && gmx[q] == gmx[q] ? okey(gmx[q]) : 0u);
        }
        if (lane == 0) {
          uint32_t* s = sb + j * 7;
          s[0] += cnt;
          for (int q = 0; q < 3; ++q) {
            s[1 + q] = s[1 + q] < r[q] ? s[1 + q] : r[q];
            s[4 + q] = s[4 + q] > r[3 + q] ? s[4 + q] : r[3 + q];
          }
        }
        __syncwarp();
      }
    }
  } else {
    for (uint32_t k = lane; k < n; k += 32) {
      const uint32_t id = idx[f + k];
      const float4 c = cent[id];
      float gmn[3], gmx[3];
      grow_box(pmin[id], pmax[id], tlas, gmn, gmx);
      const uint32_t b = bin_index((comp(c, axis) - bmin) * inv, bins);
      uint32_t* s = sb + b * 7;
      atomicAdd(s, 1u);
      for (int q = 0; q < 3; ++q) {
        if (gmn[q] == gmn[q]) atomicMin(s + 1 + q, okey(gmn[q]));
        if (gmx[q] == gmx[q]) atomicMax(s + 4 + q, okey(gmx[q]));
      }
    }
  }
  __syncwarp();
  uint32_t cnt = 0;
  float m[6] = {0, 0, 0, 0, 0, 0};
  if (lane < (int)bins) {
    const uint32_t* s = sb + lane * 7;
    cnt = s[0];
    for (int q = 0; q < 6; ++q) m[q] = ofloat(s[1 + q]);
  }
  __syncwarp();
  sweep_axis(bins, axis, bmin, bmax, cnt, m[0], m[1], m[2], m[3], m[4], m[5], best);
}

// find_best_split_plane with 2 bins (the TLAS's): every axis has the single
// plane between bin 0 and bin 1, so one warp evaluates the three axes at once
// -- per lane the bin-1 count and both bins' box keys of its elements on every
// axis, then independent warp reductions -- instead of three binning passes and
// three 32-lane sweeps.  Bin boxes start as the zero box, the cost expression
// and the strict `<` over the axes in order are sweep_axis's, so the result is
// the same bit for bit.
__device__ Best warp_split_bins2(const uint32_t* idx, const float4* pmin, const float4* pmax, const float4* cent,
                                 uint32_t f, uint32_t n, bool tlas) {
  const int lane = threadIdx.x & 31;
  float v[6];
  warp_cbounds(idx, cent, f, n, v);
  float inv[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) inv[a] = 2.0f / (v[3 + a] - v[a]);
  uint32_t c1[3] = {0u, 0u, 0u};
  uint32_t kmn[2][3][3], kmx[2][3][3];  // [bin][axis][component]
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int q = 0; q < 3; ++q) { kmn[j][a][q] = 0xffffffffu; kmx[j][a][q] = 0u; }
  for (uint32_t k = lane; k < n; k += 32) {
    const uint32_t id = idx[f + k];
    const float4 c = cent[id];
    float gmn[3], gmx[3];
    grow_box(pmin[id], pmax[id], tlas, gmn, gmx);
    uint32_t emn[3], emx[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      emn[q] = gmn[q] == gmn[q] ? okey(gmn[q]) : 0xffffffffu;
      emx[q] = gmx[q] == gmx[q] ? okey(gmx[q]) : 0u;
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const uint32_t b = bin_index((comp(c, a) - v[a]) * inv[a], 2u);
      c1[a] += b;
#pragma unroll
      for (int j = 0; j < 2; ++j)
        if (b == (uint32_t)j)
#pragma unroll
          for (int q = 0; q < 3; ++q) {
            kmn[j][a][q] = min(kmn[j][a][q], emn[q]);
            kmx[j][a][q] = max(kmx[j][a][q], emx[q]);
          }
    }
  }
  const uint32_t kzero = okey(0.0f);
  Best best{0, 0.0f, 1e30f};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (v[a] == v[3 + a]) continue;  // warp-uniform
    const uint32_t n1 = __reduce_add_sync(0xffffffffu, c1[a]);
    float m[2][6];
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        m[j][q] = ofloat(min(kzero, __reduce_min_sync(0xffffffffu, kmn[j][a][q])));
        m[j][3 + q] = ofloat(max(kzero, __reduce_max_sync(0xffffffffu, kmx[j][a][q])));
      }
    const float area_a = box_area(m[0][0], m[0][1], m[0][2], m[0][3], m[0][4], m[0][5]);
    const float area_b = box_area(m[1][0], m[1][1], m[1][2], m[1][3], m[1][4], m[1][5]);
    const float cost = __uint2float_rn(n - n1) * area_a + __uint2float_rn(n1) * area_b;
    if (cost < 1e30f && cost < best.cost) {
      const float bin_size = (v[3 + a] - v[a]) / 2.0f;
      best.axis = a;
      best.pos = v[a] + bin_size * 1.0f;
      best.cost = cost;
    }
  }
  return best;
}

// Warp-level split of node [f, f+n) of idx over the three axes in the
// reference's order; returns best.
__device__ Best warp_split(const uint32_t* idx, const float4* pmin, const float4* pmax, const float4* cent,
                           uint32_t f, uint32_t n, uint32_t bins, bool tlas, uint32_t* sb) {
  float v[6];
  warp_cbounds(idx, cent, f, n, v);
  Best best{0, 0.0f, 1e30f};
  for (int axis = 0; axis < 3; ++axis) {
    if (v[axis] == v[3 + axis]) continue;
    warp_split_axis(idx, pmin, pmax, cent, f, n, bins, tlas, sb, axis, v[axis], v[3 + axis], best);
  }
  return best;
}

// Warp-level partition of [f, f+n) (n <= 1024) by cent[axis] < pos with the
// reference's permutation; returns the left count m and the two children's
// boxes (lattice min / max of pmin / pmax: abox over [f, f+m), bbox over the
// rest; min xyz then max xyz).  Each element's side is read once: the flags of
// chunk c (elements 32c .. 32c+31) are kept as a mask in lane c.
__device__ uint32_t warp_partition(uint32_t* idx, uint32_t* tmp, uint32_t* FR, uint32_t* BL, const float4* cent,
                                   const float4* pmin, const float4* pmax, uint32_t f, uint32_t n, int axis,
                                   float pos, int* error, float* abox, float* bbox) {
  const int lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t chunks = (n + 31) / 32;
  if (chunks > 32) {
    if (lane == 0) atomicExch(error, -9);
    return 0;
  }
  uint32_t mine = 0, m = 0;
  for (uint32_t c = 0; c < chunks; ++c) {
    const uint32_t k = 32 * c + lane;
    const bool left = k < n && comp(cent[idx[f + k]], axis) < pos;
    const uint32_t bal = __ballot_sync(0xffffffffu, left);
    if ((uint32_t)lane == c) mine = bal;
    m += __popc(bal);
  }
  // LF: left elements among the first m positions
  uint32_t part = 0;
  if ((uint32_t)lane < chunks) {
    const uint32_t base = 32u * lane;
    if (base + 32 <= m) part = __popc(mine);
    else if (base < m) part = __popc(mine & ((1u << (m - base)) - 1u));
  }
  const uint32_t LF = __reduce_add_sync(0xffffffffu, part);
  const uint32_t r = m - LF;
  // FR / BL
  uint32_t lb_base = 0;
  for (uint32_t c = 0; c < chunks; ++c) {
    const uint32_t k = 32 * c + lane;
    const uint32_t bal = __shfl_sync(0xffffffffu, mine, c);
    const bool left = (bal >> lane) & 1u;
    const uint32_t lb = lb_base + __popc(bal & lt);
    if (k < n) {
      if (k < m && !left) FR[k - lb] = k;
      else if (k >= m && left && r - lb + LF - 1 < n) BL[(r - lb + LF) - 1] = k;
    }
    lb_base += __popc(bal);
  }
  __syncwarp();
  lb_base = 0;
  for (uint32_t c = 0; c < chunks; ++c) {
    const uint32_t k = 32 * c + lane;
    const uint32_t bal = __shfl_sync(0xffffffffu, mine, c);
    const bool left = (bal >> lane) & 1u;
    const uint32_t lb = lb_base + __popc(bal & lt);
    if (k < n) {
      const uint32_t d = dest_of(k, left, n, m, LF, r, lb, FR, BL);
      if (d < n) tmp[d] = idx[f + k];
      else atomicExch(error, -9);
    }
    lb_base += __popc(bal);
  }
  __syncwarp();
  float va[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
  float vb[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (uint32_t k = lane; k < n; k += 32) {
    const uint32_t id = tmp[k];
    idx[f + k] = id;
    const float4 a = pmin[id], b = pmax[id];
    float* v = k < m ? va : vb;
    v[0] = lmin(v[0], a.x); v[1] = lmin(v[1], a.y); v[2] = lmin(v[2], a.z);
    v[3] = lmax(v[3], b.x); v[4] = lmax(v[4], b.y); v[5] = lmax(v[5], b.z);
  }
  for (int c = 0; c < 3; ++c) {
    abox[c] = warp_lmin(va[c]); abox[3 + c] = warp_lmax(va[3 + c]);
    bbox[c] = warp_lmin(vb[c]); bbox[3 + c] = warp_lmax(vb[3 + c]);
  }
  __syncwarp();
  return m;
}

// ------------------------------------------------------------ block builder
// One subtree of at most kBlockCap elements built by one block of kBlockWarps
// warps, breadth first: every node of a level is split by its own warp (the
// same warp_split / warp_partition as above, on element ranges that do not
// overlap, so the warps of a level work side by side), children are given
// slots in the order the warps finish, and the slots of level L + 1 are
// exactly those handed out while level L ran.  The reference numbers its
// nodes depth first (children allocated as a pair when a node is split, the A
// subtree before the B subtree, src/scene/blas.rs:130-160), so two more
// level sweeps give every node that number: subtree sizes bottom-up, then
// child bases top-down (A's children at base + 2, B's after A's subtree).
// Everything lives in shared memory; the elements are staged under local ids.
//
// Records: as k_subtree_staged (rec[base] the small root, rec[base + 1 + L]
// local node L in depth-first pair order, interior a = local child base,
// leaf a = global first).  In direct mode (one root, the whole input: the
// per-frame TLAS) the root box is reduced here and the nodes are written in
// their final numbering (root 0, local node L at 1 + L) straight to `rec`,
// with the node count and levels in meta[0], meta[1]: the build needs no
// host round trip.
constexpr uint32_t kBlockCap = 1024;
constexpr int kBlockWarps = 16;

__host__ __device__ constexpr size_t block_smem(uint32_t cap) {
  // elements: lo, hi, centroid (float4), gid, lidx, ltmp, FR, BL;
  // nodes (2 cap): lo, hi (float4), first, count, child, desc, id, child base;
  // level starts (cap + 2), per-warp bins
  return (size_t)cap * (3 * 16 + 5 * 4) + (size_t)2 * cap * (2 * 16 + 6 * 4) + (size_t)(cap + 2) * 4 +
         (size_t)kBlockWarps * kMaxBins * 7 * 4;
}

// B2: the build has 2 bins (the TLAS's), split by warp_split_bins2; its own
// instantiation keeps the register count of the general one down.
template <bool B2>
__global__ void __launch_bounds__(32 * kBlockWarps) k_subtree_block(
    uint32_t* idx, const float4* __restrict__ pmin, const float4* __restrict__ pmax,
    const float4* __restrict__ cent, const SmallRoot* __restrict__ roots, uint32_t n_roots, uint32_t cap,
    uint32_t bins, uint32_t max_leaf, uint32_t tlas, Rec* rec, uint32_t* local_count, int* error,
    uint32_t direct_n, uint32_t* meta) {
  extern __shared__ float4 sm[];
  __shared__ uint32_t alloc, n_levels;
  __shared__ float red[kBlockWarps * 6];
  __shared__ float ax_cost[kBlockWarps], ax_pos[kBlockWarps];  // per-axis split of a level's few nodes
  const uint32_t w = blockIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool direct = direct_n != 0;
  SmallRoot R;
  if (direct) {
    R.first = 0; R.count = direct_n; R.base = 0;
  } else {
    if (w >= n_roots) return;
    R = roots[w];
  }
  if (R.count > cap || R.count == 0) {  // the host sizes cap from the roots; this cannot happen
    if (threadIdx.x == 0) atomicExch(error, -9);
    return;
  }
  float4* lmn = sm;
  float4* lmx = lmn + cap;
  float4* lcen = lmx + cap;
  float4* nlo = lcen + cap;
  float4* nhi = nlo + 2 * (size_t)cap;
  uint32_t* gid = reinterpret_cast<uint32_t*>(nhi + 2 * (size_t)cap);
  uint32_t* lidx = gid + cap;
  uint32_t* ltmp = lidx + cap;
  uint32_t* lFR = ltmp + cap;
  uint32_t* lBL = lFR + cap;
  uint32_t* nfirst = lBL + cap;
  uint32_t* ncount = nfirst + 2 * cap;
  uint32_t* nchild = ncount + 2 * cap;  // slot of A (B = A + 1); 0 = leaf
  uint32_t* ndesc = nchild + 2 * cap;   // nodes below
  uint32_t* nid = ndesc + 2 * cap;      // depth-first local id (root: unused)
  uint32_t* ncb = nid + 2 * cap;        // depth-first local id of A
  uint32_t* lstart = ncb + 2 * cap;     // first slot of every level
  uint32_t* sb = lstart + cap + 2 + warp * kMaxBins * 7;
  for (uint32_t k = threadIdx.x; k < R.count; k += blockDim.x) {
    const uint32_t id = direct ? k : idx[R.first + k];  // direct: the identity permutation
    gid[k] = id;
    lidx[k] = k;
    lmn[k] = pmin[id];
    lmx[k] = pmax[id];
    lcen[k] = cent[id];
  }
  if (direct) {
    // root box: lattice min / max of every element's box
    float v[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t k = threadIdx.x; k < R.count; k += blockDim.x) {
      const float4 a = pmin[k], b = pmax[k];
      v[0] = lmin(v[0], a.x); v[1] = lmin(v[1], a.y); v[2] = lmin(v[2], a.z);
      v[3] = lmax(v[3], b.x); v[4] = lmax(v[4], b.y); v[5] = lmax(v[5], b.z);
    }
    for (int c = 0; c < 3; ++c) { v[c] = warp_lmin(v[c]); v[3 + c] = warp_lmax(v[3 + c]); }
    if (lane == 0) for (int c = 0; c < 6; ++c) red[warp * 6 + c] = v[c];
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int q = 1; q < kBlockWarps; ++q)
        for (int c = 0; c < 6; ++c) v[c] = c < 3 ? lmin(v[c], red[q * 6 + c]) : lmax(v[c], red[q * 6 + c]);
      nlo[0] = make_float4(v[0], v[1], v[2], 0.0f);
      nhi[0] = make_float4(v[3], v[4], v[5], 0.0f);
    }
  } else if (threadIdx.x == 0) {
    nlo[0] = R.lo;
    nhi[0] = R.hi;
  }
  if (threadIdx.x == 0) {
    nfirst[0] = 0;
    ncount[0] = R.count;
    nchild[0] = 0;
    alloc = 1;
    lstart[0] = 0;
    lstart[1] = 1;
    n_levels = 1;
  }
  __syncthreads();
  // ---- topology, one level at a time (a tree of cap elements has < cap levels)
  // A level of at most kBlockWarps / 3 nodes (the top of every subtree, where
  // the nodes are largest) first evaluates its nodes' three axes on three
  // warps each; the warp of axis 0 then takes the first minimum in axis order
  // with the reference's strict < (what warp_split does in one warp).
  auto finish_node = [&](uint32_t slot, uint32_t f, uint32_t n, const Best& bs) {
    float ab[6], bb[6];
    const uint32_t m = warp_partition(lidx, ltmp + f, lFR + f, lBL + f, lcen, lmn, lmx, f, n, bs.axis, bs.pos, error,
                                      ab, bb);
    if (m == 0 && R.first + f == 0) {
      if (lane == 0) atomicExch(error, -7);
      return;
    }
    if (m == 0 || m == n) return;
    const float* amn = ab;
    const float* amx = ab + 3;
    const float* bmn = bb;
    const float* bmx = bb + 3;
    if (lane == 0) {
      const uint32_t c = atomicAdd(&alloc, 2u);
      if (c + 1 < 2 * cap) {
        nchild[slot] = c;
        nfirst[c] = f; ncount[c] = m; nchild[c] = 0;
        nlo[c] = make_float4(amn[0], amn[1], amn[2], 0.0f);
        nhi[c] = make_float4(amx[0], amx[1], amx[2], 0.0f);
        nfirst[c + 1] = f + m; ncount[c + 1] = n - m; nchild[c + 1] = 0;
        nlo[c + 1] = make_float4(bmn[0], bmn[1], bmn[2], 0.0f);
        nhi[c + 1] = make_float4(bmx[0], bmx[1], bmx[2], 0.0f);
      } else {
        atomicExch(error, -9);
      }
    }
    __syncwarp();
  };
  for (uint32_t L = 0; L < cap; ++L) {
    const uint32_t a = lstart[L], b = lstart[L + 1];
    if (a == b) break;
    if (!B2 && (b - a) * 3 <= (uint32_t)kBlockWarps) {
      if ((uint32_t)warp < (b - a) * 3) {
        const uint32_t slot = a + warp / 3;
        const int axis = warp % 3;
        const uint32_t f = nfirst[slot], n = ncount[slot];
        Best bb{axis, 0.0f, 1e30f};
        if (n > max_leaf) {
          float v[6];
          warp_cbounds(lidx, lcen, f, n, v);
          if (v[axis] != v[3 + axis])
            warp_split_axis(lidx, lmn, lmx, lcen, f, n, bins, tlas != 0, sb, axis, v[axis], v[3 + axis], bb);
        }
        if (lane == 0) {
          ax_cost[warp] = bb.cost;
          ax_pos[warp] = bb.pos;
        }
      }
      __syncthreads();
      if ((uint32_t)warp < (b - a) * 3 && warp % 3 == 0) {
        const uint32_t slot = a + warp / 3;
        const uint32_t f = nfirst[slot], n = ncount[slot];
        if (n > max_leaf) {
          Best bs{0, 0.0f, 1e30f};
          for (int ax = 0; ax < 3; ++ax)
            if (ax_cost[warp + ax] < bs.cost) bs = Best{ax, ax_pos[warp + ax], ax_cost[warp + ax]};
          finish_node(slot, f, n, bs);
        }
      }
    } else {
      for (uint32_t slot = a + warp; slot < b; slot += kBlockWarps) {
        const uint32_t f = nfirst[slot], n = ncount[slot];
        if (n <= max_leaf) continue;  // a leaf
        finish_node(slot, f, n,
                    B2 ? warp_split_bins2(lidx, lmn, lmx, lcen, f, n, tlas != 0)
                       : warp_split(lidx, lmn, lmx, lcen, f, n, bins, tlas != 0, sb));
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const uint32_t end = alloc < 2 * cap ? alloc : 2 * cap;
      lstart[L + 2] = end;
      if (end > b) n_levels = L + 2;
    }
    __syncthreads();
  }
  const uint32_t levels = n_levels;
  // ---- subtree sizes, deepest level first
  for (int L = (int)levels - 1; L >= 0; --L) {
    for (uint32_t slot = lstart[L] + threadIdx.x; slot < lstart[L + 1]; slot += blockDim.x) {
      const uint32_t c = nchild[slot];
      ndesc[slot] = c ? 2 + ndesc[c] + ndesc[c + 1] : 0;
    }
    __syncthreads();
  }
  // ---- depth-first local ids, top down: the root's children are 0 and 1,
  // A's children follow the pair, B's follow A's subtree
  if (threadIdx.x == 0) ncb[0] = 0;
  __syncthreads();
  for (uint32_t L = 0; L < levels; ++L) {
    for (uint32_t slot = lstart[L] + threadIdx.x; slot < lstart[L + 1]; slot += blockDim.x) {
      const uint32_t c = nchild[slot];
      if (!c) continue;
      const uint32_t cb = ncb[slot];
      nid[c] = cb;
      nid[c + 1] = cb + 1;
      ncb[c] = cb + 2;
      ncb[c + 1] = cb + 2 + ndesc[c];
    }
    __syncthreads();
  }
  // ---- records (direct: final numbering, local id L at 1 + L)
  const uint32_t shift = direct ? 1u : 0u;
  const uint32_t total = lstart[levels];
  for (uint32_t slot = threadIdx.x; slot < total; slot += blockDim.x) {
    const uint32_t c = nchild[slot];
    float4 lo = nlo[slot], hi = nhi[slot];
    if (c) {
      lo.w = __uint_as_float(ncb[slot] + shift);
      hi.w = __uint_as_float(0u);
    } else {
      lo.w = __uint_as_float(R.first + nfirst[slot]);
      hi.w = __uint_as_float(ncount[slot]);
    }
    const uint32_t local = slot == 0 ? 0u : 1u + nid[slot];
    if (local < 2 * R.count - 1) rec[R.base + local] = Rec{lo, hi};
    else atomicExch(error, -9);
  }
  for (uint32_t k = threadIdx.x; k < R.count; k += blockDim.x) idx[R.first + k] = gid[lidx[k]];
  if (threadIdx.x == 0) {
    if (direct) {
      meta[0] = 1u + ndesc[0];
      meta[1] = levels;
    } else {
      local_count[w] = ndesc[0];
      local_count[n_roots + w] = levels;
    }
  }
}

// P[first] and P[first + count] of every node of a level (its left count is
// their difference), for one copy to the host.
__global__ void k_level_pfl(const LNode* __restrict__ ln, uint32_t na, const uint32_t* __restrict__ P,
                            uint32_t* out) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= na) return;
  out[2 * j] = P[ln[j].first];
  out[2 * j + 1] = P[ln[j].first + ln[j].count];
}

__global__ void k_iota(uint32_t* idx, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) idx[i] = i;
}

__global__ void k_init_roots(const SmallRoot* __restrict__ roots, uint32_t n_roots, Rec* rec) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_roots) return;
  const SmallRoot R = roots[i];
  rec[R.base] = Rec{make_float4(R.lo.x, R.lo.y, R.lo.z, __uint_as_float(R.first)),
                    make_float4(R.hi.x, R.hi.y, R.hi.z, __uint_as_float(R.count))};
}

// ------------------------------------------------------------ emit
struct Place { uint32_t final_index, base, pad0, pad1; };  // per small root

__global__ void k_emit_small(const SmallRoot* __restrict__ roots, const Place* __restrict__ places,
                             const uint32_t* __restrict__ local_count, const Rec* __restrict__ rec, uint32_t n_roots,
                             Rec* out, uint32_t capacity, int* error) {
  const uint32_t r = blockIdx.x;
  if (r >= n_roots) return;
  const SmallRoot R = roots[r];
  const Place P = places[r];
  const uint32_t cnt = local_count[r];
  for (uint32_t L = threadIdx.x; L <= cnt; L += blockDim.x) {
    Rec x = rec[R.base + L];
    const bool interior = __float_as_uint(x.hi.w) == 0u;
    if (interior) x.lo.w = __uint_as_float(P.base + __float_as_uint(x.lo.w));
    const uint32_t where = L == 0 ? P.final_index : P.base + (L - 1);
    if (where < capacity) out[where] = x;
    else atomicExch(error, -9);
  }
}

__global__ void k_emit_nodes(const uint32_t* __restrict__ where, const Rec* __restrict__ src, uint32_t n, Rec* out,
                             uint32_t capacity, int* error) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (where[i] < capacity) out[where[i]] = src[i];
  else atomicExch(error, -9);
}

inline size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

// Raises k_subtree_block's shared-memory limit for the current device (once).
cudaError_t block_attr() {
  static std::atomic<uint64_t> done{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint64_t bit = dev < 64 ? (uint64_t)1 << dev : 0;
  if (bit && (done.load() & bit)) return cudaSuccess;
  e = cudaFuncSetAttribute(k_subtree_block<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)block_smem(kBlockCap));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_subtree_block<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)block_smem(kBlockCap));
  if (e == cudaSuccess && bit) done.fetch_or(bit);
  return e;
}

}  // namespace

uint32_t direct_max() { return kBlockCap; }

cudaError_t build_direct(const Input& in, const Params& p, uint32_t* out_nodes, uint32_t* out_idx, uint32_t* meta,
                         cudaStream_t st) {
  if (in.n == 0 || in.n > kBlockCap || p.bins < 2 || p.bins > (uint32_t)kMaxBins) return cudaErrorInvalidValue;
  cudaError_t e = block_attr();
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(meta, 0, 4 * sizeof(uint32_t), st);
  if (e != cudaSuccess) return e;
  (p.bins == 2u ? k_subtree_block<true> : k_subtree_block<false>)<<<1, 32 * kBlockWarps, block_smem(in.n), st>>>(
      out_idx, in.pmin, in.pmax, in.cent, nullptr, 1, in.n, p.bins, p.max_leaf, p.tlas,
      reinterpret_cast<Rec*>(out_nodes), nullptr, reinterpret_cast<int*>(meta + 2), in.n, meta);
  return cudaGetLastError();
}

void Scratch::release() {
  if (buf) cudaFree(buf);
  buf = nullptr;
  bytes = 0;
}

cudaError_t prep_triangles(const float4* prims, uint32_t n, float4* pmin, float4* pmax, float4* cent,
                           cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_prep_triangles<<<(n + 255) / 256, 256, 0, st>>>(prims, n, pmin, pmax, cent);
  return cudaGetLastError();
}

cudaError_t prep_instances(const float* bounds9, uint32_t n, float4* pmin, float4* pmax, float4* cent,
                           cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_prep_instances<<<(n + 255) / 256, 256, 0, st>>>(bounds9, n, pmin, pmax, cent);
  return cudaGetLastError();
}

namespace {

struct HNode {
  uint32_t first, count;
  float mn[3], mx[3];
  int32_t child = -1;  // index of A in hnodes (B = child + 1)
  int32_t small = -1;  // index in small roots
  uint64_t desc = 0;   // descendants (2 * interior nodes below and including self if interior)
  uint32_t depth = 1;  // level of the node (root 1)
};

float key_to_float(uint32_t k) {
  const uint32_t b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  float f;
  std::memcpy(&f, &b, 4);
  return f;
}

}  // namespace

int build(const Input& in, const Params& p, uint32_t* out_nodes, uint32_t* out_idx, uint32_t* node_count,
          Scratch& scratch, cudaStream_t st, std::string* err, uint32_t* levels) {
  const uint32_t n = in.n;
  if (n == 0 || p.bins < 2 || p.bins > (uint32_t)kMaxBins) {
    if (err) *err = "bvh::build: need n > 0 and 2 <= bins <= 32";
    return -1;
  }
  // ---- a tree of at most kBlockCap elements: one block, one launch
  if (n <= kBlockCap) {
    if (scratch.bytes < 256) {
      scratch.release();
      cudaError_t e = pt::dev_alloc((void**)&scratch.buf, 256);
      if (e != cudaSuccess) { scratch.buf = nullptr; if (err) *err = "bvh scratch alloc"; return (int)e; }
      scratch.bytes = 256;
    }
    uint32_t* meta = (uint32_t*)scratch.buf;
    cudaError_t e = build_direct(in, p, out_nodes, out_idx, meta, st);
    ++scratch.launches;
    uint32_t h[4] = {0, 0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, meta, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { if (err) *err = "bvh block build"; return (int)e; }
    if ((int)h[2] == -9) { if (err) *err = "bvh: internal index check failed"; return -9; }
    if ((int)h[2] == -7) {
      if (err) *err = "degenerate split: the reference's partition would underflow (blas.rs:114-121)";
      return -7;
    }
    *node_count = h[0];
    if (levels) *levels = h[1];
    return 0;
  }
  // ---- scratch layout
  // Subtrees of at most `small` elements go to one block each.
  const uint32_t small = kSmall;
  const uint32_t max_level_nodes = n / (small + 1) + 1;
  const size_t off_tmp = 0;
  const size_t off_fr = align_up(off_tmp + (size_t)n * 4);
  const size_t off_bl = align_up(off_fr + (size_t)n * 4);
  const size_t off_flags = align_up(off_bl + (size_t)n * 4);
  const size_t off_P = align_up(off_flags + (size_t)n * 4);
  const size_t off_sums = align_up(off_P + (size_t)(n + 1) * 4);
  const uint32_t scan_blocks = (n + 1 + kScanBlock * kScanItems - 1) / (kScanBlock * kScanItems);
  const size_t off_rec = align_up(off_sums + (size_t)scan_blocks * 4);
  const size_t off_lcnt = align_up(off_rec + (size_t)(2 * (size_t)n) * 32);
  const size_t off_cb = align_up(off_lcnt + (size_t)(n + 4) * 4);  // counts and levels of the small roots
  const size_t off_bins = align_up(off_cb + (size_t)max_level_nodes * 6 * 4);
  const size_t off_split = align_up(off_bins + (size_t)max_level_nodes * 3 * kMaxBins * 7 * 4);
  const size_t off_child = align_up(off_split + (size_t)max_level_nodes * 2 * 4);
  const size_t off_tiles = align_up(off_child + (size_t)max_level_nodes * 12 * 4);
  const size_t max_tiles = (size_t)n / kTile + max_level_nodes + 1;
  const size_t off_lnodes = align_up(off_tiles + max_tiles * sizeof(Tile));
  const size_t off_roots = align_up(off_lnodes + (size_t)max_level_nodes * sizeof(LNode));
  const size_t max_roots = (size_t)n / 2 + 2;
  const size_t off_places = align_up(off_roots + max_roots * sizeof(SmallRoot));
  const size_t off_pfl = align_up(off_places + max_roots * sizeof(Place));
  const size_t off_err = align_up(off_pfl + (size_t)max_level_nodes * 2 * 4);
  const size_t total = align_up(off_err + 256);
  if (scratch.bytes < total) {
    scratch.release();
    cudaError_t e = pt::dev_alloc((void**)&scratch.buf, total);
    if (e != cudaSuccess) { scratch.buf = nullptr; if (err) *err = "bvh scratch alloc"; return (int)e; }
    scratch.bytes = total;
  }
  char* S = (char*)scratch.buf;
  uint32_t* tmp = (uint32_t*)(S + off_tmp);
  uint32_t* FR = (uint32_t*)(S + off_fr);
  uint32_t* BL = (uint32_t*)(S + off_bl);
  uint32_t* flags = (uint32_t*)(S + off_flags);
  uint32_t* P = (uint32_t*)(S + off_P);
  uint32_t* sums = (uint32_t*)(S + off_sums);
  Rec* rec = (Rec*)(S + off_rec);
  uint32_t* lcnt = (uint32_t*)(S + off_lcnt);
  LevelAcc acc{(uint32_t*)(S + off_cb), (uint32_t*)(S + off_bins), (uint32_t*)(S + off_split),
               (uint32_t*)(S + off_child)};
  Tile* d_tiles = (Tile*)(S + off_tiles);
  LNode* d_lnodes = (LNode*)(S + off_lnodes);
  SmallRoot* d_roots = (SmallRoot*)(S + off_roots);
  Place* d_places = (Place*)(S + off_places);
  uint32_t* d_pfl = (uint32_t*)(S + off_pfl);
  int* d_err = (int*)(S + off_err);

  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t x) { if (e == cudaSuccess && x != cudaSuccess) e = x; };
  // identity permutation, written on the device (no host buffer, no wait)
  k_iota<<<(n + 255) / 256, 256, 0, st>>>(out_idx, n);
  ++scratch.launches;
  chk(cudaGetLastError());
  chk(cudaMemsetAsync(d_err, 0, 4, st));
  // root box
  uint32_t root_keys[6];
  {
    uint32_t init[6];
    const float fm = FLT_MAX, fmn = -FLT_MAX;
    uint32_t bm, bmn;
    std::memcpy(&bm, &fm, 4);
    std::memcpy(&bmn, &fmn, 4);
    const uint32_t kmax = bm | 0x80000000u, kmin = ~bmn;
    for (int c = 0; c < 3; ++c) { init[c] = kmax; init[3 + c] = kmin; }
    chk(cudaMemcpyAsync(flags, init, 24, cudaMemcpyHostToDevice, st));
    const uint32_t blocks = std::min<uint32_t>(1024, (n + 255) / 256);
    k_range_box<<<blocks, 256, 0, st>>>(out_idx, in.pmin, in.pmax, 0, n, flags);
    ++scratch.launches;
    chk(cudaGetLastError());
    chk(cudaMemcpyAsync(root_keys, flags, 24, cudaMemcpyDeviceToHost, st));
    chk(cudaStreamSynchronize(st));
  }
  if (e != cudaSuccess) { if (err) *err = "bvh root box"; return (int)e; }
  std::vector<HNode> h;
  HNode root;
  root.first = 0;
  root.count = n;
  for (int c = 0; c < 3; ++c) { root.mn[c] = key_to_float(root_keys[c]); root.mx[c] = key_to_float(root_keys[3 + c]); }
  h.push_back(root);
  std::vector<SmallRoot> roots;
  auto classify = [&](uint32_t hi) {
    HNode& x = h[hi];
    if (x.count <= p.max_leaf) return 0;  // leaf
    if (x.count <= small) {
      SmallRoot R{};
      R.first = x.first;
      R.count = x.count;
      R.lo = make_float4(x.mn[0], x.mn[1], x.mn[2], 0.0f);
      R.hi = make_float4(x.mx[0], x.mx[1], x.mx[2], 0.0f);
      x.small = (int32_t)roots.size();
      roots.push_back(R);
      return 0;
    }
    return 1;  // active
  };
  std::vector<uint32_t> active;
  if (classify(0)) active.push_back(0);
  int host_error = 0;
  // ---- phase 1
  while (!active.empty() && e == cudaSuccess) {
    const uint32_t na = (uint32_t)active.size();
    std::vector<LNode> ln(na);
    std::vector<Tile> tiles;
    // tiles of at least kTile elements, about kTilesPerLevel of them for the
    // level: every SM busy, few blocks merging into each node's bins
    uint64_t level_elems = 0;
    for (uint32_t j = 0; j < na; ++j) level_elems += h[active[j]].count;
    const uint32_t tile = (uint32_t)std::max<uint64_t>(kTile, (level_elems + kTilesPerLevel - 1) / kTilesPerLevel);
    for (uint32_t j = 0; j < na; ++j) {
      const HNode& x = h[active[j]];
      ln[j] = LNode{x.first, x.count};
      for (uint32_t s = 0; s < x.count; s += tile) tiles.push_back(Tile{j, x.first + s, std::min(tile, x.count - s), 0});
    }
    const uint32_t nt = (uint32_t)tiles.size();
    chk(cudaMemcpyAsync(d_lnodes, ln.data(), na * sizeof(LNode), cudaMemcpyHostToDevice, st));
    chk(cudaMemcpyAsync(d_tiles, tiles.data(), nt * sizeof(Tile), cudaMemcpyHostToDevice, st));
    k_level_init<<<na, 128, 0, st>>>(acc, na);
    ++scratch.launches;
    k_level_cbounds<<<nt, 256, 0, st>>>(d_tiles, out_idx, in.cent, acc);
    ++scratch.launches;
    k_level_bins<<<nt, 256, 0, st>>>(d_tiles, out_idx, in.pmin, in.pmax, in.cent, acc, p.bins, p.tlas);
    ++scratch.launches;
    k_level_sweep<<<(na * 32 + 127) / 128, 128, 0, st>>>(acc, na, p.bins);
    ++scratch.launches;
    chk(cudaMemsetAsync(flags, 0, (size_t)n * 4, st));
    k_level_flags<<<nt, 256, 0, st>>>(d_tiles, out_idx, in.cent, acc, flags);
    ++scratch.launches;
    k_scan_reduce<<<scan_blocks, kScanBlock, 0, st>>>(flags, n, sums);
    ++scratch.launches;
    k_scan_sums<<<1, 1024, 0, st>>>(sums, scan_blocks);
    ++scratch.launches;
    k_scan_apply<<<scan_blocks, kScanBlock, 0, st>>>(flags, n, sums, P);
    ++scratch.launches;
    k_level_frbl<<<nt, 256, 0, st>>>(d_tiles, d_lnodes, flags, P, FR, BL);
    ++scratch.launches;
    k_level_scatter<<<nt, 256, 0, st>>>(d_tiles, d_lnodes, flags, P, FR, BL, out_idx, tmp, d_err);
    ++scratch.launches;
    k_level_copy_child<<<nt, 256, 0, st>>>(d_tiles, d_lnodes, P, tmp, out_idx, in.pmin, in.pmax, acc);
    ++scratch.launches;
    chk(cudaGetLastError());
    std::vector<uint32_t> child_keys((size_t)na * 12);
    std::vector<uint32_t> pfl((size_t)na * 2), pf(na), pl(na);
    chk(cudaMemcpyAsync(child_keys.data(), acc.child, (size_t)na * 48, cudaMemcpyDeviceToHost, st));
    // m per node = P[first + count] - P[first], both gathered into one copy
    k_level_pfl<<<(na + 127) / 128, 128, 0, st>>>(d_lnodes, na, P, d_pfl);
    ++scratch.launches;
    chk(cudaMemcpyAsync(pfl.data(), d_pfl, (size_t)na * 8, cudaMemcpyDeviceToHost, st));
    chk(cudaStreamSynchronize(st));
    for (uint32_t j = 0; j < na; ++j) {
      pf[j] = pfl[2 * (size_t)j];
      pl[j] = pfl[2 * (size_t)j + 1];
    }
    if (e != cudaSuccess) break;
    std::vector<uint32_t> next;
    for (uint32_t j = 0; j < na; ++j) {
      const uint32_t hi = active[j];
      const uint32_t m = pl[j] - pf[j];
      const uint32_t f = h[hi].first, cnt = h[hi].count;
      if (m == 0 && f == 0) { host_error = -7; continue; }
      if (m == 0 || m == cnt) continue;  // stays a leaf (after the reference's permutation)
      const int32_t ca = (int32_t)h.size();
      HNode A, B;
      A.first = f; A.count = m;
      B.first = f + m; B.count = cnt - m;
      for (int c = 0; c < 3; ++c) {
        A.mn[c] = key_to_float(child_keys[j * 12 + c]); A.mx[c] = key_to_float(child_keys[j * 12 + 3 + c]);
        B.mn[c] = key_to_float(child_keys[j * 12 + 6 + c]); B.mx[c] = key_to_float(child_keys[j * 12 + 9 + c]);
      }
      A.depth = B.depth = h[hi].depth + 1;
      h.push_back(A);
      h.push_back(B);
      h[hi].child = ca;
      if (classify(ca)) next.push_back(ca);
      if (classify(ca + 1)) next.push_back(ca + 1);
    }
    active.swap(next);
  }
  if (e != cudaSuccess) { if (err) *err = "bvh phase 1"; return (int)e; }
  // ---- phase 2
  const uint32_t nr = (uint32_t)roots.size();
  std::vector<uint32_t> local(nr, 0), local_levels(nr, 1);
  if (nr) {
    size_t base = 0;
    for (auto& R : roots) { R.base = (uint32_t)base; base += 2 * (size_t)R.count - 1; }
    chk(cudaMemcpyAsync(d_roots, roots.data(), nr * sizeof(SmallRoot), cudaMemcpyHostToDevice, st));
    k_init_roots<<<(nr + 127) / 128, 128, 0, st>>>(d_roots, nr, rec);
    ++scratch.launches;
    uint32_t cap = 1;
    for (const auto& R : roots) cap = R.count > cap ? R.count : cap;
    chk(block_attr());
    if (cap > kBlockCap) { if (err) *err = "bvh: subtree larger than the block builder's capacity"; return -9; }
    (p.bins == 2u ? k_subtree_block<true> : k_subtree_block<false>)<<<nr, 32 * kBlockWarps, block_smem(cap), st>>>(
        out_idx, in.pmin, in.pmax, in.cent, d_roots, nr, cap, p.bins, p.max_leaf, p.tlas, rec, lcnt, d_err, 0u,
        nullptr);
    ++scratch.launches;
    chk(cudaGetLastError());
    chk(cudaMemcpyAsync(local.data(), lcnt, nr * 4, cudaMemcpyDeviceToHost, st));
    chk(cudaMemcpyAsync(local_levels.data(), lcnt + nr, nr * 4, cudaMemcpyDeviceToHost, st));
  }
  int dev_error = 0;
  chk(cudaMemcpyAsync(&dev_error, d_err, 4, cudaMemcpyDeviceToHost, st));
  chk(cudaStreamSynchronize(st));
  if (e != cudaSuccess) { if (err) *err = "bvh phase 2"; return (int)e; }
  if (dev_error == -9) { if (err) *err = "bvh: internal index check failed"; return -9; }
  if (host_error || dev_error) {
    if (err) *err = "degenerate split: the reference's partition would underflow (blas.rs:114-121)";
    return -7;
  }
  // ---- numbering: descendants bottom-up (children have larger indices)
  for (size_t i = h.size(); i-- > 0;) {
    HNode& x = h[i];
    if (x.small >= 0) x.desc = local[x.small];
    else if (x.child >= 0) x.desc = 2 + h[x.child].desc + h[x.child + 1].desc;
    else x.desc = 0;
  }
  const uint64_t total_nodes = 1 + h[0].desc;
  std::vector<uint32_t> where;
  std::vector<Rec> hrec;
  std::vector<Place> places(nr);
  // top-down placement: (hnode, final index, child base)
  std::vector<std::array<uint64_t, 3>> work{{0, 0, 1}};
  while (!work.empty()) {
    const auto wv = work.back();
    work.pop_back();
    const HNode& x = h[wv[0]];
    const uint32_t fi = (uint32_t)wv[1], base = (uint32_t)wv[2];
    if (x.small >= 0) {
      places[x.small] = Place{fi, base, 0, 0};
      continue;
    }
    Rec r;
    r.lo = make_float4(x.mn[0], x.mn[1], x.mn[2], 0.0f);
    r.hi = make_float4(x.mx[0], x.mx[1], x.mx[2], 0.0f);
    if (x.child >= 0) {
      uint32_t a = base, zero = 0;
      std::memcpy(&r.lo.w, &a, 4);
      std::memcpy(&r.hi.w, &zero, 4);
      work.push_back({(uint64_t)x.child + 1, (uint64_t)base + 1, (uint64_t)base + 2 + h[x.child].desc});
      work.push_back({(uint64_t)x.child, (uint64_t)base, (uint64_t)base + 2});
    } else {
      std::memcpy(&r.lo.w, &x.first, 4);
      std::memcpy(&r.hi.w, &x.count, 4);
    }
    where.push_back(fi);
    hrec.push_back(r);
  }
  Rec* out = (Rec*)out_nodes;
  const uint32_t cap = 2 * n - 1;
  if (total_nodes > cap) { if (err) *err = "bvh: node count exceeds 2n-1"; return -9; }
  const uint32_t nh = (uint32_t)where.size();
  uint32_t* d_where = nullptr;
  Rec* d_hrec = nullptr;
  if (nh) {
    chk(pt::dev_alloc((void**)&d_where, (size_t)nh * 4));
    chk(pt::dev_alloc((void**)&d_hrec, (size_t)nh * sizeof(Rec)));
    chk(cudaMemcpyAsync(d_where, where.data(), nh * 4, cudaMemcpyHostToDevice, st));
    chk(cudaMemcpyAsync(d_hrec, hrec.data(), nh * sizeof(Rec), cudaMemcpyHostToDevice, st));
    if (e == cudaSuccess) k_emit_nodes<<<(nh + 255) / 256, 256, 0, st>>>(d_where, d_hrec, nh, out, cap, d_err);
    ++scratch.launches;
  }
  if (nr) {
    chk(cudaMemcpyAsync(d_places, places.data(), nr * sizeof(Place), cudaMemcpyHostToDevice, st));
    k_emit_small<<<nr, 128, 0, st>>>(d_roots, d_places, lcnt, rec, nr, out, cap, d_err);
    ++scratch.launches;
  }
  chk(cudaGetLastError());
  chk(cudaStreamSynchronize(st));
  if (d_where) cudaFree(d_where);
  if (d_hrec) cudaFree(d_hrec);
  if (e != cudaSuccess) { if (err) *err = "bvh emit"; return (int)e; }
  int emit_error = 0;
  chk(cudaMemcpy(&emit_error, d_err, 4, cudaMemcpyDeviceToHost));
  if (emit_error) { if (err) *err = "bvh: internal index check failed"; return -9; }
  *node_count = (uint32_t)total_nodes;
  if (levels) {
    uint32_t lv = 0;
    for (const HNode& x : h) {
      const uint32_t d = x.small >= 0 ? x.depth - 1 + local_levels[x.small] : x.depth;
      lv = d > lv ? d : lv;
    }
    *levels = lv;
  }
  return 0;
}

}  // namespace bvh
