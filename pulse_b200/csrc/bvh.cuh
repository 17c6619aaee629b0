// bvh.cuh -- binned-SAH BVH build on the device, bit-identical to the
// reference's recursive CPU builders (src/scene/blas.rs:44-314 for BLAS,
// src/scene/tlas.rs:29-263 for the TLAS).
//
// Why the result can be bit-identical: every floating-point quantity of the
// reference build is either a per-primitive formula (centroid, bin index), a
// min/max reduction (exact and order-independent once min/max is a lattice --
// NaN-ignoring, -0 below +0), an integer count, or a short sequential sweep over
// <= 32 bins that is evaluated here in the reference's order.  The two-pointer
// partition (blas.rs:113-122) is an unstable permutation; it is reproduced in
// closed form: with m left elements, F = [0, m) and B = [m, n), the t-th right
// element of F goes to b_{t-1} - 1 (b_0 = n, b_s = position of the s-th left
// element of B counted from the end), the t-th left element of B from the end
// goes to the t-th right position of F, a right element at m goes to b_r - 1,
// right elements after m move down by one, left elements of F stay.  Node
// numbering is the recursion's: a node's children are allocated as a pair when
// it is split, the A subtree before the B subtree, so the final index of every
// node follows from subtree sizes (children base of A = base + 2, of B =
// base + 2 + 2 * interior nodes under A).
#pragma once
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

namespace bvh {

struct Params {
  uint32_t bins;      // 2..32
  uint32_t max_leaf;  // leaf when count <= max_leaf
  uint32_t tlas;      // 0 BLAS (triangles), 1 TLAS (instance bounds)
};

// Device inputs, indexed by primitive id: node box (pmin, pmax) and centroid.
// BLAS: pmin/pmax = lattice min/max of the three vertices (from +/-FLT_MAX),
//       centroid = pmin + 0.5 * (pmax - pmin) (blas.rs:47-59).
// TLAS: pmin/pmax = bounds_min / bounds_max, centroid = center (tlas.rs via
//       src/scene/mod.rs:625-680).
struct Input {
  const float4* pmin;
  const float4* pmax;
  const float4* cent;
  uint32_t n;
};

// Scratch owned by the caller between builds (grown on demand).
struct Scratch {
  void* buf = nullptr;
  size_t bytes = 0;
  uint64_t launches = 0;  // kernels launched by build() through this scratch
  void release();
};

// Builds into out_nodes (capacity 2n-1 nodes of 8 words) and out_idx (n).
// Returns 0, -7 (the reference would panic: partition underflow) or a CUDA
// error code (> 0); *node_count receives the number of nodes and *levels (if
// given) the number of levels of the tree (root alone: 1).
int build(const Input& in, const Params& p, uint32_t* out_nodes, uint32_t* out_idx, uint32_t* node_count,
          Scratch& scratch, cudaStream_t st, std::string* err, uint32_t* levels = nullptr);

// The whole tree of n <= direct_max() elements in one launch of one block, no
// host round trip (the per-frame TLAS): same tree as build().  meta (4 device
// words) receives the node count, the levels and an error code (0, -7 where
// the reference's partition would underflow, -9 on an internal index check);
// the caller reads it after the stream's work.  out_idx needs no initial
// contents.
uint32_t direct_max();
cudaError_t build_direct(const Input& in, const Params& p, uint32_t* out_nodes, uint32_t* out_idx, uint32_t* meta,
                         cudaStream_t st);

// Per-primitive inputs from std430 primitives (3 float4 per triangle).
cudaError_t prep_triangles(const float4* prims, uint32_t n, float4* pmin, float4* pmax, float4* cent,
                           cudaStream_t st);
// Per-primitive inputs from instance bounds (n x 9 floats: min, max, center).
cudaError_t prep_instances(const float* bounds9, uint32_t n, float4* pmin, float4* pmax, float4* cent,
                           cudaStream_t st);

}  // namespace bvh
