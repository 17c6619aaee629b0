// scene_prep.cu -- scene preparation kernels (see scene_prep.cuh).
#include <cfloat>

#include "pt_math.cuh"
#include "scene_prep.cuh"

namespace prep {

using namespace pt;

namespace {

__global__ void k_soup(const float* __restrict__ pos, const float* __restrict__ nrm, const float* __restrict__ uv,
                       const uint32_t* __restrict__ idx, uint32_t ntris, float4* prims, float4* tdata) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntris) return;
  const uint32_t v[3] = {idx[3 * t], idx[3 * t + 1], idx[3 * t + 2]};
  for (int k = 0; k < 3; ++k) {
    prims[3 * t + k] = make_float4(pos[3 * v[k]], pos[3 * v[k] + 1], pos[3 * v[k] + 2], 0.0f);
    tdata[5 * t + k] = make_float4(nrm[3 * v[k]], nrm[3 * v[k] + 1], nrm[3 * v[k] + 2], 0.0f);
  }
  tdata[5 * t + 3] = make_float4(uv[2 * v[0]], uv[2 * v[0] + 1], uv[2 * v[1]], uv[2 * v[1] + 1]);
  tdata[5 * t + 4] = make_float4(uv[2 * v[2]], uv[2 * v[2] + 1], 0.0f, 0.0f);
}

// 4x4 inverse by the adjugate from 2x2 minors (D. Eberly, "The Laplace
// Expansion Theorem: Computing the Determinants and Inverses of Matrices").
// Same operation order as the CPU restatement (glam's own order is not
// available offline).
__device__ void inverse4(const float* src, float* dst) {
#define A(r, c) src[(c)*4 + (r)]
  const float s0 = A(0, 0) * A(1, 1) - A(1, 0) * A(0, 1);
  const float s1 = A(0, 0) * A(1, 2) - A(1, 0) * A(0, 2);
  const float s2 = A(0, 0) * A(1, 3) - A(1, 0) * A(0, 3);
  const float s3 = A(0, 1) * A(1, 2) - A(1, 1) * A(0, 2);
  const float s4 = A(0, 1) * A(1, 3) - A(1, 1) * A(0, 3);
  const float s5 = A(0, 2) * A(1, 3) - A(1, 2) * A(0, 3);
  const float c5 = A(2, 2) * A(3, 3) - A(3, 2) * A(2, 3);
  const float c4 = A(2, 1) * A(3, 3) - A(3, 1) * A(2, 3);
  const float c3 = A(2, 1) * A(3, 2) - A(3, 1) * A(2, 2);
  const float c2 = A(2, 0) * A(3, 3) - A(3, 0) * A(2, 3);
  const float c1 = A(2, 0) * A(3, 2) - A(3, 0) * A(2, 2);
  const float c0 = A(2, 0) * A(3, 1) - A(3, 0) * A(2, 1);
  const float det = s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
  const float id = 1.0f / det;
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
#undef A
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) dst[c * 4 + r] = b[r][c];
}

__global__ void k_instances(const InstanceIn* __restrict__ in, uint32_t n, const float4* __restrict__ blas_nodes,
                            float4* inst_out, float* bounds9, const uint32_t* __restrict__ slot) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const InstanceIn x = in[j];
  const uint32_t i = slot ? slot[j] : j;
  float inv[16];
  inverse4(x.object_world, inv);
  float4* o = inst_out + (size_t)i * 10;
  for (int c = 0; c < 4; ++c) {
    o[c] = make_float4(x.object_world[4 * c], x.object_world[4 * c + 1], x.object_world[4 * c + 2], x.object_world[4 * c + 3]);
    o[4 + c] = make_float4(inv[4 * c], inv[4 * c + 1], inv[4 * c + 2], inv[4 * c + 3]);
  }
  o[8] = make_float4(__uint_as_float(x.triangle_offset), __uint_as_float(x.triangle_count),
                     __uint_as_float(x.index_offset), __uint_as_float(x.node_offset));
  o[9] = make_float4(__uint_as_float(x.material_index), 0.0f, 0.0f, 0.0f);
  // World bounds of the root box (src/scene/mod.rs:625-658).
  const float4 lo = blas_nodes[2 * (size_t)x.node_offset], hi = blas_nodes[2 * (size_t)x.node_offset + 1];
  const M4 m{o[0], o[1], o[2], o[3]};
  const float3 corners[8] = {v3(lo.x, lo.y, lo.z), v3(hi.x, lo.y, lo.z), v3(lo.x, hi.y, lo.z), v3(lo.x, lo.y, hi.z),
                             v3(hi.x, hi.y, lo.z), v3(lo.x, hi.y, hi.z), v3(hi.x, lo.y, hi.z), v3(hi.x, hi.y, hi.z)};
  float3 wmin = v3(FLT_MAX, FLT_MAX, FLT_MAX), wmax = v3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
  float3 tc[8];
  for (int c = 0; c < 8; ++c) tc[c] = transform_position(m, corners[c]);
  for (int c = 0; c < 8; ++c) wmin = vmin(wmin, tc[c]);
  for (int c = 0; c < 8; ++c) wmax = vmax(wmax, tc[c]);
  const float3 center = add(wmin, muls(sub(wmax, wmin), 0.5f));
  float* b = bounds9 + (size_t)i * 9;
  b[0] = wmin.x; b[1] = wmin.y; b[2] = wmin.z;
  b[3] = wmax.x; b[4] = wmax.y; b[5] = wmax.z;
  b[6] = center.x; b[7] = center.y; b[8] = center.z;
}

__global__ void k_light_cdfs(const LightIn* __restrict__ lights, uint32_t n, const float4* __restrict__ prims,
                             float* tri_cdfs, float* mesh_areas) {
  const uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= n) return;
  const LightIn L = lights[l];
  float* cdf = tri_cdfs + L.cdf_offset;
  for (uint32_t t = 0; t < L.triangle_count; ++t) {
    const float4* p = prims + (size_t)(L.triangle_offset + t) * 3;
    const float3 p0 = xyz(p[0]), p1 = xyz(p[1]), p2 = xyz(p[2]);
    const float a = length(sub(p1, p0));
    const float b = length(sub(p2, p0));
    const float c = length(sub(p2, p1));
    const float s = 0.5f * (a + b + c);
    cdf[t] = sqrtf(s * (s - a) * (s - b) * (s - c));
  }
  float total = 0.0f;
  for (uint32_t t = 0; t < L.triangle_count; ++t) total = total + cdf[t];
  float prev = 0.0f;
  for (uint32_t t = 0; t < L.triangle_count; ++t) {
    const float cur = prev + cdf[t] / total;
    cdf[t] = cur;
    prev = cur;
  }
  mesh_areas[l] = total;
}

__global__ void k_strength_cdf(const LightIn* __restrict__ lights, uint32_t n, const float4* __restrict__ materials,
                               float* strength_cdf) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  float total = 0.0f;
  for (uint32_t l = 0; l < n; ++l) {
    const float3 em = xyz(materials[3 * (size_t)lights[l].material + 1]);
    const float s = dot(em, em);
    strength_cdf[l] = s;
    total = total + s;
  }
  float prev = 0.0f;
  for (uint32_t l = 0; l < n; ++l) {
    const float cur = prev + strength_cdf[l] / total;
    strength_cdf[l] = cur;
    prev = cur;
  }
}

}  // namespace

cudaError_t soup(const float* pos, const float* nrm, const float* uv, const uint32_t* idx, uint32_t ntris,
                 float4* prims, float4* tdata, cudaStream_t st) {
  if (!ntris) return cudaSuccess;
  k_soup<<<(ntris + 255) / 256, 256, 0, st>>>(pos, nrm, uv, idx, ntris, prims, tdata);
  return cudaGetLastError();
}

cudaError_t instances(const InstanceIn* in, uint32_t n, const float4* blas_nodes, float4* inst_out, float* bounds9,
                      cudaStream_t st, const uint32_t* slot) {
  if (!n) return cudaSuccess;
  k_instances<<<(n + 127) / 128, 128, 0, st>>>(in, n, blas_nodes, inst_out, bounds9, slot);
  return cudaGetLastError();
}

cudaError_t lights(const LightIn* lights, uint32_t n_lights, const float4* prims, const float4* materials,
                   float* tri_cdfs, float* mesh_areas, float* strength_cdf, cudaStream_t st) {
  if (!n_lights) return cudaSuccess;
  k_light_cdfs<<<(n_lights + 63) / 64, 64, 0, st>>>(lights, n_lights, prims, tri_cdfs, mesh_areas);
  k_strength_cdf<<<1, 32, 0, st>>>(lights, n_lights, materials, strength_cdf);
  return cudaGetLastError();
}

}  // namespace prep
