// scene_prep.cuh -- device side of the reference's scene preparation systems.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace prep {

// prepare_extracted_mesh_assets (src/scene/mod.rs:410-424): triangle soup of
// positions and of normals/UVs through the index buffer (copies only).
cudaError_t soup(const float* pos, const float* nrm, const float* uv, const uint32_t* idx, uint32_t ntris,
                 float4* prims, float4* tdata, cudaStream_t st);

struct InstanceIn {
  float object_world[16];
  uint32_t triangle_offset, triangle_count, index_offset, node_offset, material_index, pad[3];
};

// prepare_mesh_instances (src/scene/mod.rs:561-681) per instance: the 160 B
// record with the inverse transform, and the world bounds of the BLAS root
// (8 transformed corners) with their centre -> bounds9.  With `slot`, input i
// writes record and bounds slot[i] (an incremental update of some instances).
cudaError_t instances(const InstanceIn* in, uint32_t n, const float4* blas_nodes, float4* inst_out, float* bounds9,
                      cudaStream_t st, const uint32_t* slot = nullptr);

struct LightIn { uint32_t instance, triangle_offset, triangle_count, cdf_offset, material; };

// create_triangle_area_cdf / create_emission_strength_cdf (src/scene/mod.rs:700-742),
// one thread per light (sequential sums in the reference's order).
cudaError_t lights(const LightIn* lights, uint32_t n_lights, const float4* prims, const float4* materials,
                   float* tri_cdfs, float* mesh_areas, float* strength_cdf, cudaStream_t st);

}  // namespace prep
