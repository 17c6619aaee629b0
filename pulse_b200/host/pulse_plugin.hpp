// pulse_plugin.hpp -- the reference's plugin surface on top of the C ABI.
//
// The Bevy plugin of the reference (src/lib.rs:13-37, src/scene/mod.rs:38-131,
// src/path_tracer/mod.rs:35-166, src/path_tracer/node.rs:40-119,
// src/path_tracer/pt_upscaling/node.rs:29-96) restated as plain C++ types and
// systems: the same names, the same per-frame order and the same rules
// (accumulation reset on camera motion, render-target resolution, skip of
// instances whose mesh or material is not prepared, silent skip of a frame
// without a scene), with every GPU step a call of include/pulse_cuda.h.
// A host engine calls these systems once per frame in the order of
// PulsePlugin::frame.
#pragma once
#include <array>
#include <cstdint>
#include <map>
#include <optional>
#include <string>
#include <utility>
#include <vector>

#include "../../include/pulse_cuda.h"

namespace pulse {

using Mat4 = std::array<float, 16>;  // column-major, GlobalTransform::compute_matrix()
using AssetId = uint64_t;

struct UVec2 {
  uint32_t x = 0, y = 0;
  bool operator==(const UVec2& o) const { return x == o.x && y == o.y; }
};

// The StandardMaterial subset pulse reads (src/scene/mod.rs:255-262); colors
// as rgba_to_vec4 returns them.
struct StandardMaterial {
  std::array<float, 4> base_color{1, 1, 1, 1};
  std::array<float, 4> emissive{0, 0, 0, 1};
  float perceptual_roughness = 0.5f, reflectance = 0.5f, metallic = 0.0f;
};

// A mesh asset with the attributes the extraction reads (src/scene/mod.rs:376-409).
struct Mesh {
  std::vector<std::array<float, 3>> positions, normals;  // ATTRIBUTE_POSITION, ATTRIBUTE_NORMAL
  std::vector<std::array<float, 2>> uvs;                 // ATTRIBUTE_UV_0
  enum class IndexKind { None, U16, U32 } index_kind = IndexKind::None;
  std::vector<uint16_t> indices_u16;
  std::vector<uint32_t> indices_u32;
};

// Asset changes of one frame (Bevy's AssetEvent-driven extraction).
template <class T>
struct ExtractedAssets {
  std::vector<std::pair<AssetId, T>> new_or_modified;
  std::vector<AssetId> removed;
  bool empty() const { return new_or_modified.empty() && removed.empty(); }
};

// One extracted (mesh, material, transform) of the scene (src/scene/mod.rs:517-525).
struct MeshInstance {
  AssetId mesh = 0, material = 0;
  Mat4 transform{};
};

// PulsePathTracerCamera (src/path_tracer/mod.rs:100-105).
struct PulsePathTracerCamera {
  std::optional<UVec2> resolution;
  uint32_t accumulation_count = 0;
  Mat4 previous_transform{};
};

// reset_accumulation_on_movement (src/path_tracer/mod.rs:107-118): 0 when the
// camera's transform changed, else one more frame.
void reset_accumulation_on_movement(const Mat4& current_transform, PulsePathTracerCamera& camera);

// The render-target size of prepare_path_tracer_render_targets
// (src/path_tracer/mod.rs:153-156): the camera's resolution, else the view's
// physical size, else 720 x 480.
UVec2 path_tracer_resolution(const PulsePathTracerCamera& camera, std::optional<UVec2> physical_target_size);

// PulseCamera of the realtime plugin (src/pulse/mod.rs:69-73).
struct PulseCamera {
  std::optional<UVec2> resolution;
};

// Resolution of the realtime GI target (src/pulse/mod.rs:115-118): the
// camera's, else the view's physical size, else 720 x 480.
UVec2 pulse_resolution(const PulseCamera& camera, std::optional<UVec2> physical_target_size);

// PulseMaterial of prepare_material_assets (src/scene/mod.rs:255-262).
PulseMaterial to_pulse_material(const StandardMaterial& m);

// Widened index buffer of a mesh (U16 -> U32); nullopt when the mesh has none.
std::optional<std::vector<uint32_t>> mesh_indices(const Mesh& m);

// Why a mesh cannot be prepared ("" when it can): a missing POSITION, NORMAL or
// UV_0 attribute (the reference unwraps and panics), attribute lengths that
// differ, no index buffer (the reference logs and skips), or an index out of
// range.
std::string mesh_problem(const Mesh& m);

// The render world's state: context, scene, prepared assets (PulsePlugin +
// PulseScenePlugin resources).
class PulsePlugin {
 public:
  explicit PulsePlugin(int32_t device = 0, PulseBvhParams blas = {20, 8}, PulseBvhParams tlas = {2, 1});
  ~PulsePlugin();
  PulsePlugin(const PulsePlugin&) = delete;
  PulsePlugin& operator=(const PulsePlugin&) = delete;

  // prepare_extracted_mesh_assets (src/scene/mod.rs:372-448): uploads new or
  // modified meshes (BLAS on the GPU), removes removed ones.  Meshes that
  // cannot be prepared are skipped and listed in skipped_meshes().
  int32_t prepare_extracted_mesh_assets(const ExtractedAssets<Mesh>& extracted);
  // prepare_material_assets + prepare_material_data (src/scene/mod.rs:255-297):
  // when anything changed, every material gets an index in id order.
  int32_t prepare_material_data(const ExtractedAssets<StandardMaterial>& extracted);
  // prepare_mesh_instances (src/scene/mod.rs:561-697): instances whose mesh or
  // material is not prepared are skipped; the library builds the instance
  // records, lights and TLAS.  A frame whose list differs from the last one
  // only in transforms goes through pulse_instances_update (same scene).
  int32_t prepare_mesh_instances(const std::vector<MeshInstance>& instances);
  // Whether the last prepare_mesh_instances took the incremental path.
  bool last_incremental() const { return last_incremental_; }

  PulseCtx* ctx() const { return ctx_; }
  PulseScene* scene() const { return scene_; }
  bool scene_ready() const { return ready_; }
  const std::vector<AssetId>& skipped_meshes() const { return skipped_; }
  std::optional<uint32_t> material_index(AssetId id) const;
  std::string last_error() const;

 private:
  PulseCtx* ctx_ = nullptr;
  PulseScene* scene_ = nullptr;
  PulseBvhParams blas_, tlas_;
  std::map<AssetId, uint32_t> mesh_ids_;              // PulseMeshes: asset -> library mesh id
  std::map<AssetId, PulseMaterial> materials_;        // PulseMaterials
  std::map<AssetId, uint32_t> material_indices_;      // PulseMaterialIndices
  std::vector<AssetId> skipped_;
  std::vector<PulseInstanceDesc> last_;  // the instance list of the last prepared frame
  bool last_incremental_ = false;
  bool full_ = true;  // meshes changed since the last prepared frame
  bool ready_ = false;
};

// PulsePathTracerRenderTarget (src/path_tracer/mod.rs:120-166): recreated
// when the resolution changes.
class PulsePathTracerRenderTarget {
 public:
  ~PulsePathTracerRenderTarget();
  int32_t prepare(PulseCtx* ctx, UVec2 size);
  PulseTarget* texture() const { return target_; }
  uint32_t width() const { return size_.x; }
  uint32_t height() const { return size_.y; }

 private:
  PulseTarget* target_ = nullptr;
  UVec2 size_{};
};

// PulseGIRenderTarget (src/pulse/mod.rs:75-80, :94-133): the realtime GI
// output (Rgba32Float), recreated when the resolution changes.  The
// reference's PulseShadowRenderTarget is bound by the pass but never written by
// gi.wgsl, so it has no counterpart.
using PulseGIRenderTarget = PulsePathTracerRenderTarget;

// A decoded G-buffer: size.x * size.y texels in device memory (or host memory
// with on_host), e.g. from pulse_gbuffer_primary.
struct GBufferView {
  const PulseGBufferTexel* texels = nullptr;
  UVec2 size{};
  bool on_host = false;
};

// PulseNode::run (src/pulse/node.rs:38-127): the GI pass over the G-buffer
// into the target (params from pulse_default_gi_params for the reference's
// pass); returns PULSE_OK without rendering when the scene is not ready (the
// reference's silent skip).
int32_t pulse_node_run(const PulsePlugin& plugin, const GBufferView& gbuffer, PulseGIRenderTarget& target,
                       const PulseRenderParams& params);

// PulsePathTracerNode::run (src/path_tracer/node.rs:40-119): one frame into
// the target with the camera's accumulation count; returns PULSE_OK without
// rendering when the scene is not ready (the reference's silent skip).
int32_t path_tracer_node_run(const PulsePlugin& plugin, const PulseView& view, const PulsePathTracerCamera& camera,
                             PulsePathTracerRenderTarget& target, const PulseRenderParams& params);

// PulsePathTracerUpscalingNode::run (src/path_tracer/pt_upscaling/node.rs:29-96):
// the target resampled to the view (nearest, as the reference's sampler) as
// RGBA16F texels into dst (device memory, or host memory with dst_on_host).
// PulseUpscalingNode::run of the realtime plugin (src/upscaling/node.rs,
// upscaling.wgsl: the same default-sampler blit of the GI target) is this call
// on a PulseGIRenderTarget.
int32_t upscaling_node_run(const PulsePathTracerRenderTarget& target, UVec2 view_size, void* dst, bool dst_on_host);

}  // namespace pulse
