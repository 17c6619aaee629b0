// pulse_plugin.cpp -- see pulse_plugin.hpp.
#include "pulse_plugin.hpp"

#include <cstring>

namespace pulse {

void reset_accumulation_on_movement(const Mat4& current_transform, PulsePathTracerCamera& camera) {
  if (current_transform != camera.previous_transform) {  // float comparison, as GlobalTransform's PartialEq
    camera.accumulation_count = 0;
  } else {
    camera.accumulation_count += 1;
  }
  camera.previous_transform = current_transform;
}

UVec2 path_tracer_resolution(const PulsePathTracerCamera& camera, std::optional<UVec2> physical_target_size) {
  if (camera.resolution) return *camera.resolution;
  if (physical_target_size) return *physical_target_size;
  return UVec2{720, 480};
}

UVec2 pulse_resolution(const PulseCamera& camera, std::optional<UVec2> physical_target_size) {
  if (camera.resolution) return *camera.resolution;
  if (physical_target_size) return *physical_target_size;
  return UVec2{720, 480};
}

PulseMaterial to_pulse_material(const StandardMaterial& m) {
  PulseMaterial p{};
  std::memcpy(p.base_color, m.base_color.data(), 16);
  std::memcpy(p.emissive, m.emissive.data(), 16);
  p.perceptual_roughness = m.perceptual_roughness;
  p.reflectance = m.reflectance;
  p.metallic = m.metallic;
  return p;
}

std::optional<std::vector<uint32_t>> mesh_indices(const Mesh& m) {
  switch (m.index_kind) {
    case Mesh::IndexKind::U16: return std::vector<uint32_t>(m.indices_u16.begin(), m.indices_u16.end());
    case Mesh::IndexKind::U32: return m.indices_u32;
    default: return std::nullopt;
  }
}

std::string mesh_problem(const Mesh& m) {
  if (m.positions.empty()) return "mesh has no POSITION attribute";
  if (m.normals.empty()) return "mesh has no NORMAL attribute";
  if (m.uvs.empty()) return "mesh has no UV_0 attribute";
  if (m.normals.size() != m.positions.size() || m.uvs.size() != m.positions.size())
    return "mesh attributes differ in length";
  const auto idx = mesh_indices(m);
  if (!idx) return "Cannot load mesh with no index buffer.";
  if (idx->size() < 3) return "mesh has no triangle";
  for (uint32_t i : *idx)
    if (i >= m.positions.size()) return "mesh index out of range";
  return "";
}

PulsePlugin::PulsePlugin(int32_t device, PulseBvhParams blas, PulseBvhParams tlas) : blas_(blas), tlas_(tlas) {
  if (pulse_ctx_create(device, &ctx_) != PULSE_OK) {
    ctx_ = nullptr;
    return;
  }
  if (pulse_scene_create(ctx_, &scene_) != PULSE_OK) scene_ = nullptr;
}

PulsePlugin::~PulsePlugin() {
  if (scene_) pulse_scene_destroy(scene_);
  if (ctx_) pulse_ctx_destroy(ctx_);
}

std::string PulsePlugin::last_error() const { return ctx_ ? pulse_last_error(ctx_) : "no CUDA device"; }

std::optional<uint32_t> PulsePlugin::material_index(AssetId id) const {
  const auto it = material_indices_.find(id);
  if (it == material_indices_.end()) return std::nullopt;
  return it->second;
}

int32_t PulsePlugin::prepare_extracted_mesh_assets(const ExtractedAssets<Mesh>& extracted) {
  if (!scene_) return PULSE_ERR_NO_DEVICE;
  for (const auto& [id, mesh] : extracted.new_or_modified) {
    if (!mesh_problem(mesh).empty()) {
      skipped_.push_back(id);
      continue;
    }
    const std::vector<uint32_t> idx = *mesh_indices(mesh);
    uint32_t mesh_id = 0;
    const int32_t rc = pulse_mesh_upload(scene_, &mesh.positions[0][0], &mesh.normals[0][0], &mesh.uvs[0][0],
                                         (uint32_t)mesh.positions.size(), idx.data(), (uint32_t)idx.size(), &blas_,
                                         &mesh_id);
    if (rc != PULSE_OK) return rc;
    full_ = true;  // the concatenated mesh data changes: the next instances are prepared in full
    const auto old = mesh_ids_.find(id);
    if (old != mesh_ids_.end()) pulse_mesh_remove(scene_, old->second);
    mesh_ids_[id] = mesh_id;
  }
  for (AssetId id : extracted.removed) {
    const auto it = mesh_ids_.find(id);
    if (it == mesh_ids_.end()) continue;
    full_ = true;
    pulse_mesh_remove(scene_, it->second);
    mesh_ids_.erase(it);
  }
  return PULSE_OK;
}

int32_t PulsePlugin::prepare_material_data(const ExtractedAssets<StandardMaterial>& extracted) {
  if (!scene_) return PULSE_ERR_NO_DEVICE;
  for (const auto& [id, m] : extracted.new_or_modified) materials_[id] = to_pulse_material(m);
  for (AssetId id : extracted.removed) materials_.erase(id);
  if (extracted.empty()) return PULSE_OK;  // material data is the same as last frame's
  std::vector<PulseMaterial> data;
  material_indices_.clear();
  for (const auto& [id, m] : materials_) {
    material_indices_[id] = (uint32_t)data.size();
    data.push_back(m);
  }
  // Instances of the last frame may use indices the new list no longer has:
  // they are rebuilt by the next prepare_mesh_instances.
  ready_ = false;
  return pulse_materials_set(scene_, data.empty() ? nullptr : data.data(), (uint32_t)data.size()) == PULSE_OK
             ? PULSE_OK
             : PULSE_ERR_INVALID_ARG;
}

int32_t PulsePlugin::prepare_mesh_instances(const std::vector<MeshInstance>& instances) {
  if (!scene_) return PULSE_ERR_NO_DEVICE;
  std::vector<PulseInstanceDesc> descs;
  for (const MeshInstance& in : instances) {
    const auto mi = mesh_ids_.find(in.mesh);
    const auto ma = material_indices_.find(in.material);
    if (mi == mesh_ids_.end() || ma == material_indices_.end()) continue;
    PulseInstanceDesc d{};
    std::memcpy(d.object_world, in.transform.data(), 64);
    d.mesh_id = mi->second;
    d.material_index = ma->second;
    descs.push_back(d);
  }
  // The reference rebuilds everything every frame; when only transforms moved
  // since the last frame the result is the same with pulse_instances_update.
  bool same = ready_ && !full_ && descs.size() == last_.size();
  std::vector<uint32_t> moved;
  std::vector<float> worlds;
  for (size_t i = 0; same && i < descs.size(); ++i) {
    same = descs[i].mesh_id == last_[i].mesh_id && descs[i].material_index == last_[i].material_index;
    if (same && std::memcmp(descs[i].object_world, last_[i].object_world, 64) != 0) {
      moved.push_back((uint32_t)i);
      worlds.insert(worlds.end(), descs[i].object_world, descs[i].object_world + 16);
    }
  }
  int32_t rc = PULSE_OK;
  if (same) {
    last_incremental_ = true;
    if (!moved.empty()) rc = pulse_instances_update(scene_, moved.data(), worlds.data(), (uint32_t)moved.size(), &tlas_);
  } else {
    last_incremental_ = false;
    rc = pulse_instances_set(scene_, descs.empty() ? nullptr : descs.data(), (uint32_t)descs.size(), &tlas_);
  }
  ready_ = rc == PULSE_OK;
  if (ready_) {
    last_ = std::move(descs);
    full_ = false;
  }
  return rc;
}

PulsePathTracerRenderTarget::~PulsePathTracerRenderTarget() {
  if (target_) pulse_target_destroy(target_);
}

int32_t PulsePathTracerRenderTarget::prepare(PulseCtx* ctx, UVec2 size) {
  if (target_ && size == size_) return PULSE_OK;
  if (target_) pulse_target_destroy(target_);
  target_ = nullptr;
  const int32_t rc = pulse_target_create(ctx, size.x, size.y, &target_);
  if (rc == PULSE_OK) size_ = size;
  else target_ = nullptr;
  return rc;
}

int32_t path_tracer_node_run(const PulsePlugin& plugin, const PulseView& view, const PulsePathTracerCamera& camera,
                             PulsePathTracerRenderTarget& target, const PulseRenderParams& params) {
  if (!plugin.scene_ready() || !target.texture()) return PULSE_OK;
  const int32_t rc = pulse_render_forward(plugin.scene(), &view, target.texture(), camera.accumulation_count, &params);
  return rc == PULSE_ERR_NOT_READY ? PULSE_OK : rc;
}

int32_t pulse_node_run(const PulsePlugin& plugin, const GBufferView& gbuffer, PulseGIRenderTarget& target,
                       const PulseRenderParams& params) {
  if (!plugin.scene_ready() || !target.texture()) return PULSE_OK;
  const int32_t rc = pulse_render_gi(plugin.scene(), gbuffer.texels, gbuffer.size.x, gbuffer.size.y,
                                     gbuffer.on_host ? 1u : 0u, target.texture(), &params);
  return rc == PULSE_ERR_NOT_READY ? PULSE_OK : rc;
}

int32_t upscaling_node_run(const PulsePathTracerRenderTarget& target, UVec2 view_size, void* dst, bool dst_on_host) {
  if (!target.texture()) return PULSE_OK;
  return pulse_target_resample(target.texture(), view_size.x, view_size.y, 0, dst, dst_on_host ? 1u : 0u);
}

}  // namespace pulse
