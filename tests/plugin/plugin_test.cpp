// Test driver of the C++ plugin surface (pulse_b200/host/pulse_plugin.hpp).
//   plugin_test cpu                      the systems' rules, no device needed
//   plugin_test render <scene> <out>     a scene file written by tests/test_plugin_gpu.py rendered frame by
//                                        frame through the plugin systems; writes the target's texels and
//                                        the upscaled RGBA16F image
//   plugin_test gi <scene> <out>         the same frames through the realtime plugin: primary-hit G-buffer,
//                                        the GI node into the GI target, the upscaling node
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "../../pulse_b200/host/pulse_plugin.hpp"

using namespace pulse;

static int failures = 0;
#define CHECK(c)                                                        \
  do {                                                                  \
    if (!(c)) {                                                         \
      std::fprintf(stderr, "check failed: %s (line %d)\n", #c, __LINE__); \
      ++failures;                                                       \
    }                                                                   \
  } while (0)

static Mat4 translation(float x, float y, float z) {
  Mat4 m{};
  m[0] = m[5] = m[10] = m[15] = 1.0f;
  m[12] = x; m[13] = y; m[14] = z;
  return m;
}

static int cpu_tests() {
  // reset_accumulation_on_movement: 0 on motion, +1 otherwise (src/path_tracer/mod.rs:107-118)
  PulsePathTracerCamera cam;
  cam.previous_transform = translation(0, 0, 0);
  const Mat4 a = translation(0, 0, 3), b = translation(0, 1, 3);
  reset_accumulation_on_movement(a, cam);
  CHECK(cam.accumulation_count == 0);
  reset_accumulation_on_movement(a, cam);
  CHECK(cam.accumulation_count == 1);
  reset_accumulation_on_movement(a, cam);
  CHECK(cam.accumulation_count == 2);
  reset_accumulation_on_movement(b, cam);
  CHECK(cam.accumulation_count == 0);
  Mat4 c = b;
  c[12] = -0.0f;  // -0 == +0: not a motion
  reset_accumulation_on_movement(c, cam);
  CHECK(cam.accumulation_count == 1);
  // render-target resolution (src/path_tracer/mod.rs:153-156)
  PulsePathTracerCamera r;
  CHECK((path_tracer_resolution(r, std::nullopt) == UVec2{720, 480}));
  CHECK((path_tracer_resolution(r, UVec2{1920, 1080}) == UVec2{1920, 1080}));
  r.resolution = UVec2{320, 200};
  CHECK((path_tracer_resolution(r, UVec2{1920, 1080}) == UVec2{320, 200}));
  // realtime GI target resolution (src/pulse/mod.rs:115-118)
  PulseCamera pc;
  CHECK((pulse_resolution(pc, std::nullopt) == UVec2{720, 480}));
  CHECK((pulse_resolution(pc, UVec2{1280, 720}) == UVec2{1280, 720}));
  pc.resolution = UVec2{64, 48};
  CHECK((pulse_resolution(pc, UVec2{1280, 720}) == UVec2{64, 48}));
  // StandardMaterial subset -> PulseMaterial (src/scene/mod.rs:255-262)
  StandardMaterial sm;
  sm.base_color = {0.1f, 0.2f, 0.3f, 0.4f};
  sm.emissive = {5.0f, 6.0f, 7.0f, 1.0f};
  sm.perceptual_roughness = 0.25f;
  sm.reflectance = 0.75f;
  sm.metallic = 1.0f;
  const PulseMaterial pm = to_pulse_material(sm);
  CHECK(pm.base_color[2] == 0.3f && pm.emissive[1] == 6.0f && pm.perceptual_roughness == 0.25f &&
        pm.reflectance == 0.75f && pm.metallic == 1.0f);
  // index buffers and mesh checks (src/scene/mod.rs:376-409)
  Mesh m;
  m.positions = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}};
  m.normals = {{0, 0, 1}, {0, 0, 1}, {0, 0, 1}};
  m.uvs = {{0, 0}, {1, 0}, {0, 1}};
  CHECK(mesh_problem(m) == "Cannot load mesh with no index buffer.");
  m.index_kind = Mesh::IndexKind::U16;
  m.indices_u16 = {0, 1, 2};
  CHECK(mesh_problem(m).empty());
  const auto wide = mesh_indices(m);
  CHECK(wide && wide->size() == 3 && (*wide)[2] == 2u);
  m.indices_u16 = {0, 1, 3};
  CHECK(mesh_problem(m) == "mesh index out of range");
  Mesh no_normals = m;
  no_normals.normals.clear();
  CHECK(mesh_problem(no_normals) == "mesh has no NORMAL attribute");
  Mesh no_uv = m;
  no_uv.uvs.clear();
  CHECK(mesh_problem(no_uv) == "mesh has no UV_0 attribute");
  if (failures) return 1;
  std::printf("cpu ok\n");
  return 0;
}

template <class T>
static T rd(std::ifstream& f) {
  T v;
  f.read(reinterpret_cast<char*>(&v), sizeof(T));
  return v;
}
template <class T>
static void rdv(std::ifstream& f, T* p, size_t n) {
  f.read(reinterpret_cast<char*>(p), sizeof(T) * n);
}

static int render(const char* scene_path, const char* out_path, bool gi) {
  std::ifstream f(scene_path, std::ios::binary);
  if (!f) return 2;
  const uint32_t bins = rd<uint32_t>(f), leaf = rd<uint32_t>(f);
  PulsePlugin plugin(0, PulseBvhParams{bins, leaf}, PulseBvhParams{2, 1});
  if (!plugin.ctx()) return 3;
  ExtractedAssets<Mesh> meshes;
  const uint32_t nm = rd<uint32_t>(f);
  for (uint32_t i = 0; i < nm; ++i) {
    const uint32_t nv = rd<uint32_t>(f), ni = rd<uint32_t>(f), kind = rd<uint32_t>(f);
    Mesh m;
    m.positions.resize(nv);
    m.normals.resize(nv);
    m.uvs.resize(nv);
    rdv(f, &m.positions[0][0], nv * 3);
    rdv(f, &m.normals[0][0], nv * 3);
    rdv(f, &m.uvs[0][0], nv * 2);
    if (kind == 1) {
      m.index_kind = Mesh::IndexKind::U16;
      m.indices_u16.resize(ni);
      rdv(f, m.indices_u16.data(), ni);
    } else {
      m.index_kind = Mesh::IndexKind::U32;
      m.indices_u32.resize(ni);
      rdv(f, m.indices_u32.data(), ni);
    }
    meshes.new_or_modified.emplace_back(i + 1, std::move(m));
  }
  ExtractedAssets<StandardMaterial> materials;
  const uint32_t nmat = rd<uint32_t>(f);
  for (uint32_t i = 0; i < nmat; ++i) {
    StandardMaterial sm;
    rdv(f, sm.base_color.data(), 4);
    rdv(f, sm.emissive.data(), 4);
    sm.perceptual_roughness = rd<float>(f);
    sm.reflectance = rd<float>(f);
    sm.metallic = rd<float>(f);
    materials.new_or_modified.emplace_back(i + 1, sm);
  }
  std::vector<MeshInstance> instances(rd<uint32_t>(f));
  for (MeshInstance& in : instances) {
    in.mesh = rd<uint32_t>(f) + 1;
    in.material = rd<uint32_t>(f) + 1;
    rdv(f, in.transform.data(), 16);
  }
  PulseView view{};
  rdv(f, view.inverse_view_proj, 16);
  rdv(f, view.world_position, 3);
  const uint32_t W = rd<uint32_t>(f), H = rd<uint32_t>(f), frames = rd<uint32_t>(f);
  PulseRenderParams params;
  pulse_default_params(&params);
  params.nee_mode = rd<uint32_t>(f);
  params.max_depth = rd<uint32_t>(f);
  params.light_pick = rd<uint32_t>(f);
  params.quirks = rd<uint32_t>(f);
  const uint32_t up_w = rd<uint32_t>(f), up_h = rd<uint32_t>(f);
  if (!f) return 4;
  // optional animation: (frame, instance, transform) rows applied before that frame
  struct Move { uint32_t frame, instance; Mat4 transform; };
  const uint32_t n_moves = rd<uint32_t>(f);
  if (!f || n_moves > 4096) return 4;
  std::vector<Move> moves(n_moves);
  for (Move& mv : moves) {
    mv.frame = rd<uint32_t>(f);
    mv.instance = rd<uint32_t>(f);
    rdv(f, mv.transform.data(), 16);
    if (!f || mv.instance >= instances.size()) return 4;
  }
  uint32_t incremental = 0;
  // frame loop: the render world's systems in the reference's order
  PulsePathTracerCamera camera;
  camera.resolution = UVec2{W, H};
  camera.previous_transform = translation(1e9f, 0, 0);  // the first frame counts as a motion
  const Mat4 camera_transform = translation(0, 0, 3);
  PulsePathTracerRenderTarget target;
  PulseCamera gi_camera;
  gi_camera.resolution = UVec2{W, H};
  PulseRenderParams gi_params;
  pulse_default_gi_params(&gi_params);
  gi_params.quirks = params.quirks;
  std::vector<PulseGBufferTexel> gbuffer((size_t)W * H);
  const ExtractedAssets<Mesh> no_meshes;
  const ExtractedAssets<StandardMaterial> no_materials;
  for (uint32_t k = 0; k < frames; ++k) {
    if (plugin.prepare_extracted_mesh_assets(k == 0 ? meshes : no_meshes) != PULSE_OK) return 5;
    if (plugin.prepare_material_data(k == 0 ? materials : no_materials) != PULSE_OK) return 6;
    for (const Move& mv : moves)
      if (mv.frame == k) instances[mv.instance].transform = mv.transform;
    if (plugin.prepare_mesh_instances(instances) != PULSE_OK) return 7;
    incremental += plugin.last_incremental() ? 1 : 0;
    if (gi) {
      const UVec2 res = pulse_resolution(gi_camera, std::nullopt);
      if (target.prepare(plugin.ctx(), res) != PULSE_OK) return 8;
      if (pulse_gbuffer_primary(plugin.scene(), &view, res.x, res.y, &params, gbuffer.data(), 1) != PULSE_OK) return 12;
      if (pulse_node_run(plugin, GBufferView{gbuffer.data(), res, true}, target, gi_params) != PULSE_OK) return 9;
      continue;
    }
    reset_accumulation_on_movement(camera_transform, camera);
    if (target.prepare(plugin.ctx(), path_tracer_resolution(camera, std::nullopt)) != PULSE_OK) return 8;
    if (path_tracer_node_run(plugin, view, camera, target, params) != PULSE_OK) return 9;
  }
  std::vector<float> img((size_t)W * H * 4);
  if (pulse_target_download(target.texture(), img.data()) != PULSE_OK) return 10;
  std::vector<uint16_t> up((size_t)up_w * up_h * 4);
  if (upscaling_node_run(target, UVec2{up_w, up_h}, up.data(), true) != PULSE_OK) return 11;
  std::ofstream o(out_path, std::ios::binary);
  o.write(reinterpret_cast<const char*>(img.data()), img.size() * 4);
  o.write(reinterpret_cast<const char*>(up.data()), up.size() * 2);
  std::printf("render ok %u frames, accumulation_count %u, incremental %u\n", frames, camera.accumulation_count,
              incremental);
  return 0;
}

int main(int argc, char** argv) {
  if (argc >= 2 && std::string(argv[1]) == "cpu") return cpu_tests();
  if (argc >= 4 && std::string(argv[1]) == "render") return render(argv[2], argv[3], false);
  if (argc >= 4 && std::string(argv[1]) == "gi") return render(argv[2], argv[3], true);
  std::fprintf(stderr, "usage: plugin_test cpu | render <scene> <out> | gi <scene> <out>\n");
  return 2;
}
