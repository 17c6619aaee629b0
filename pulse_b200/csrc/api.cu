// api.cu -- the extern "C" entry points declared in include/pulse_cuda.h.
//
// Host side of the drop-in boundary: contexts, scenes (device copies of the
// scene bind group plus derived layouts), render targets, validation of
// untrusted scene buffers before any kernel reads them, and launches.
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/pulse_cuda.h"
#include "bvh.cuh"
#include "dev_alloc.h"
#include "kernels.h"
#include "wavefront.h"
#include "adjoint.h"
#include "scene_prep.cuh"

namespace pt {
namespace {
std::atomic<uint32_t> g_fail_allocs{0};  // armed by pulse_debug_fail_allocations
}
cudaError_t dev_alloc(void** p, size_t bytes) {
  uint32_t n = g_fail_allocs.load();
  while (n > 0 && !g_fail_allocs.compare_exchange_weak(n, n - 1)) {
  }
  if (n > 0) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(p, bytes);
}
}  // namespace pt

struct DevBufC {
  void* p = nullptr;
  size_t bytes = 0;
};

struct PulseCtx {
  int device = 0;
  DevBufC wf;  // wavefront path buffers (grown on demand)
  DevBufC gstage;  // device staging of host G-buffers (grown on demand)
  cudaStream_t stream = nullptr;  // current stream (own or caller's)
  cudaStream_t own_stream = nullptr;
  std::string err;
  pt::Counters* d_counters = nullptr;
  PulseStats stats{};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool timed = false;                     // ev0/ev1 bracket the last render
  cudaGraphExec_t batch_exec = nullptr;   // last batched frame, updated in place
  // Pipelined frames (pulse_ctx_set_pipeline(ctx, 2)): pulse_render_forward
  // traces on lane[i], alternating, each lane with its own path buffers, so a
  // frame's first launches can fill the SMs its predecessor's draining
  // launches leave idle.  lane_done[i] follows the last frame on lane i;
  // lane_pending[i]: the context's stream has not waited for it yet.
  uint32_t pipeline = 1;
  cudaStream_t lane[2] = {nullptr, nullptr};
  DevBufC lane_wf[2];
  cudaEvent_t lane_done[2] = {nullptr, nullptr};
  cudaEvent_t ev_fork = nullptr;
  bool lane_pending[2] = {false, false};
  int next_lane = 0;
};

namespace {

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

int32_t set_err(PulseCtx* ctx, int32_t code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}
int32_t cuda_err(PulseCtx* ctx, cudaError_t e, const char* what) {
  if (e == cudaErrorMemoryAllocation) return set_err(ctx, PULSE_ERR_OOM, std::string(what) + ": out of device memory");
  return set_err(ctx, PULSE_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// The context's stream waits for the pipelined frames still in flight on the
// lanes: every entry point except the pipelined render, the double-buffered
// instance update and the asynchronous download calls this first, so that
// whatever it reads, writes or frees is used by no running frame.
void quiesce(PulseCtx* ctx) {
  for (int i = 0; i < 2; ++i)
    if (ctx->lane_pending[i]) {
      cudaStreamWaitEvent(ctx->stream, ctx->lane_done[i], 0);
      ctx->lane_pending[i] = false;
    }
}

}  // namespace

struct MeshRec {
  uint32_t id = 0, ntris = 0, node_count = 0, levels = 1;
  bool alive = false;
  DevBuf prims, tdata, nodes, idx;
};

struct PulseScene {
  PulseCtx* ctx = nullptr;
  bool ready = false;
  // The 13 buffers of the bind group (device) and their row counts.
  PulseSceneBuffers counts{};
  DevBuf primitives, triangle_data, triangle_indices, blas_nodes, tlas_nodes, instance_indices, instances,
      materials, strength_cdf, tri_cdfs, mesh_areas, light_indices;
  // Derived layouts.
  DevBuf inst_light, tri_bvh;
  bool tri_bvh_current = false;  // tri_bvh gathered from the current primitives and triangle_indices
  pt::DevScene dev{};
  // Scene-preparation path.
  std::vector<MeshRec> meshes;
  std::vector<std::array<uint32_t, 4>> mesh_table;  // per mesh id: tri_off, count, idx_off, node_off (~0u if none)
  bool meshes_dirty = true;
  std::vector<PulseMaterial> host_materials;
  // Inputs of the last successful pulse_instances_set (the light list follows
  // the materials, so a material change re-runs the instance preparation).
  bool prepped = false;
  std::vector<PulseInstanceDesc> last_inst;
  PulseBvhParams last_tlas{2, 1};
  uint32_t materials_needed = 0;  // 1 + the largest material index the instances use
  std::vector<prep::InstanceIn> last_ii;  // the instance inputs of the last pulse_instances_set
  DevBuf inst_bounds;                     // world bounds + centre of every instance (9 floats)
  bvh::Scratch bvh_scratch;
  DevBuf tmp_a, tmp_b, tmp_c, tmp_d;
  // Per-frame instance preparation inputs and TLAS build inputs, grown and
  // kept (a cudaFree per frame would synchronize the device).
  DevBuf prep_ii, prep_lights, prep_slot, tlas_min, tlas_max, tlas_cent;
  DevBuf tlas_meta;  // node count, levels, error code of a one-launch TLAS build
  // The same four words in mapped pinned host memory, stored there by a kernel
  // after the build: reading them needs no copy engine, so it does not queue
  // behind an asynchronous image download still running.
  uint32_t* meta_host = nullptr;
  uint32_t* meta_mapped = nullptr;  // its device-side address

  // Double-buffered per-frame state.  pulse_instances_set writes a frame's
  // instance records, light CDFs and TLAS into the set that no queued work
  // reads, on a stream of its own (upd_stream), while the previous frame still
  // traces on the context's stream; once that update is complete the sets
  // swap, and the next render reads the new one.  ev_back_free is recorded on
  // the context's stream at each swap: every kernel that can read the set
  // which then becomes the back set was queued before it.
  struct FrameSet {
    DevBuf tlas_nodes, instance_indices, instances, strength_cdf, tri_cdfs, mesh_areas, light_indices, inst_light,
        inst_bounds, prep_ii, prep_lights, tlas_min, tlas_max, tlas_cent, tlas_meta;
    uint32_t* meta_host = nullptr;
    uint32_t* meta_mapped = nullptr;
  };
  FrameSet back;
  cudaStream_t upd_stream = nullptr;
  cudaEvent_t ev_back_free = nullptr, ev_upd0 = nullptr, ev_upd1 = nullptr;
  bool back_free_recorded = false;
  // The same on the context's lanes (pipelined frames), where frames ran.
  cudaEvent_t ev_back_free_lane[2] = {nullptr, nullptr};
  bool back_free_lane_recorded[2] = {false, false};
  // Set by a successful pulse_instances_set; cleared by every call that
  // writes what the update reads (meshes, materials, caller buffers), so that
  // the update on upd_stream never has to wait for the context's stream.
  bool async_ok = false;
  void swap_sets() {
    FrameSet& b = back;
    std::swap(tlas_nodes, b.tlas_nodes);
    std::swap(instance_indices, b.instance_indices);
    std::swap(instances, b.instances);
    std::swap(strength_cdf, b.strength_cdf);
    std::swap(tri_cdfs, b.tri_cdfs);
    std::swap(mesh_areas, b.mesh_areas);
    std::swap(light_indices, b.light_indices);
    std::swap(inst_light, b.inst_light);
    std::swap(inst_bounds, b.inst_bounds);
    std::swap(prep_ii, b.prep_ii);
    std::swap(prep_lights, b.prep_lights);
    std::swap(tlas_min, b.tlas_min);
    std::swap(tlas_max, b.tlas_max);
    std::swap(tlas_cent, b.tlas_cent);
    std::swap(tlas_meta, b.tlas_meta);
    std::swap(meta_host, b.meta_host);
    std::swap(meta_mapped, b.meta_mapped);
  }
  void free_back() {
    FrameSet& b = back;
    for (DevBuf* x : {&b.tlas_nodes, &b.instance_indices, &b.instances, &b.strength_cdf, &b.tri_cdfs, &b.mesh_areas,
                      &b.light_indices, &b.inst_light, &b.inst_bounds, &b.prep_ii, &b.prep_lights, &b.tlas_min,
                      &b.tlas_max, &b.tlas_cent, &b.tlas_meta})
      free_buf(*x);
    if (b.meta_host) cudaFreeHost(b.meta_host);
    b.meta_host = b.meta_mapped = nullptr;
    back_free_recorded = false;
    back_free_lane_recorded[0] = back_free_lane_recorded[1] = false;
    async_ok = false;
  }

  std::vector<DevBuf*> bind_group() {
    return {&primitives, &triangle_data, &triangle_indices, &blas_nodes, &tlas_nodes, &instance_indices,
            &instances, &materials, &strength_cdf, &tri_cdfs, &mesh_areas, &light_indices};
  }
  void free_all() {
    for (DevBuf* b : bind_group()) free_buf(*b);
    free_buf(inst_light);
    free_buf(tri_bvh);
    tri_bvh_current = false;
    free_buf(inst_bounds);
    free_back();
    ready = false;
  }
  void free_meshes() {
    for (MeshRec& m : meshes) { free_buf(m.prims); free_buf(m.tdata); free_buf(m.nodes); free_buf(m.idx); }
    meshes.clear();
  }
  static void free_buf(DevBuf& b) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
  }
};

struct PulseTarget {
  PulseCtx* ctx = nullptr;
  uint32_t W = 0, H = 0;
  float4* image = nullptr;
  void* stage = nullptr;  // device staging of pulse_target_resample's host output
  size_t stage_bytes = 0;
  // pulse_target_download_async: the copy runs on copy_stream after the frame
  // (ev_ready) and signals ev_copied; the next write of the image waits for it.
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_ready = nullptr, ev_copied = nullptr;
  bool copy_pending = false;
  // The last pipelined frame into this target (on a lane of the context).
  cudaEvent_t ev_frame = nullptr;
  bool frame_pending = false;
};

namespace {
// Before a call writes t->image from its first kernel on: wait (on the
// context's stream) for an asynchronous download still reading it.
void target_write_fence(PulseTarget* t) {
  if (t->copy_pending) cudaStreamWaitEvent(t->ctx->stream, t->ev_copied, 0);
}
}  // namespace

namespace {

cudaError_t upload(DevBuf& b, const void* host, size_t bytes, cudaStream_t st) {
  if (b.p) { cudaFree(b.p); b.p = nullptr; }
  b.bytes = bytes;
  const size_t alloc = bytes ? bytes : 16;
  cudaError_t e = pt::dev_alloc((void**)&b.p, alloc);
  if (e != cudaSuccess) { b.p = nullptr; return e; }
  if (bytes) return cudaMemcpyAsync(b.p, host, bytes, cudaMemcpyHostToDevice, st);
  return cudaMemsetAsync(b.p, 0, alloc, st);
}

cudaError_t ensure(DevBuf& b, size_t bytes);

// upload() into a buffer that is kept when large enough: no cudaFree (which
// would synchronize the device) on the per-frame path.  Stream-ordered: work
// already enqueued reads the old contents.
cudaError_t upload_keep(DevBuf& b, const void* host, size_t bytes, cudaStream_t st) {
  cudaError_t e = ensure(b, bytes);
  if (e != cudaSuccess || bytes == 0) return e;
  return cudaMemcpyAsync(b.p, host, bytes, cudaMemcpyHostToDevice, st);
}

cudaError_t ensure(DevBuf& b, size_t bytes) {
  if (b.p && b.bytes >= bytes) return cudaSuccess;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
  cudaError_t e = pt::dev_alloc((void**)&b.p, bytes ? bytes : 16);
  if (e == cudaSuccess) b.bytes = bytes ? bytes : 16;
  else b.p = nullptr;
  return e;
}

// ---------------------------------------------------------------- validation
// Checks that every index a kernel will follow stays inside its buffer and that
// every BVH reachable from a root is a tree (a node reached twice is rejected),
// so device traversal never leaves its buffers; its loops are additionally
// bounded by the iteration cap as in the reference.
// *nested: whether every child box lies inside its parent's box (true for every
// tree the library builds; the traversal's fast slab test relies on it).
static bool box_inside(const PulseBvhNode& c, const PulseBvhNode& p) {
  for (int k = 0; k < 3; ++k)
    if (c.aabb_min[k] < p.aabb_min[k] || c.aabb_max[k] > p.aabb_max[k]) return false;
  return true;
}

// Elements of one tree (triangles of a mesh, instances of a TLAS) stay below
// 2^29, so node indices stay below 2^30: the traversal's stack entries use the
// two top bits as tags.
constexpr uint32_t kMaxTreeElems = 1u << 29;

std::string validate(const PulseSceneBuffers* b, bool* nested, uint32_t* tlas_levels, uint32_t* blas_levels) {
  *nested = true;
  *tlas_levels = *blas_levels = 1;
  const uint32_t K = b->instance_count, L = b->light_count, P = b->primitive_count, TI = b->triangle_index_count,
                 BN = b->blas_node_count, TN = b->tlas_node_count, II = b->instance_index_count,
                 M = b->material_count, C = b->light_cdf_count;
  if (P && (!b->primitives || !b->triangle_data)) return "primitives/triangle_data missing";
  if (TI && !b->triangle_indices) return "triangle_indices missing";
  if (BN && !b->blas_nodes) return "blas_nodes missing";
  if (TN == 0 || !b->tlas_nodes) return "tlas_nodes missing (an empty scene still has the invalid root node)";
  if (K >= kMaxTreeElems || TN >= 2 * kMaxTreeElems) return "2^29 or more instances or 2^30 TLAS nodes";
  if (II && !b->instance_indices) return "instance_indices missing";
  if (K && !b->instances) return "instances missing";
  if (M && !b->materials) return "materials missing";
  if (L && (!b->light_emission_strength_cdf || !b->light_mesh_areas || !b->light_indices)) return "light arrays missing";
  if (C && !b->light_triangle_area_cdfs) return "light_triangle_area_cdfs missing";
  // Instances, and each distinct mesh range they reference (walked once).
  for (uint32_t i = 0; i < K; ++i) {
    const PulseMeshInstance& in = b->instances[i];
    const uint64_t to = in.triangle_offset, tc = in.triangle_count, io = in.index_offset, no = in.node_offset;
    if (tc == 0) return "instance " + std::to_string(i) + ": mesh without triangles";
    if (tc >= kMaxTreeElems) return "instance " + std::to_string(i) + ": mesh of 2^29 or more triangles";
    if (to + tc > P) return "instance " + std::to_string(i) + ": triangles out of range";
    if (io + tc > TI) return "instance " + std::to_string(i) + ": triangle indices out of range";
    if (no >= BN) return "instance " + std::to_string(i) + ": node_offset out of range";
    if (in.material_index >= M) return "instance " + std::to_string(i) + ": material_index out of range";
  }
  std::vector<std::array<uint32_t, 3>> meshes;
  for (uint32_t i = 0; i < K; ++i) {
    const PulseMeshInstance& in = b->instances[i];
    meshes.push_back({in.index_offset, in.triangle_count, in.node_offset});
  }
  std::sort(meshes.begin(), meshes.end());
  meshes.erase(std::unique(meshes.begin(), meshes.end()), meshes.end());
  std::vector<uint32_t> mark(BN, 0);
  uint32_t walk = 0;
  for (const auto& mk : meshes) {
    const uint64_t io = mk[0], tc = mk[1], no = mk[2];
    for (uint64_t s = 0; s < tc; ++s)
      if (b->triangle_indices[io + s] >= tc) return "mesh at index_offset " + std::to_string(io) + ": triangle index out of range";
    ++walk;
    std::vector<std::array<uint32_t, 2>> stack{{0, 1}};  // node, level
    while (!stack.empty()) {
      const uint64_t g = no + stack.back()[0];
      const uint32_t lv = stack.back()[1];
      stack.pop_back();
      *blas_levels = std::max(*blas_levels, lv);
      if (g >= BN) return "mesh at node_offset " + std::to_string(no) + ": BLAS node out of range";
      if (mark[g] == walk) return "mesh at node_offset " + std::to_string(no) + ": BLAS is not a tree";
      mark[g] = walk;
      const PulseBvhNode& nd = b->blas_nodes[g];
      if (nd.count > 0) {
        if ((uint64_t)nd.a + nd.count > tc) return "mesh at node_offset " + std::to_string(no) + ": BLAS leaf out of range";
      } else {
        if (no + (uint64_t)nd.a + 1 >= BN) return "mesh at node_offset " + std::to_string(no) + ": BLAS child out of range";
        if (!box_inside(b->blas_nodes[no + nd.a], nd) || !box_inside(b->blas_nodes[no + nd.a + 1], nd)) *nested = false;
        stack.push_back({nd.a + 1, lv + 1});
        stack.push_back({nd.a, lv + 1});
      }
    }
  }
  // TLAS.
  {
    std::vector<uint8_t> tseen(TN, 0);
    const PulseBvhNode& r = b->tlas_nodes[0];
    if (!(r.a == 0 && r.count == 0)) {
      std::vector<std::array<uint32_t, 2>> stack{{0, 1}};  // node, level
      while (!stack.empty()) {
        const uint64_t n = stack.back()[0];
        const uint32_t lv = stack.back()[1];
        stack.pop_back();
        *tlas_levels = std::max(*tlas_levels, lv);
        if (n >= TN) return "TLAS node out of range";
        if (tseen[n]) return "TLAS is not a tree";
        tseen[n] = 1;
        const PulseBvhNode& nd = b->tlas_nodes[n];
        if (nd.count > 0) {
          if ((uint64_t)nd.a + nd.count > II) return "TLAS leaf out of range";
          for (uint32_t k = 0; k < nd.count; ++k)
            if (b->instance_indices[nd.a + k] >= K) return "TLAS instance index out of range";
        } else {
          if ((uint64_t)nd.a + 1 >= TN) return "TLAS child out of range";
          if (!box_inside(b->tlas_nodes[nd.a], nd) || !box_inside(b->tlas_nodes[nd.a + 1], nd)) *nested = false;
          stack.push_back({nd.a + 1, lv + 1});
          stack.push_back({nd.a, lv + 1});
        }
      }
    }
  }
  // Lights.
  for (uint32_t l = 0; l < L; ++l) {
    const PulseLightDataIndex& li = b->light_indices[l];
    if (li.mesh_instance_index >= K) return "light " + std::to_string(l) + ": instance out of range";
    const uint32_t tc = b->instances[li.mesh_instance_index].triangle_count;
    if (tc == 0) return "light " + std::to_string(l) + ": emissive instance without triangles";
    if ((uint64_t)li.cdf_offset + tc > C) return "light " + std::to_string(l) + ": CDF out of range";
  }
  return "";
}

int32_t check_params(PulseCtx* ctx, const PulseRenderParams* p) {
  if (!p) return set_err(ctx, PULSE_ERR_INVALID_ARG, "params is NULL");
  if (p->spp == 0 || p->spp > 65536) return set_err(ctx, PULSE_ERR_INVALID_ARG, "spp must be in [1, 65536]");
  if (p->max_depth > 4096) return set_err(ctx, PULSE_ERR_INVALID_ARG, "max_depth must be <= 4096");
  if (p->nee_mode > 2) return set_err(ctx, PULSE_ERR_INVALID_ARG, "nee_mode must be 0, 1 or 2");
  if (p->light_pick > 1) return set_err(ctx, PULSE_ERR_INVALID_ARG, "light_pick must be 0 or 1");
  if (p->stack_depth == 0 || p->stack_depth > 64) return set_err(ctx, PULSE_ERR_INVALID_ARG, "stack_depth must be in [1, 64]");
  if (p->iter_cap == 0) return set_err(ctx, PULSE_ERR_INVALID_ARG, "iter_cap must be > 0");
  if (p->kernel > 2) return set_err(ctx, PULSE_ERR_INVALID_ARG, "kernel must be 0, 1 or 2");
  if (p->trace_blocks > 8) return set_err(ctx, PULSE_ERR_INVALID_ARG, "trace_blocks must be <= 8");
  if (p->block_size != 0 && p->block_size != 64 && p->block_size != 128)
    return set_err(ctx, PULSE_ERR_INVALID_ARG, "block_size must be 0, 64 or 128");
  if (p->ray_sort > 1) return set_err(ctx, PULSE_ERR_INVALID_ARG, "ray_sort must be 0 or 1");
  return PULSE_OK;
}

pt::TraceCfg trace_cfg(const PulseRenderParams* p, const pt::DevScene& S) {
  pt::TraceCfg t;
  t.stack_depth = p->stack_depth;
  t.iter_cap = p->iter_cap;
  pt::trace_stacks(t, S.tlas_levels, S.blas_levels);
  t.eps_tri = p->eps_tri;
  t.eps_par = p->eps_par;
  t.quirks = p->quirks != 0;
  t.step_policy = p->step_policy;
  t.block = p->block_size ? p->block_size : 128;
  t.ray_sort = p->ray_sort;
  return t;
}
pt::PathCfg path_cfg(const PulseRenderParams* p) {
  pt::PathCfg c;
  c.max_depth = p->max_depth;
  c.spp = p->spp;
  c.nee_mode = p->nee_mode;
  c.light_pick = p->light_pick;
  c.seed = p->seed;
  c.wf_segments = p->wf_segments ? p->wf_segments : pt::kDefaultWfSegments;  // unused by the megakernel
  c.eps_origin = p->eps_origin;
  c.eps_shadow = p->eps_shadow;
  c.quirks = p->quirks != 0;
  c.no_rr = p->no_roulette != 0;
  return c;
}

int32_t read_counters(PulseCtx* ctx) {
  pt::Counters c;
  cudaError_t e = cudaMemcpyAsync(&c, ctx->d_counters, sizeof(c), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_err(ctx, e, "read counters");
  ctx->stats.iter_cap_hits = c.iter_cap_hits;
  ctx->stats.stack_overflows = c.stack_overflows;
  return PULSE_OK;
}

}  // namespace

extern "C" {

void pulse_default_params(PulseRenderParams* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->max_depth = 5;
  p->spp = 1;
  p->nee_mode = 0;
  p->light_pick = 0;
  p->seed = 0;
  p->quirks = 1;
  p->stack_depth = 32;
  p->iter_cap = 100000;
  p->eps_origin = 0.001f;
  p->eps_tri = 0.001f;
  p->eps_par = 1e-4f;
  p->eps_shadow = 0.005f;
}

int32_t pulse_ctx_create(int32_t device, PulseCtx** out) {
  if (!out) return PULSE_ERR_INVALID_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return PULSE_ERR_NO_DEVICE;
  if (device < 0 || device >= n) return PULSE_ERR_INVALID_ARG;
  PulseCtx* c = new PulseCtx();
  c->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
  c->stream = c->own_stream;
  if (e == cudaSuccess) e = pt::dev_alloc((void**)&c->d_counters, sizeof(pt::Counters));
  if (e == cudaSuccess) e = cudaMemset(c->d_counters, 0, sizeof(pt::Counters));
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
  if (e != cudaSuccess) {
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    if (c->d_counters) cudaFree(c->d_counters);
    delete c;
    return e == cudaErrorMemoryAllocation ? PULSE_ERR_OOM : PULSE_ERR_CUDA;
  }
  *out = c;
  return PULSE_OK;
}

int32_t pulse_ctx_destroy(PulseCtx* ctx) {
  if (!ctx) return PULSE_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  quiesce(ctx);
  cudaStreamSynchronize(ctx->stream);
  cudaFree(ctx->d_counters);
  cudaEventDestroy(ctx->ev0);
  cudaEventDestroy(ctx->ev1);
  if (ctx->wf.p) cudaFree(ctx->wf.p);
  if (ctx->gstage.p) cudaFree(ctx->gstage.p);
  if (ctx->batch_exec) cudaGraphExecDestroy(ctx->batch_exec);
  for (int i = 0; i < 2; ++i) {
    if (ctx->lane[i]) {
      cudaStreamSynchronize(ctx->lane[i]);
      cudaStreamDestroy(ctx->lane[i]);
    }
    if (ctx->lane_done[i]) cudaEventDestroy(ctx->lane_done[i]);
    if (ctx->lane_wf[i].p) cudaFree(ctx->lane_wf[i].p);
  }
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  cudaStreamSynchronize(ctx->own_stream);
  cudaStreamDestroy(ctx->own_stream);
  delete ctx;
  return PULSE_OK;
}

const char* pulse_last_error(const PulseCtx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int32_t pulse_ctx_set_stream(PulseCtx* ctx, void* stream) {
  if (!ctx) return PULSE_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  quiesce(ctx);
  cudaStreamSynchronize(ctx->stream);
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  return PULSE_OK;
}

int32_t pulse_debug_fail_allocations(uint32_t n) {
  pt::g_fail_allocs.store(n);
  return PULSE_OK;
}

int32_t pulse_ctx_get_stream(const PulseCtx* ctx, void** out) {
  if (!ctx || !out) return PULSE_ERR_INVALID_ARG;
  // ordered after the pipelined frames in flight, so that work the caller
  // orders after this stream sees their images
  PulseCtx* c = const_cast<PulseCtx*>(ctx);
  cudaSetDevice(c->device);
  quiesce(c);
  *out = (void*)ctx->stream;
  return PULSE_OK;
}

int32_t pulse_ctx_set_pipeline(PulseCtx* ctx, uint32_t depth) {
  if (!ctx) return PULSE_ERR_INVALID_ARG;
  if (depth != 1 && depth != 2) return set_err(ctx, PULSE_ERR_INVALID_ARG, "pipeline depth must be 1 or 2");
  cudaSetDevice(ctx->device);
  quiesce(ctx);
  if (depth == 2) {
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 2 && e == cudaSuccess; ++i) {
      if (!ctx->lane[i]) e = cudaStreamCreateWithFlags(&ctx->lane[i], cudaStreamNonBlocking);
      if (e == cudaSuccess && !ctx->lane_done[i])
        e = cudaEventCreateWithFlags(&ctx->lane_done[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess && !ctx->ev_fork) e = cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_err(ctx, e, "pulse_ctx_set_pipeline");
  }
  ctx->pipeline = depth;
  return PULSE_OK;
}

int32_t pulse_sync(PulseCtx* ctx) {
  if (!ctx) return PULSE_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  quiesce(ctx);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? PULSE_OK : cuda_err(ctx, e, "sync");
}

int32_t pulse_get_stats(const PulseCtx* ctx, PulseStats* out) {
  if (!ctx || !out) return PULSE_ERR_INVALID_ARG;
  PulseCtx* c = const_cast<PulseCtx*>(ctx);  // refreshes the cached device tallies
  cudaSetDevice(c->device);
  quiesce(c);
  if (int32_t rc = read_counters(c)) return rc;  // synchronizes the stream
  if (c->timed) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, c->ev0, c->ev1) == cudaSuccess) c->stats.last_render_ms = ms;
    cudaGetLastError();  // an unfinished or uncaptured event pair is not an error of later calls
  }
  *out = c->stats;
  return PULSE_OK;
}

int32_t pulse_scene_create(PulseCtx* ctx, PulseScene** out) {
  if (!ctx || !out) return PULSE_ERR_INVALID_ARG;
  PulseScene* s = new PulseScene();
  s->ctx = ctx;
  *out = s;
  return PULSE_OK;
}

int32_t pulse_scene_destroy(PulseScene* s) {
  if (!s) return PULSE_ERR_INVALID_ARG;
  cudaSetDevice(s->ctx->device);
  quiesce(s->ctx);
  cudaStreamSynchronize(s->ctx->stream);
  s->free_all();
  s->free_meshes();
  s->bvh_scratch.release();
  for (DevBuf* x : {&s->tmp_a, &s->tmp_b, &s->tmp_c, &s->tmp_d, &s->prep_ii, &s->prep_lights, &s->prep_slot,
                    &s->tlas_min, &s->tlas_max, &s->tlas_cent, &s->tlas_meta})
    PulseScene::free_buf(*x);
  if (s->meta_host) cudaFreeHost(s->meta_host);
  if (s->upd_stream) cudaStreamDestroy(s->upd_stream);
  for (cudaEvent_t ev : {s->ev_back_free, s->ev_upd0, s->ev_upd1, s->ev_back_free_lane[0], s->ev_back_free_lane[1]})
    if (ev) cudaEventDestroy(ev);
  delete s;
  return PULSE_OK;
}

// Derived layouts (tri_bvh per distinct mesh range, instance -> light map) and
// the device view; the 13 bind-group buffers must be in place.  tri_bvh depends
// on the meshes only, so it is gathered again only after they changed.
static cudaError_t finalize_scene(PulseScene* s, const std::vector<std::array<uint32_t, 3>>& ranges,
                                  const std::vector<int32_t>& inst_light, cudaStream_t st) {
  const PulseSceneBuffers& c = s->counts;
  cudaError_t e = upload_keep(s->inst_light, inst_light.data(), inst_light.size() * 4, st);
  const size_t tri_bvh_bytes = (size_t)c.triangle_index_count * 48;
  if (!s->tri_bvh_current || s->tri_bvh.bytes < tri_bvh_bytes) {
    s->tri_bvh_current = false;
    if (e == cudaSuccess) e = ensure(s->tri_bvh, tri_bvh_bytes);
    for (const auto& r : ranges) {  // {triangle_offset, index_offset, count}
      if (e != cudaSuccess) break;
      e = pt::launch_gather_tri_bvh((const float4*)s->primitives.p, (const uint32_t*)s->triangle_indices.p,
                                    (float4*)s->tri_bvh.p, r[0], r[1], r[2], st);
    }
    if (e != cudaSuccess) return e;
    s->tri_bvh_current = true;
    s->ctx->stats.kernel_launches += ranges.size();
  }
  if (e != cudaSuccess) return e;
  pt::DevScene& d = s->dev;
  d.tri_bvh = (const float4*)s->tri_bvh.p;
  d.primitives = (const float4*)s->primitives.p;
  d.triangle_data = (const float4*)s->triangle_data.p;
  d.triangle_indices = (const uint32_t*)s->triangle_indices.p;
  d.blas_nodes = (const float4*)s->blas_nodes.p;
  d.tlas_nodes = (const float4*)s->tlas_nodes.p;
  d.instance_indices = (const uint32_t*)s->instance_indices.p;
  d.instances = (const float4*)s->instances.p;
  d.materials = (const float4*)s->materials.p;
  d.strength_cdf = (const float*)s->strength_cdf.p;
  d.tri_cdfs = (const float*)s->tri_cdfs.p;
  d.mesh_areas = (const float*)s->mesh_areas.p;
  d.light_indices = (const uint2*)s->light_indices.p;
  d.inst_light = (const int32_t*)s->inst_light.p;
  d.instance_count = c.instance_count;
  d.light_count = c.light_count;
  return cudaSuccess;
}

int32_t pulse_scene_set_buffers(PulseScene* s, const PulseSceneBuffers* b) {
  if (!s || !b) return PULSE_ERR_INVALID_ARG;
  PulseCtx* ctx = s->ctx;
  bool nested = true;
  uint32_t tlas_levels = 1, blas_levels = 1;
  const std::string why = validate(b, &nested, &tlas_levels, &blas_levels);
  if (!why.empty()) return set_err(ctx, PULSE_ERR_INVALID_ARG, "scene buffers: " + why);
  cudaSetDevice(ctx->device);
  quiesce(ctx);
  cudaStream_t st = ctx->stream;
  cudaStreamSynchronize(st);
  s->free_all();
  s->free_meshes();
  s->mesh_table.clear();
  s->meshes_dirty = true;
  const uint32_t K = b->instance_count, L = b->light_count;
  cudaError_t e = cudaSuccess;
  auto up = [&](DevBuf& d, const void* h, size_t bytes) {
    if (e == cudaSuccess) e = upload(d, h, bytes, st);
  };
  up(s->primitives, b->primitives, (size_t)b->primitive_count * 48);
  up(s->triangle_data, b->triangle_data, (size_t)b->primitive_count * 80);
  up(s->triangle_indices, b->triangle_indices, (size_t)b->triangle_index_count * 4);
  up(s->blas_nodes, b->blas_nodes, (size_t)b->blas_node_count * 32);
  up(s->tlas_nodes, b->tlas_nodes, (size_t)b->tlas_node_count * 32);
  up(s->instance_indices, b->instance_indices, (size_t)b->instance_index_count * 4);
  up(s->instances, b->instances, (size_t)K * 160);
  up(s->materials, b->materials, (size_t)b->material_count * 48);
  up(s->strength_cdf, b->light_emission_strength_cdf, (size_t)L * 4);
  up(s->tri_cdfs, b->light_triangle_area_cdfs, (size_t)b->light_cdf_count * 4);
  up(s->mesh_areas, b->light_mesh_areas, (size_t)L * 4);
  up(s->light_indices, b->light_indices, (size_t)L * 8);
  s->counts = *b;
  s->prepped = false;
  s->last_inst.clear();
  s->materials_needed = 0;
  for (uint32_t i = 0; i < K; ++i)
    s->materials_needed = std::max(s->materials_needed, b->instances[i].material_index + 1);
  std::vector<int32_t> inst_light(K ? K : 1, -1);
  for (uint32_t l = 0; l < L; ++l) {
    const uint32_t ii = b->light_indices[l].mesh_instance_index;
    if (inst_light[ii] < 0) inst_light[ii] = (int32_t)l;
  }
  std::vector<std::array<uint32_t, 3>> ranges;
  for (uint32_t i = 0; i < K; ++i) {
    const PulseMeshInstance& in = b->instances[i];
    ranges.push_back({in.triangle_offset, in.index_offset, in.triangle_count});
  }
  std::sort(ranges.begin(), ranges.end());
  ranges.erase(std::unique(ranges.begin(), ranges.end()), ranges.end());
  if (e == cudaSuccess) e = finalize_scene(s, ranges, inst_light, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    s->free_all();
    return cuda_err(ctx, e, "scene upload");
  }
  s->dev.fast_slabs = nested ? 1u : 0u;
  s->dev.tlas_levels = tlas_levels;
  s->dev.blas_levels = blas_levels;
  s->ready = true;
  return PULSE_OK;
}

// --------------------------------------------------------- BVH entry points
static int32_t build_to_host(PulseCtx* ctx, const bvh::Input& in, const bvh::Params& bp, PulseBvhNode* nodes_out,
                             uint32_t* node_count, uint32_t* idx_out, bvh::Scratch& scratch) {
  cudaStream_t st = ctx->stream;
  const uint32_t n = in.n;
  DevBuf dn, di;
  cudaError_t e = ensure(dn, (size_t)(2 * (size_t)n - 1) * 32);
  if (e == cudaSuccess) e = ensure(di, (size_t)n * 4);
  if (e != cudaSuccess) {
    PulseScene::free_buf(dn);
    PulseScene::free_buf(di);
    return cuda_err(ctx, e, "bvh buffers");
  }
  std::string why;
  uint32_t cnt = 0;
  cudaEventRecord(ctx->ev0, st);
  const int rc = bvh::build(in, bp, (uint32_t*)dn.p, (uint32_t*)di.p, &cnt, scratch, st, &why);
  cudaEventRecord(ctx->ev1, st);
  int32_t out = PULSE_OK;
  if (rc == -7) out = set_err(ctx, PULSE_ERR_DEGENERATE, why);
  else if (rc == -9) out = set_err(ctx, PULSE_ERR_CUDA, why);
  else if (rc < 0) out = set_err(ctx, PULSE_ERR_INVALID_ARG, why);
  else if (rc > 0) out = cuda_err(ctx, (cudaError_t)rc, why.c_str());
  if (out == PULSE_OK) {
    e = cudaMemcpyAsync(nodes_out, dn.p, (size_t)cnt * 32, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && idx_out) e = cudaMemcpyAsync(idx_out, di.p, (size_t)n * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) out = cuda_err(ctx, e, "bvh download");
    *node_count = cnt;
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) == cudaSuccess) ctx->stats.last_build_ms = ms;
  }
  PulseScene::free_buf(dn);
  PulseScene::free_buf(di);
  return out;
}

int32_t pulse_build_blas(PulseCtx* ctx, const PulsePrimitive* prims, uint32_t n, const PulseBvhParams* params,
                         PulseBvhNode* nodes_out, uint32_t* node_count, uint32_t* tri_indices_out) {
  if (!ctx || !prims || !params || !nodes_out || !node_count || !tri_indices_out || n == 0)
    return PULSE_ERR_INVALID_ARG;
  if (params->bins < 2 || params->bins > 32) return set_err(ctx, PULSE_ERR_INVALID_ARG, "bins must be in [2, 32]");
  cudaSetDevice(ctx->device);
  quiesce(ctx);
  cudaStream_t st = ctx->stream;
  DevBuf dp, pmin, pmax, cent;
  cudaError_t e = upload(dp, prims, (size_t)n * 48, st);
  if (e == cudaSuccess) e = ensure(pmin, (size_t)n * 16);
  if (e == cudaSuccess) e = ensure(pmax, (size_t)n * 16);
  if (e == cudaSuccess) e = ensure(cent, (size_t)n * 16);
  if (e == cudaSuccess)
    e = bvh::prep_triangles((const float4*)dp.p, n, (float4*)pmin.p, (float4*)pmax.p, (float4*)cent.p, st);
  int32_t rc = PULSE_OK;
  if (e != cudaSuccess) rc = cuda_err(ctx, e, "build_blas inputs");
  bvh::Scratch scratch;
  if (rc == PULSE_OK) {
    bvh::Input in{(const float4*)pmin.p, (const float4*)pmax.p, (const float4*)cent.p, n};
    rc = build_to_host(ctx, in, bvh::Params{params->bins, params->max_leaf, 0}, nodes_out, node_count,
                       tri_indices_out, scratch);
  }
  scratch.release();
  for (DevBuf* x : {&dp, &pmin, &pmax, &cent}) PulseScene::free_buf(*x);
  return rc;
}

int32_t pulse_build_tlas(PulseCtx* ctx, const float* bounds9, uint32_t n, const PulseBvhParams* params,
                         PulseBvhNode* nodes_out, uint32_t* node_count, uint32_t* idx_out) {
  if (!ctx || !params || !nodes_out || !node_count || (n && (!bounds9 || !idx_out))) return PULSE_ERR_INVALID_ARG;
  if (n == 0) {
    std::memset(nodes_out, 0, 32);
    *node_count = 1;
    return PULSE_OK;
  }
  if (params->bins < 2 || params->bins > 32) return set_err(ctx, PULSE_ERR_INVALID_ARG, "bins must be in [2, 32]");
  cudaSetDevice(ctx->device);
  quiesce(ctx);
  cudaStream_t st = ctx->stream;
  DevBuf db, pmin, pmax, cent;
  cudaError_t e = upload(db, bounds9, (size_t)n * 36, st);
  if (e == cudaSuccess) e = ensure(pmin, (size_t)n * 16);
  if (e == cudaSuccess) e = ensure(pmax, (size_t)n * 16);
  if (e == cudaSuccess) e = ensure(cent, (size_t)n * 16);
  if (e == cudaSuccess)
    e = bvh::prep_instances((const float*)db.p, n, (float4*)pmin.p, (float4*)pmax.p, (float4*)cent.p, st);
  int32_t rc = PULSE_OK;
  if (e != cudaSuccess) rc = cuda_err(ctx, e, "build_tlas inputs");
  bvh::Scratch scratch;
  if (rc == PULSE_OK) {
    bvh::Input in{(const float4*)pmin.p, (const float4*)pmax.p, (const float4*)cent.p, n};
    rc = build_to_host(ctx, in, bvh::Params{params->bins, params->max_leaf, 1}, nodes_out, node_count, idx_out,
                       scratch);
  }
  scratch.release();
  for (DevBuf* x : {&db, &pmin, &pmax, &cent}) PulseScene::free_buf(*x);
  return rc;
}

// ------------------------------------------------- scene-preparation path
int32_t pulse_mesh_upload(PulseScene* s, const float* pos, const float* nrm, const float* uv, uint32_t nverts,
                          const uint32_t* idx, uint32_t nidx, const PulseBvhParams* params, uint32_t* mesh_id) {
  if (!s || !pos || !nrm || !uv || !idx || !params || !mesh_id) return PULSE_ERR_INVALID_ARG;
  PulseCtx* ctx = s->ctx;
  if (nidx == 0 || nidx % 3 != 0) return set_err(ctx, PULSE_ERR_INVALID_ARG, "index count must be a positive multiple of 3");
  if (nidx / 3 >= kMaxTreeElems) return set_err(ctx, PULSE_ERR_INVALID_ARG, "a mesh must have fewer than 2^29 triangles");
  if (params->bins < 2 || params->bins > 32) return set_err(ctx, PULSE_ERR_INVALID_ARG, "bins must be in [2, 32]");
  for (uint32_t i = 0; i < nidx; ++i)
    if (idx[i] >= nverts) return set_err(ctx, PULSE_ERR_INVALID_ARG, "vertex index out of range");
  cudaSetDevice(ctx->device);
  quiesce(ctx);
  cudaStream_t st = ctx->stream;
  const uint32_t nt = nidx / 3;
  MeshRec m;
  m.id = (uint32_t)s->meshes.size();
  m.ntris = nt;
  DevBuf dpos, dnrm, duv, didx, pmin, pmax, cent;
  cudaError_t e = upload(dpos, pos, (size_t)nverts * 12, st);
  if (e == cudaSuccess) e = upload(dnrm, nrm, (size_t)nverts * 12, st);
  if (e == cudaSuccess) e = upload(duv, uv, (size_t)nverts * 8, st);
  if (e == cudaSuccess) e = upload(didx, idx, (size_t)nidx * 4, st);
  if (e == cudaSuccess) e = ensure(m.prims, (size_t)nt * 48);
  if (e == cudaSuccess) e = ensure(m.tdata, (size_t)nt * 80);
  if (e == cudaSuccess)
    e = prep::soup((const float*)dpos.p, (const float*)dnrm.p, (const float*)duv.p, (const uint32_t*)didx.p, nt,
                   (float4*)m.prims.p, (float4*)m.tdata.p, st);
  if (e == cudaSuccess) e = ensure(pmin, (size_t)nt * 16);
  if (e == cudaSuccess) e = ensure(pmax, (size_t)nt * 16);
  if (e == cudaSuccess) e = ensure(cent, (size_t)nt * 16);
  if (e == cudaSuccess)
    e = bvh::prep_triangles((const float4*)m.prims.p, nt, (float4*)pmin.p, (float4*)pmax.p, (float4*)cent.p, st);
  if (e == cudaSuccess) e = ensure(m.nodes, (size_t)(2 * (size_t)nt - 1) * 32);
  if (e == cudaSuccess) e = ensure(m.idx, (size_t)nt * 4);
  int32_t rc = PULSE_OK;
  if (e != cudaSuccess) rc = cuda_err(ctx, e, "mesh upload");
  if (rc == PULSE_OK) {
    std::string why;
    bvh::Input in{(const float4*)pmin.p, (const float4*)pmax.p, (const float4*)cent.p, nt};
    cudaEventRecord(ctx->ev0, st);
    const int r = bvh::build(in, bvh::Params{params->bins, params->max_leaf, 0}, (uint32_t*)m.nodes.p,
                             (uint32_t*)m.idx.p, &m.node_count, s->bvh_scratch, st, &why, &m.levels);
    cudaEventRecord(ctx->ev1, st);
    if (r == -7) rc = set_err(ctx, PULSE_ERR_DEGENERATE, why);
    else if (r == -9) rc = set_err(ctx, PULSE_ERR_CUDA, why);
    else if (r < 0) rc = set_err(ctx, PULSE_ERR_INVALID_ARG, why);
    else if (r > 0) rc = cuda_err(ctx, (cudaError_t)r, why.c_str());
    float ms = 0.0f;
    if (rc == PULSE_OK && cudaEventSynchronize(ctx->ev1) == cudaSuccess &&
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) == cudaSuccess)
      ctx->stats.last_build_ms = ms;
  }
  for (DevBuf* x : {&dpos, &dnrm, &duv, &didx, &pmin, &pmax, &cent}) PulseScene::free_buf(*x);
  if (rc != PULSE_OK) {
    for (DevBuf* x : {&m.prims, &m.tdata, &m.nodes, &m.idx}) PulseScene::free_buf(*x);
    return rc;
  }
  m.alive = true;
  s->meshes.push_back(m);
  s->meshes_dirty = true;
  *mesh_id = m.id;
  return PULSE_OK;
}

int32_t pulse_mesh_remove(PulseScene* s, uint32_t mesh_id) {
  if (!s || mesh_id >= s->meshes.size() || !s->meshes[mesh_id].alive) return PULSE_ERR_INVALID_ARG;
  cudaSetDevice(s->ctx->device);
  quiesce(s->ctx);
  cudaStreamSynchronize(s->ctx->stream);
  MeshRec& m = s->meshes[mesh_id];
  for (DevBuf* x : {&m.prims, &m.tdata, &m.nodes, &m.idx}) PulseScene::free_buf(*x);
  m.alive = false;
  s->meshes_dirty = true;
  return PULSE_OK;
}

int32_t pulse_materials_set(PulseScene* s, const PulseMaterial* mats, uint32_t n) {
  if (!s || (n && !mats)) return PULSE_ERR_INVALID_ARG;
  PulseCtx* ctx = s->ctx;
  if (s->ready && !s->prepped && n < s->materials_needed)
    return set_err(ctx, PULSE_ERR_INVALID_ARG,
                   "materials: the instances use material " + std::to_string(s->materials_needed - 1));
  cudaSetDevice(ctx->device);
  quiesce(ctx);
  cudaStream_t st = ctx->stream;
  s->async_ok = false;  // the next instance update reads these materials: it queues behind this copy
  s->host_materials.assign(mats, mats + n);
  cudaError_t e;
  if (n && s->materials.p && s->materials.bytes == (size_t)n * 48) {
    e = cudaMemcpyAsync(s->materials.p, mats, (size_t)n * 48, cudaMemcpyHostToDevice, st);  // stream-ordered
  } else {
    cudaStreamSynchronize(st);  // no render in flight reads the old buffer
    e = upload(s->materials, mats, (size_t)n * 48, st);
  }
  if (e != cudaSuccess) return cuda_err(ctx, e, "materials");
  s->counts.material_count = n;
  s->dev.materials = (const float4*)s->materials.p;
  if (s->prepped) {
    if (n < s->materials_needed) {  // the last instances no longer fit: wait for pulse_instances_set
      s->ready = false;
      return PULSE_OK;
    }
    // prepare_mesh_instances derives the lights from the materials' emission
    // (src/scene/mod.rs:583-622): rebuild the instance records and light CDFs.
    const std::vector<PulseInstanceDesc> inst = s->last_inst;
    const PulseBvhParams tp = s->last_tlas;
    return pulse_instances_set(s, inst.data(), (uint32_t)inst.size(), &tp);
  }
  return PULSE_OK;
}

// prepare_mesh_data (src/scene/mod.rs:471-510): concatenation of every live
// mesh in id order with its offsets.
static cudaError_t concat_meshes(PulseScene* s) {
  cudaStream_t st = s->ctx->stream;
  s->tri_bvh_current = false;
  uint64_t nt = 0, nn = 0;
  s->mesh_table.assign(s->meshes.size(), {~0u, 0u, ~0u, ~0u});
  for (const MeshRec& m : s->meshes) {
    if (!m.alive) continue;
    s->mesh_table[m.id] = {(uint32_t)nt, m.ntris, (uint32_t)nt, (uint32_t)nn};
    nt += m.ntris;
    nn += m.node_count;
  }
  cudaError_t e = ensure(s->primitives, nt * 48);
  if (e == cudaSuccess) e = ensure(s->triangle_data, nt * 80);
  if (e == cudaSuccess) e = ensure(s->triangle_indices, nt * 4);
  if (e == cudaSuccess) e = ensure(s->blas_nodes, nn * 32);
  for (const MeshRec& m : s->meshes) {
    if (!m.alive || e != cudaSuccess) continue;
    const auto& t = s->mesh_table[m.id];
    e = cudaMemcpyAsync((char*)s->primitives.p + (size_t)t[0] * 48, m.prims.p, (size_t)m.ntris * 48, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync((char*)s->triangle_data.p + (size_t)t[0] * 80, m.tdata.p, (size_t)m.ntris * 80, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync((char*)s->triangle_indices.p + (size_t)t[2] * 4, m.idx.p, (size_t)m.ntris * 4, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync((char*)s->blas_nodes.p + (size_t)t[3] * 32, m.nodes.p, (size_t)m.node_count * 32, cudaMemcpyDeviceToDevice, st);
  }
  s->counts.primitive_count = (uint32_t)nt;
  s->counts.triangle_index_count = (uint32_t)nt;
  s->counts.blas_node_count = (uint32_t)nn;
  if (e == cudaSuccess) s->meshes_dirty = false;
  return e;
}

// The TLAS over the n instance bounds in s->inst_bounds (src/scene/tlas.rs:29-65).
// Up to bvh::direct_max() instances the build is one launch with no host
// round trip: *pending is set and finish_tlas reads the node count and levels
// once the caller has synchronized its stream.
__global__ void k_meta_to_host(const uint32_t* __restrict__ meta, volatile uint32_t* host) {
  if (threadIdx.x < 4) host[threadIdx.x] = meta[threadIdx.x];
}

static int32_t rebuild_tlas(PulseScene* s, uint32_t n, const PulseBvhParams* tp, uint32_t* count, uint32_t* levels,
                            bool* pending, cudaStream_t st) {
  PulseCtx* ctx = s->ctx;
  const uint64_t bvh_launches0 = s->bvh_scratch.launches;
  *count = 1;
  *levels = 1;
  *pending = false;
  cudaError_t e = cudaSuccess;
  int32_t rc = PULSE_OK;
  if (n == 0) {
    const uint32_t zero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    e = upload(s->tlas_nodes, zero, 32, st);
    if (e == cudaSuccess) e = ensure(s->instance_indices, 4);
    return e == cudaSuccess ? PULSE_OK : cuda_err(ctx, e, "TLAS");
  }
  DevBuf& pmin = s->tlas_min;
  DevBuf& pmax = s->tlas_max;
  DevBuf& cent = s->tlas_cent;
  e = ensure(pmin, (size_t)n * 16);
  if (e == cudaSuccess) e = ensure(pmax, (size_t)n * 16);
  if (e == cudaSuccess) e = ensure(cent, (size_t)n * 16);
  if (e == cudaSuccess) e = ensure(s->tlas_nodes, (size_t)(2 * (size_t)n - 1) * 32);
  if (e == cudaSuccess) e = ensure(s->instance_indices, (size_t)n * 4);
  if (e == cudaSuccess)
    e = bvh::prep_instances((const float*)s->inst_bounds.p, n, (float4*)pmin.p, (float4*)pmax.p, (float4*)cent.p,
                            st);
  if (e != cudaSuccess) rc = cuda_err(ctx, e, "TLAS inputs");
  if (rc == PULSE_OK && n <= bvh::direct_max()) {
    bvh::Input in{(const float4*)pmin.p, (const float4*)pmax.p, (const float4*)cent.p, n};
    e = ensure(s->tlas_meta, 16);
    if (e == cudaSuccess && !s->meta_host) {
      e = cudaHostAlloc((void**)&s->meta_host, 16, cudaHostAllocMapped);
      if (e == cudaSuccess) e = cudaHostGetDevicePointer((void**)&s->meta_mapped, s->meta_host, 0);
      if (e != cudaSuccess && s->meta_host) {
        cudaFreeHost(s->meta_host);
        s->meta_host = nullptr;
      }
    }
    if (e == cudaSuccess)
      e = bvh::build_direct(in, bvh::Params{tp->bins, tp->max_leaf, 1}, (uint32_t*)s->tlas_nodes.p,
                            (uint32_t*)s->instance_indices.p, (uint32_t*)s->tlas_meta.p, st);
    if (e == cudaSuccess) {
      k_meta_to_host<<<1, 32, 0, st>>>((const uint32_t*)s->tlas_meta.p, s->meta_mapped);
      e = cudaGetLastError();
    }
    if (e != cudaSuccess) return cuda_err(ctx, e, "TLAS");
    *pending = true;
    ctx->stats.kernel_launches += 3;
    return PULSE_OK;
  }
  if (rc == PULSE_OK) {
    std::string why;
    bvh::Input in{(const float4*)pmin.p, (const float4*)pmax.p, (const float4*)cent.p, n};
    const int r = bvh::build(in, bvh::Params{tp->bins, tp->max_leaf, 1}, (uint32_t*)s->tlas_nodes.p,
                             (uint32_t*)s->instance_indices.p, count, s->bvh_scratch, st, &why, levels);
    if (r == -7) rc = set_err(ctx, PULSE_ERR_DEGENERATE, why);
    else if (r == -9) rc = set_err(ctx, PULSE_ERR_CUDA, why);
    else if (r < 0) rc = set_err(ctx, PULSE_ERR_INVALID_ARG, why);
    else if (r > 0) rc = cuda_err(ctx, (cudaError_t)r, why.c_str());
  }
  ctx->stats.kernel_launches += 1 + (s->bvh_scratch.launches - bvh_launches0);
  return rc;
}

// Node count and levels of a TLAS built by rebuild_tlas with *pending set
// (the context's stream must have been synchronized after the build).
static int32_t finish_tlas(PulseScene* s, uint32_t* count, uint32_t* levels) {
  uint32_t h[4];
  for (int k = 0; k < 4; ++k) h[k] = reinterpret_cast<volatile uint32_t*>(s->meta_host)[k];
  if ((int)h[2] == -7)
    return set_err(s->ctx, PULSE_ERR_DEGENERATE,
                   "TLAS: degenerate split, the reference's partition would underflow (src/scene/tlas.rs)");
  if (h[2] != 0 || h[0] == 0) return set_err(s->ctx, PULSE_ERR_CUDA, "TLAS: internal index check failed");
  *count = h[0];
  *levels = h[1];
  return PULSE_OK;
}

// The scene's update stream (highest priority, so that its small kernels take
// the first free block slots while a frame traces) and its events.
static bool ensure_update_stream(PulseScene* s) {
  if (!s->upd_stream) {
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (cudaStreamCreateWithPriority(&s->upd_stream, cudaStreamNonBlocking, greatest) != cudaSuccess) {
      s->upd_stream = nullptr;
      cudaGetLastError();
      return false;
    }
  }
  if (!s->ev_back_free && cudaEventCreateWithFlags(&s->ev_back_free, cudaEventDisableTiming) != cudaSuccess)
    s->ev_back_free = nullptr;
  if (!s->ev_upd0 && cudaEventCreate(&s->ev_upd0) != cudaSuccess) s->ev_upd0 = nullptr;
  if (!s->ev_upd1 && cudaEventCreate(&s->ev_upd1) != cudaSuccess) s->ev_upd1 = nullptr;
  for (int i = 0; i < 2; ++i)
    if (!s->ev_back_free_lane[i] &&
        cudaEventCreateWithFlags(&s->ev_back_free_lane[i], cudaEventDisableTiming) != cudaSuccess)
      s->ev_back_free_lane[i] = nullptr;
  cudaGetLastError();
  return s->ev_back_free && s->ev_upd0 && s->ev_upd1 && s->ev_back_free_lane[0] && s->ev_back_free_lane[1];
}

int32_t pulse_instances_set(PulseScene* s, const PulseInstanceDesc* inst, uint32_t n, const PulseBvhParams* tp) {
  if (!s || (n && !inst) || !tp) return PULSE_ERR_INVALID_ARG;
  PulseCtx* ctx = s->ctx;
  if (tp->bins < 2 || tp->bins > 32) return set_err(ctx, PULSE_ERR_INVALID_ARG, "TLAS bins must be in [2, 32]");
  if (n >= kMaxTreeElems) return set_err(ctx, PULSE_ERR_INVALID_ARG, "fewer than 2^29 instances");
  cudaSetDevice(ctx->device);
  // Double-buffered update (see PulseScene::FrameSet) when nothing it reads
  // has been written since the last successful call and the TLAS is a
  // one-launch build; otherwise the update runs on the context's stream, in
  // place, after the work queued there.
  const bool fast = s->async_ok && s->ready && !s->meshes_dirty && s->tri_bvh_current && n > 0 &&
                    n <= bvh::direct_max() && ensure_update_stream(s);
  if (!fast) quiesce(ctx);  // the in-place update follows every frame in flight
  cudaStream_t st = ctx->stream;
  if (!fast) cudaEventRecord(ctx->ev0, st);
  cudaError_t e = cudaSuccess;
  if (s->meshes_dirty) e = concat_meshes(s);
  if (e != cudaSuccess) return cuda_err(ctx, e, "mesh concatenation");
  // Instance records and the light list (src/scene/mod.rs:583-622).
  std::vector<prep::InstanceIn> ii(n);
  std::vector<prep::LightIn> lights;
  std::vector<PulseLightDataIndex> lidx;
  std::vector<int32_t> inst_light(n ? n : 1, -1);
  uint32_t cdf_len = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const PulseInstanceDesc& d = inst[i];
    if (d.mesh_id >= s->mesh_table.size() || s->mesh_table[d.mesh_id][0] == ~0u)
      return set_err(ctx, PULSE_ERR_INVALID_ARG, "instance " + std::to_string(i) + ": unknown mesh");
    if (d.material_index >= s->host_materials.size())
      return set_err(ctx, PULSE_ERR_INVALID_ARG, "instance " + std::to_string(i) + ": material out of range");
    const auto& t = s->mesh_table[d.mesh_id];
    std::memcpy(ii[i].object_world, d.object_world, 64);
    ii[i].triangle_offset = t[0];
    ii[i].triangle_count = t[1];
    ii[i].index_offset = t[2];
    ii[i].node_offset = t[3];
    ii[i].material_index = d.material_index;
    const float* em = s->host_materials[d.material_index].emissive;
    const float len = std::sqrt(em[0] * em[0] + em[1] * em[1] + em[2] * em[2]);
    if (len > 0.0001f) {
      inst_light[i] = (int32_t)lights.size();
      lights.push_back(prep::LightIn{i, t[0], t[1], cdf_len, d.material_index});
      lidx.push_back(PulseLightDataIndex{cdf_len, i});
      cdf_len += t[1];
    }
  }
  const uint32_t L = (uint32_t)lights.size();
  cudaEvent_t t0 = ctx->ev0, t1 = ctx->ev1;
  if (fast) {
    // The back set was last read by work queued before the previous swap;
    // after this swap the set the queued frames read is the back set, read by
    // nothing queued after this point.
    st = s->upd_stream;
    t0 = s->ev_upd0;
    t1 = s->ev_upd1;
    if (s->back_free_recorded) cudaStreamWaitEvent(st, s->ev_back_free, 0);
    for (int i = 0; i < 2; ++i)
      if (s->back_free_lane_recorded[i]) cudaStreamWaitEvent(st, s->ev_back_free_lane[i], 0);
    s->swap_sets();
    cudaEventRecord(s->ev_back_free, ctx->stream);
    s->back_free_recorded = true;
    for (int i = 0; i < 2; ++i)
      if (ctx->lane[i] && s->ev_back_free_lane[i]) {
        cudaEventRecord(s->ev_back_free_lane[i], ctx->lane[i]);
        s->back_free_lane_recorded[i] = true;
      }
    cudaEventRecord(t0, st);
  }
  s->async_ok = false;
  DevBuf& d_ii = s->prep_ii;
  DevBuf& d_lights = s->prep_lights;
  e = upload_keep(d_ii, ii.data(), (size_t)n * sizeof(prep::InstanceIn), st);
  if (e == cudaSuccess) e = ensure(s->instances, (size_t)n * 160);
  if (e == cudaSuccess) e = ensure(s->inst_bounds, (size_t)n * 36);
  if (e == cudaSuccess)
    e = prep::instances((const prep::InstanceIn*)d_ii.p, n, (const float4*)s->blas_nodes.p, (float4*)s->instances.p,
                        (float*)s->inst_bounds.p, st);
  if (e == cudaSuccess) e = upload_keep(d_lights, lights.data(), (size_t)L * sizeof(prep::LightIn), st);
  if (e == cudaSuccess) e = ensure(s->tri_cdfs, (size_t)cdf_len * 4);
  if (e == cudaSuccess) e = ensure(s->mesh_areas, (size_t)L * 4);
  if (e == cudaSuccess) e = ensure(s->strength_cdf, (size_t)L * 4);
  if (e == cudaSuccess) e = upload_keep(s->light_indices, lidx.data(), (size_t)L * 8, st);
  if (e == cudaSuccess)
    e = prep::lights((const prep::LightIn*)d_lights.p, L, (const float4*)s->primitives.p, (const float4*)s->materials.p,
                     (float*)s->tri_cdfs.p, (float*)s->mesh_areas.p, (float*)s->strength_cdf.p, st);
  int32_t rc = PULSE_OK;
  if (e != cudaSuccess) rc = cuda_err(ctx, e, "instance preparation");
  ctx->stats.kernel_launches += (n ? 1 : 0) + (L ? 2 : 0);
  // TLAS (src/scene/tlas.rs:29-65).
  uint32_t tlas_count = 1, tlas_levels = 1;
  bool pending = false;
  if (rc == PULSE_OK) rc = rebuild_tlas(s, n, tp, &tlas_count, &tlas_levels, &pending, st);
  if (rc == PULSE_OK) {
    std::vector<std::array<uint32_t, 3>> ranges;
    for (const MeshRec& m : s->meshes)
      if (m.alive) ranges.push_back({s->mesh_table[m.id][0], s->mesh_table[m.id][2], m.ntris});
    s->counts.instance_count = n;
    s->counts.light_count = L;
    s->counts.instance_index_count = n;
    s->counts.light_cdf_count = cdf_len;
    e = finalize_scene(s, ranges, inst_light, st);
    cudaEventRecord(t1, st);
    // The fast path waits for its own stream only: the previous frame may
    // still be tracing on the context's stream, and whatever is queued there
    // from now on starts after the update has completed.
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = cuda_err(ctx, e, "scene finalize");
    if (rc == PULSE_OK && pending) rc = finish_tlas(s, &tlas_count, &tlas_levels);
    s->counts.tlas_node_count = tlas_count;
    s->dev.fast_slabs = 1u;  // trees built here nest by construction
    s->dev.tlas_levels = tlas_levels;
    s->dev.blas_levels = 1;
    for (const MeshRec& m : s->meshes)
      if (m.alive && m.levels > s->dev.blas_levels) s->dev.blas_levels = m.levels;
    float ms = 0.0f;
    if (rc == PULSE_OK && cudaEventElapsedTime(&ms, t0, t1) == cudaSuccess) ctx->stats.last_upload_ms = ms;
  }
  if (fast && rc != PULSE_OK) cudaStreamSynchronize(st);  // nothing of a failed update stays in flight
  s->ready = rc == PULSE_OK;
  s->async_ok = rc == PULSE_OK;
  if (rc == PULSE_OK) {
    if (s->last_inst.data() != inst) s->last_inst.assign(inst, inst + n);
    s->last_ii = ii;
    s->last_tlas = *tp;
    s->prepped = true;
    s->materials_needed = 0;
    for (uint32_t i = 0; i < n; ++i) s->materials_needed = std::max(s->materials_needed, inst[i].material_index + 1);
  }
  return rc;
}

int32_t pulse_instances_update(PulseScene* s, const uint32_t* idx, const float* object_world, uint32_t n,
                               const PulseBvhParams* tlas_params) {
  if (!s || (n && (!idx || !object_world))) return PULSE_ERR_INVALID_ARG;
  PulseCtx* ctx = s->ctx;
  if (!s->ready || !s->prepped || s->meshes_dirty)
    return set_err(ctx, PULSE_ERR_NOT_READY, "instances_update needs a scene prepared by pulse_instances_set "
                                             "with no mesh change since");
  const PulseBvhParams tp = tlas_params ? *tlas_params : s->last_tlas;
  if (tp.bins < 2 || tp.bins > 32) return set_err(ctx, PULSE_ERR_INVALID_ARG, "TLAS bins must be in [2, 32]");
  const uint32_t K = (uint32_t)s->last_ii.size();
  std::vector<uint8_t> seen(K, 0);
  for (uint32_t k = 0; k < n; ++k) {
    if (idx[k] >= K)
      return set_err(ctx, PULSE_ERR_INVALID_ARG, "update " + std::to_string(k) + ": instance index out of range");
    if (seen[idx[k]]++)
      return set_err(ctx, PULSE_ERR_INVALID_ARG, "update " + std::to_string(k) + ": instance index repeated");
  }
  cudaSetDevice(ctx->device);
  quiesce(ctx);
  cudaStream_t st = ctx->stream;
  cudaEventRecord(ctx->ev0, st);
  std::vector<prep::InstanceIn> ii(n);
  for (uint32_t k = 0; k < n; ++k) {
    ii[k] = s->last_ii[idx[k]];
    std::memcpy(ii[k].object_world, object_world + 16 * (size_t)k, 64);
  }
  DevBuf& d_ii = s->prep_ii;
  DevBuf& d_slot = s->prep_slot;
  cudaError_t e = upload_keep(d_ii, ii.data(), (size_t)n * sizeof(prep::InstanceIn), st);
  if (e == cudaSuccess) e = upload_keep(d_slot, idx, (size_t)n * 4, st);
  if (e == cudaSuccess)
    e = prep::instances((const prep::InstanceIn*)d_ii.p, n, (const float4*)s->blas_nodes.p, (float4*)s->instances.p,
                        (float*)s->inst_bounds.p, st, (const uint32_t*)d_slot.p);
  int32_t rc = e == cudaSuccess ? PULSE_OK : cuda_err(ctx, e, "instance update");
  ctx->stats.kernel_launches += n ? 1 : 0;
  uint32_t tlas_count = 1, tlas_levels = 1;
  bool pending = false;
  if (rc == PULSE_OK) rc = rebuild_tlas(s, K, &tp, &tlas_count, &tlas_levels, &pending, st);
  if (rc == PULSE_OK) {
    s->dev.tlas_nodes = (const float4*)s->tlas_nodes.p;
    s->dev.instance_indices = (const uint32_t*)s->instance_indices.p;
    cudaEventRecord(ctx->ev1, st);
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = cuda_err(ctx, e, "instance update");
    if (rc == PULSE_OK && pending) rc = finish_tlas(s, &tlas_count, &tlas_levels);
    s->counts.tlas_node_count = tlas_count;
    s->dev.tlas_levels = tlas_levels;
    float ms = 0.0f;
    if (rc == PULSE_OK && cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) == cudaSuccess) ctx->stats.last_upload_ms = ms;
  }
  if (rc != PULSE_OK) {
    s->ready = false;  // records and TLAS may disagree; the next pulse_instances_set repairs the scene
    return rc;
  }
  for (uint32_t k = 0; k < n; ++k) {
    s->last_ii[idx[k]] = ii[k];
    std::memcpy(s->last_inst[idx[k]].object_world, object_world + 16 * (size_t)k, 64);
  }
  s->last_tlas = tp;
  return PULSE_OK;
}

int32_t pulse_scene_counts(PulseScene* s, PulseSceneBuffers* out) {
  if (!s || !out) return PULSE_ERR_INVALID_ARG;
  *out = s->counts;
  out->primitives = nullptr; out->triangle_data = nullptr; out->triangle_indices = nullptr;
  out->blas_nodes = nullptr; out->tlas_nodes = nullptr; out->instance_indices = nullptr;
  out->instances = nullptr; out->materials = nullptr; out->light_emission_strength_cdf = nullptr;
  out->light_triangle_area_cdfs = nullptr; out->light_mesh_areas = nullptr; out->light_indices = nullptr;
  return PULSE_OK;
}

int32_t pulse_scene_download(PulseScene* s, const PulseSceneBuffers* dst) {
  if (!s || !dst) return PULSE_ERR_INVALID_ARG;
  if (!s->ready) return set_err(s->ctx, PULSE_ERR_NOT_READY, "scene has no buffers");
  cudaSetDevice(s->ctx->device);
  quiesce(s->ctx);
  cudaStream_t st = s->ctx->stream;
  const PulseSceneBuffers& c = s->counts;
  cudaError_t e = cudaSuccess;
  auto dl = [&](const void* h, const DevBuf& d, size_t bytes) {
    if (h && bytes && e == cudaSuccess) e = cudaMemcpyAsync((void*)h, d.p, bytes, cudaMemcpyDeviceToHost, st);
  };
  dl(dst->primitives, s->primitives, (size_t)c.primitive_count * 48);
  dl(dst->triangle_data, s->triangle_data, (size_t)c.primitive_count * 80);
  dl(dst->triangle_indices, s->triangle_indices, (size_t)c.triangle_index_count * 4);
  dl(dst->blas_nodes, s->blas_nodes, (size_t)c.blas_node_count * 32);
  dl(dst->tlas_nodes, s->tlas_nodes, (size_t)c.tlas_node_count * 32);
  dl(dst->instance_indices, s->instance_indices, (size_t)c.instance_index_count * 4);
  dl(dst->instances, s->instances, (size_t)c.instance_count * 160);
  dl(dst->materials, s->materials, (size_t)c.material_count * 48);
  dl(dst->light_emission_strength_cdf, s->strength_cdf, (size_t)c.light_count * 4);
  dl(dst->light_triangle_area_cdfs, s->tri_cdfs, (size_t)c.light_cdf_count * 4);
  dl(dst->light_mesh_areas, s->mesh_areas, (size_t)c.light_count * 4);
  dl(dst->light_indices, s->light_indices, (size_t)c.light_count * 8);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? PULSE_OK : cuda_err(s->ctx, e, "scene download");
}

int32_t pulse_target_create(PulseCtx* ctx, uint32_t W, uint32_t H, PulseTarget** out) {
  if (!ctx || !out || W == 0 || H == 0 || (uint64_t)W * H > (1ull << 31)) return PULSE_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  PulseTarget* t = new PulseTarget();
  t->ctx = ctx;
  t->W = W;
  t->H = H;
  cudaError_t e = pt::dev_alloc((void**)&t->image, (size_t)W * H * 16);
  if (e == cudaSuccess) e = cudaMemsetAsync(t->image, 0, (size_t)W * H * 16, ctx->stream);
  if (e != cudaSuccess) {
    if (t->image) cudaFree(t->image);
    delete t;
    return cuda_err(ctx, e, "target create");
  }
  *out = t;
  return PULSE_OK;
}

int32_t pulse_target_destroy(PulseTarget* t) {
  if (!t) return PULSE_ERR_INVALID_ARG;
  cudaSetDevice(t->ctx->device);
  quiesce(t->ctx);
  cudaStreamSynchronize(t->ctx->stream);
  if (t->copy_stream) {
    cudaStreamSynchronize(t->copy_stream);
    cudaStreamDestroy(t->copy_stream);
    cudaEventDestroy(t->ev_ready);
    cudaEventDestroy(t->ev_copied);
  }
  if (t->ev_frame) cudaEventDestroy(t->ev_frame);
  cudaFree(t->image);
  if (t->stage) cudaFree(t->stage);
  delete t;
  return PULSE_OK;
}

int32_t pulse_target_download_async(PulseTarget* t, float* host) {
  if (!t || !host) return PULSE_ERR_INVALID_ARG;
  PulseCtx* ctx = t->ctx;
  cudaSetDevice(ctx->device);
  cudaError_t e = cudaSuccess;
  if (!t->copy_stream) {
    e = cudaStreamCreateWithFlags(&t->copy_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&t->ev_ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&t->ev_copied, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_err(ctx, e, "pulse_target_download_async: stream");
  }
  e = cudaEventRecord(t->ev_ready, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(t->copy_stream, t->ev_ready, 0);
  // the last pipelined frame into this target runs on a lane, not on the
  // context's stream
  if (e == cudaSuccess && t->frame_pending) e = cudaStreamWaitEvent(t->copy_stream, t->ev_frame, 0);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(host, t->image, (size_t)t->W * t->H * 16, cudaMemcpyDeviceToHost, t->copy_stream);
  if (e == cudaSuccess) e = cudaEventRecord(t->ev_copied, t->copy_stream);
  if (e != cudaSuccess) return cuda_err(ctx, e, "pulse_target_download_async");
  t->copy_pending = true;
  return PULSE_OK;
}

int32_t pulse_target_download_wait(PulseTarget* t) {
  if (!t) return PULSE_ERR_INVALID_ARG;
  if (!t->copy_pending) return PULSE_OK;
  cudaSetDevice(t->ctx->device);
  const cudaError_t e = cudaEventSynchronize(t->ev_copied);
  if (e != cudaSuccess) return cuda_err(t->ctx, e, "pulse_target_download_wait");
  t->copy_pending = false;
  return PULSE_OK;
}

int32_t pulse_target_device_ptr(const PulseTarget* t, void** out) {
  if (!t || !out) return PULSE_ERR_INVALID_ARG;
  *out = t->image;
  return PULSE_OK;
}

int32_t pulse_target_download(PulseTarget* t, float* host) {
  if (!t || !host) return PULSE_ERR_INVALID_ARG;
  PulseCtx* ctx = t->ctx;
  cudaSetDevice(ctx->device);
  quiesce(ctx);
  cudaError_t e = cudaMemcpyAsync(host, t->image, (size_t)t->W * t->H * 16, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? PULSE_OK : cuda_err(ctx, e, "target download");
}

int32_t pulse_target_upload(PulseTarget* t, const float* host) {
  if (!t || !host) return PULSE_ERR_INVALID_ARG;
  PulseCtx* ctx = t->ctx;
  cudaSetDevice(ctx->device);
  quiesce(ctx);
  target_write_fence(t);
  cudaError_t e = cudaMemcpyAsync(t->image, host, (size_t)t->W * t->H * 16, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? PULSE_OK : cuda_err(ctx, e, "target upload");
}

int32_t pulse_target_resample(PulseTarget* t, uint32_t out_w, uint32_t out_h, uint32_t filter, void* dst,
                              uint32_t dst_on_host) {
  if (!t) return PULSE_ERR_INVALID_ARG;
  PulseCtx* ctx = t->ctx;
  if (!dst) return set_err(ctx, PULSE_ERR_INVALID_ARG, "pulse_target_resample: dst is NULL");
  if (filter > 1) return set_err(ctx, PULSE_ERR_INVALID_ARG, "pulse_target_resample: filter must be 0 or 1");
  if (out_w == 0 || out_h == 0 || out_w > 65535 || out_h > 65535)
    return set_err(ctx, PULSE_ERR_INVALID_ARG, "pulse_target_resample: output size must be in [1, 65535]");
  cudaSetDevice(ctx->device);
  quiesce(ctx);
  const size_t bytes = (size_t)out_w * out_h * 8;
  void* out = dst;
  cudaError_t e = cudaSuccess;
  if (dst_on_host) {
    if (t->stage_bytes < bytes) {
      cudaStreamSynchronize(ctx->stream);
      if (t->stage) cudaFree(t->stage);
      t->stage = nullptr;
      t->stage_bytes = 0;
      e = pt::dev_alloc((void**)&t->stage, bytes);
      if (e != cudaSuccess) return cuda_err(ctx, e, "pulse_target_resample: staging buffer");
      t->stage_bytes = bytes;
    }
    out = t->stage;
  }
  e = pt::launch_resample(t->image, t->W, t->H, out, out_w, out_h, filter, ctx->stream);
  if (e == cudaSuccess && dst_on_host) {
    e = cudaMemcpyAsync(dst, t->stage, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  }
  if (e != cudaSuccess) return cuda_err(ctx, e, "pulse_target_resample");
  ctx->stats.kernel_launches += 1;
  return PULSE_OK;
}

// Grows the context's wavefront buffers to hold `paths` paths.
static cudaError_t grow_wf_buf(DevBufC& wf, size_t paths) {
  const size_t need = pt::wf_bytes(paths);
  if (wf.bytes >= need) return cudaSuccess;
  if (wf.p) cudaFree(wf.p);
  wf.p = nullptr;
  wf.bytes = 0;
  const cudaError_t e = pt::dev_alloc((void**)&wf.p, need);
  if (e == cudaSuccess) wf.bytes = need;
  return e;
}
static cudaError_t grow_wf(PulseCtx* ctx, size_t paths) { return grow_wf_buf(ctx->wf, paths); }

static pt::FrameCfg frame_cfg(const PulseView* view, const PulseTarget* t, uint32_t accumulation_count) {
  pt::FrameCfg fc;
  const float* m = view->inverse_view_proj;
  fc.ivp = pt::M4{make_float4(m[0], m[1], m[2], m[3]), make_float4(m[4], m[5], m[6], m[7]),
                  make_float4(m[8], m[9], m[10], m[11]), make_float4(m[12], m[13], m[14], m[15])};
  fc.eye = make_float3(view->world_position[0], view->world_position[1], view->world_position[2]);
  fc.W = t->W;
  fc.H = t->H;
  fc.acc = accumulation_count;
  return fc;
}

static int32_t render_impl(PulseScene* s, const PulseView* view, PulseTarget* t, uint32_t accumulation_count,
                           const PulseRenderParams* p, PulseWorkCounters* wc) {
  if (!s || !view || !t) return PULSE_ERR_INVALID_ARG;
  PulseCtx* ctx = s->ctx;
  if (t->ctx != ctx) return set_err(ctx, PULSE_ERR_INVALID_ARG, "target belongs to another context");
  if (int32_t rc = check_params(ctx, p)) return rc;
  if (!s->ready) return set_err(ctx, PULSE_ERR_NOT_READY, "scene has no buffers");
  if ((uint64_t)t->W * t->H * p->spp >= (1ull << 31))
    return set_err(ctx, PULSE_ERR_INVALID_ARG, "render: width * height * spp must be below 2^31");
  cudaSetDevice(ctx->device);
  // A pipelined frame (wavefront, no work counters) runs on the next lane and
  // leaves the context's stream free; anything else first waits for the
  // frames in flight.
  const bool piped = ctx->pipeline > 1 && p->kernel != 1 && !wc;
  if (!piped) quiesce(ctx);
  const pt::FrameCfg fc = frame_cfg(view, t, accumulation_count);
  unsigned long long* d_work = nullptr;
  cudaError_t e = cudaSuccess;
  if (wc) {
    e = pt::dev_alloc((void**)&d_work, 8 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemsetAsync(d_work, 0, 8 * sizeof(unsigned long long), ctx->stream);
    if (e != cudaSuccess) return cuda_err(ctx, e, "work counters");
  }
  uint32_t launches = 0;
  if (p->kernel != 1) {  // 0 (auto) and 2: the wavefront
    const size_t paths = (size_t)t->W * t->H * p->spp;
    const int ln = ctx->next_lane;
    DevBufC& wfb = piped ? ctx->lane_wf[ln] : ctx->wf;
    cudaStream_t st = piped ? ctx->lane[ln] : ctx->stream;
    e = grow_wf_buf(wfb, paths);
    if (e != cudaSuccess) {
      if (d_work) cudaFree(d_work);
      return cuda_err(ctx, e, "wavefront buffers");
    }
    // an asynchronous download of the last frame overlaps this frame's
    // tracing: only the accumulation (the frame's last kernel) waits for it
    cudaEvent_t image_wait = t->copy_pending ? t->ev_copied : nullptr;
    if (piped) {
      // the frame starts after the work queued on the context's stream (no
      // frame is queued there); its accumulation also waits for the previous
      // pipelined frame into this target, joined into the copy stream's
      // event when a download is pending too
      cudaEventRecord(ctx->ev_fork, ctx->stream);
      cudaStreamWaitEvent(st, ctx->ev_fork, 0);
      if (!t->ev_frame) e = cudaEventCreateWithFlags(&t->ev_frame, cudaEventDisableTiming);
      if (e == cudaSuccess && t->frame_pending) {
        if (t->copy_pending) {
          cudaStreamWaitEvent(t->copy_stream, t->ev_frame, 0);
          e = cudaEventRecord(t->ev_copied, t->copy_stream);
        } else {
          image_wait = t->ev_frame;
        }
      }
      if (e != cudaSuccess) {
        if (d_work) cudaFree(d_work);
        return cuda_err(ctx, e, "pipelined frame");
      }
    }
    const pt::WfBuffers B = pt::wf_carve(wfb.p, paths);
    const pt::WfScene one = pt::wf_scene(s->dev, path_cfg(p), fc, t->image);
    cudaEventRecord(ctx->ev0, st);
    e = pt::wf_render((int)p->nee_mode, trace_cfg(p, s->dev), &one, 1, p->wf_segments, p->trace_blocks, B,
                      ctx->d_counters, d_work, &launches, st, image_wait);
    cudaEventRecord(ctx->ev1, st);
    if (piped && e == cudaSuccess) {
      cudaEventRecord(ctx->lane_done[ln], st);
      ctx->lane_pending[ln] = true;
      cudaEventRecord(t->ev_frame, st);
      t->frame_pending = true;
      ctx->next_lane = ln ^ 1;
    }
  } else {
    target_write_fence(t);
    cudaEventRecord(ctx->ev0, ctx->stream);
    e = pt::launch_render_mega(s->dev, trace_cfg(p, s->dev), path_cfg(p), fc, t->image, ctx->d_counters, d_work,
                               p->min_blocks, ctx->stream);
    launches = 1;
    cudaEventRecord(ctx->ev1, ctx->stream);
  }
  ctx->timed = true;
  if (e != cudaSuccess) {
    if (d_work) cudaFree(d_work);
    return cuda_err(ctx, e, "render");
  }
  ctx->stats.kernel_launches += launches;
  const uint64_t paths = (uint64_t)t->W * t->H * p->spp;
  ctx->stats.paths += paths;
  if (wc) {
    unsigned long long h[8];
    e = cudaMemcpyAsync(h, d_work, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d_work);
    if (e != cudaSuccess) return cuda_err(ctx, e, "work counters");
    std::memset(wc, 0, sizeof(*wc));
    wc->paths = paths;
    wc->rays = h[0];
    wc->tlas_interior = h[1];
    wc->blas_entries = h[2];
    wc->blas_interior = h[3];
    wc->tri_tests = h[4];
    wc->hits = h[5];
    wc->nee = h[6];
    wc->bytes = 32 * wc->rays + 64 * wc->tlas_interior + 196 * wc->blas_entries + 64 * wc->blas_interior +
                52 * wc->tri_tests + 132 * wc->hits + 268 * wc->nee + 32 * paths;
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) == cudaSuccess) ctx->stats.last_render_ms = ms;
  }
  return PULSE_OK;
}

int32_t pulse_render_forward(PulseScene* s, const PulseView* view, PulseTarget* t, uint32_t accumulation_count,
                             const PulseRenderParams* p) {
  return render_impl(s, view, t, accumulation_count, p, nullptr);
}

int32_t pulse_render_count(PulseScene* s, const PulseView* view, PulseTarget* t, uint32_t accumulation_count,
                           const PulseRenderParams* p, PulseWorkCounters* out) {
  if (!out) return PULSE_ERR_INVALID_ARG;
  return render_impl(s, view, t, accumulation_count, p, out);
}

// ---------------------------------------------------------------- realtime GI
void pulse_default_gi_params(PulseRenderParams* p) {
  if (!p) return;
  pulse_default_params(p);
  p->spp = 2;
  p->max_depth = 5;
  p->nee_mode = 1;
  p->light_pick = 0;
}

static cudaError_t grow_gstage(PulseCtx* ctx, size_t bytes) {
  if (ctx->gstage.bytes >= bytes) return cudaSuccess;
  cudaStreamSynchronize(ctx->stream);
  if (ctx->gstage.p) cudaFree(ctx->gstage.p);
  ctx->gstage.p = nullptr;
  ctx->gstage.bytes = 0;
  const cudaError_t e = pt::dev_alloc((void**)&ctx->gstage.p, bytes);
  if (e == cudaSuccess) ctx->gstage.bytes = bytes;
  return e;
}

int32_t pulse_gbuffer_primary(PulseScene* s, const PulseView* view, uint32_t w, uint32_t h,
                              const PulseRenderParams* p, PulseGBufferTexel* dst, uint32_t dst_on_host) {
  if (!s) return PULSE_ERR_INVALID_ARG;
  PulseCtx* ctx = s->ctx;
  if (!view || !dst) return set_err(ctx, PULSE_ERR_INVALID_ARG, "pulse_gbuffer_primary: NULL argument");
  if (int32_t rc = check_params(ctx, p)) return rc;
  if (!s->ready) return set_err(ctx, PULSE_ERR_NOT_READY, "scene has no buffers");
  if (w == 0 || h == 0 || (uint64_t)w * h >= (1ull << 31))
    return set_err(ctx, PULSE_ERR_INVALID_ARG, "pulse_gbuffer_primary: size must be in [1, 2^31) texels");
  if (!dst_on_host && ((uintptr_t)dst & 15u))
    return set_err(ctx, PULSE_ERR_INVALID_ARG, "pulse_gbuffer_primary: device dst must be 16-byte aligned");
  cudaSetDevice(ctx->device);
  quiesce(ctx);
  const size_t bytes = (size_t)w * h * sizeof(PulseGBufferTexel);
  cudaError_t e = dst_on_host ? grow_gstage(ctx, bytes) : cudaSuccess;
  if (e == cudaSuccess) e = grow_wf(ctx, (size_t)w * h);
  if (e != cudaSuccess) return cuda_err(ctx, e, "pulse_gbuffer_primary: buffers");
  float4* out = dst_on_host ? (float4*)ctx->gstage.p : (float4*)dst;
  PulseTarget shape{};
  shape.W = w;
  shape.H = h;
  const pt::WfScene one = pt::wf_scene(s->dev, path_cfg(p), frame_cfg(view, &shape, 0), nullptr);
  uint32_t launches = 0;
  e = pt::wf_gbuffer_primary(trace_cfg(p, s->dev), one, out, p->trace_blocks, pt::wf_carve(ctx->wf.p, (size_t)w * h),
                             ctx->d_counters, &launches, ctx->stream);
  if (e == cudaSuccess && dst_on_host) {
    e = cudaMemcpyAsync(dst, out, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  }
  if (e != cudaSuccess) return cuda_err(ctx, e, "pulse_gbuffer_primary");
  ctx->stats.kernel_launches += launches;
  ctx->stats.rays += (uint64_t)w * h;
  return PULSE_OK;
}

int32_t pulse_render_gi(PulseScene* s, const PulseGBufferTexel* gbuffer, uint32_t gw, uint32_t gh,
                        uint32_t gbuffer_on_host, PulseTarget* t, const PulseRenderParams* p) {
  if (!s || !t) return PULSE_ERR_INVALID_ARG;
  PulseCtx* ctx = s->ctx;
  if (t->ctx != ctx) return set_err(ctx, PULSE_ERR_INVALID_ARG, "target belongs to another context");
  if (!gbuffer) return set_err(ctx, PULSE_ERR_INVALID_ARG, "pulse_render_gi: gbuffer is NULL");
  if (int32_t rc = check_params(ctx, p)) return rc;
  if (!s->ready) return set_err(ctx, PULSE_ERR_NOT_READY, "scene has no buffers");
  if (gw == 0 || gh == 0 || (uint64_t)gw * gh >= (1ull << 31))
    return set_err(ctx, PULSE_ERR_INVALID_ARG, "pulse_render_gi: G-buffer size must be in [1, 2^31) texels");
  if (!gbuffer_on_host && ((uintptr_t)gbuffer & 15u))
    return set_err(ctx, PULSE_ERR_INVALID_ARG, "pulse_render_gi: device G-buffer must be 16-byte aligned");
  cudaSetDevice(ctx->device);
  quiesce(ctx);
  cudaStream_t st = ctx->stream;
  const size_t gbytes = (size_t)gw * gh * sizeof(PulseGBufferTexel);
  const size_t paths = (size_t)t->W * t->H;
  cudaError_t e = gbuffer_on_host ? grow_gstage(ctx, gbytes) : cudaSuccess;
  if (e == cudaSuccess) e = grow_wf(ctx, paths);
  if (e != cudaSuccess) return cuda_err(ctx, e, "pulse_render_gi: buffers");
  const float4* g = (const float4*)gbuffer;
  if (gbuffer_on_host) {
    e = cudaMemcpyAsync(ctx->gstage.p, gbuffer, gbytes, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_err(ctx, e, "pulse_render_gi: G-buffer upload");
    g = (const float4*)ctx->gstage.p;
  }
  pt::PathCfg pc = path_cfg(p);
  pc.nee_mode = 1;
  PulseView none{};
  target_write_fence(t);
  const pt::WfScene one = pt::wf_scene(s->dev, pc, frame_cfg(&none, t, 0), t->image);
  const pt::WfBuffers B = pt::wf_carve(ctx->wf.p, paths);
  uint32_t launches = 0;
  cudaEventRecord(ctx->ev0, st);
  e = pt::wf_render_gi(trace_cfg(p, s->dev), one, g, gw, gh, p->wf_segments, p->trace_blocks, B, ctx->d_counters,
                       &launches, st);
  cudaEventRecord(ctx->ev1, st);
  ctx->timed = true;
  if (e != cudaSuccess) return cuda_err(ctx, e, "pulse_render_gi");
  ctx->stats.kernel_launches += launches;
  ctx->stats.paths += paths * p->spp;
  return PULSE_OK;
}

int32_t pulse_trace(PulseScene* s, const PulseRay* rays, uint32_t n, const PulseRenderParams* p,
                    PulseHitRecord* hits) {
  if (!s || (!rays && n) || (!hits && n)) return PULSE_ERR_INVALID_ARG;
  PulseCtx* ctx = s->ctx;
  if (int32_t rc = check_params(ctx, p)) return rc;
  if (!s->ready) return set_err(ctx, PULSE_ERR_NOT_READY, "scene has no buffers");
  if (n == 0) return PULSE_OK;
  cudaSetDevice(ctx->device);
  quiesce(ctx);
  void* d_rays = nullptr;
  void* d_hits = nullptr;
  cudaError_t e = pt::dev_alloc((void**)&d_rays, (size_t)n * 24);
  if (e == cudaSuccess) e = pt::dev_alloc((void**)&d_hits, (size_t)n * sizeof(pt::Hit));
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_rays, rays, (size_t)n * 24, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess)
    e = pt::launch_trace_rays(s->dev, trace_cfg(p, s->dev), (const float*)d_rays, n, (pt::Hit*)d_hits,
                              ctx->d_counters,
                              ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(hits, d_hits, (size_t)n * sizeof(pt::Hit), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d_rays);
  cudaFree(d_hits);
  if (e != cudaSuccess) return cuda_err(ctx, e, "trace");
  ctx->stats.rays += n;
  ctx->stats.kernel_launches += 1;
  return read_counters(ctx);
}

// ------------------------------------------------------------------ adjoint
int32_t pulse_render_backward(PulseScene* s, const PulseView* view, uint32_t width, uint32_t height,
                              uint32_t sample_count, const PulseRenderParams* p, const float* dloss_dimage,
                              PulseMaterialGrad* grads_out) {
  if (!s) return PULSE_ERR_INVALID_ARG;
  PulseCtx* ctx = s->ctx;
  if (!view || !dloss_dimage || !grads_out)
    return set_err(ctx, PULSE_ERR_INVALID_ARG, "pulse_render_backward: NULL argument");
  if (int32_t rc = check_params(ctx, p)) return rc;
  if (!s->ready) return set_err(ctx, PULSE_ERR_NOT_READY, "scene has no buffers");
  if (p->nee_mode != 2)
    return set_err(ctx, PULSE_ERR_INVALID_ARG, "pulse_render_backward: the adjoint differentiates nee_mode 2");
  if (width == 0 || height == 0 || sample_count == 0)
    return set_err(ctx, PULSE_ERR_INVALID_ARG, "pulse_render_backward: empty image or no samples");
  const uint64_t paths = (uint64_t)width * height * sample_count;
  if (paths >= (1ull << 31)) return set_err(ctx, PULSE_ERR_INVALID_ARG, "pulse_render_backward: over 2^31 paths");
  const uint32_t n_mat = s->counts.material_count;
  std::memset(grads_out, 0, sizeof(PulseMaterialGrad) * n_mat);
  if (n_mat == 0) return PULSE_OK;
  cudaSetDevice(ctx->device);
  quiesce(ctx);
  PulseTarget tgt{};
  tgt.W = width;
  tgt.H = height;
  const pt::FrameCfg fc = frame_cfg(view, &tgt, 0);
  pt::PathCfg pc = path_cfg(p);
  pc.spp = sample_count;  // one primal frame holds every sample
  const size_t img_bytes = (size_t)width * height * 16, grad_bytes = (size_t)n_mat * pt::kGradStride * 4;
  cudaError_t e = grow_wf(ctx, paths);
  if (e != cudaSuccess) return cuda_err(ctx, e, "pulse_render_backward: path buffers");
  const pt::WfBuffers B = pt::wf_carve(ctx->wf.p, paths);
  void* d_img = nullptr;   // dloss/dimage
  void* d_prim = nullptr;  // the primal frame's image
  void* d_grad = nullptr;
  void* d_rec = nullptr;   // per-path adjoint records
  e = pt::dev_alloc((void**)&d_img, img_bytes);
  if (e == cudaSuccess) e = pt::dev_alloc((void**)&d_prim, img_bytes);
  if (e == cudaSuccess) e = pt::dev_alloc((void**)&d_rec, paths * pt::kAdjRecBytes);
  if (e == cudaSuccess) e = pt::dev_alloc((void**)&d_grad, grad_bytes);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_img, dloss_dimage, img_bytes, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_grad, 0, grad_bytes, ctx->stream);
  uint32_t launches = 0;
  if (e == cudaSuccess) {
    cudaEventRecord(ctx->ev0, ctx->stream);
    e = pt::launch_backward(s->dev, trace_cfg(p, s->dev), pc, fc, B, (float4*)d_rec, (float4*)d_prim, p->wf_segments,
                            p->trace_blocks,
                            (const float4*)d_img, (float*)d_grad, n_mat, ctx->d_counters, &launches, ctx->stream);
    cudaEventRecord(ctx->ev1, ctx->stream);
    ctx->timed = true;
  }
  std::vector<float> h((size_t)n_mat * pt::kGradStride);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), d_grad, grad_bytes, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d_img);
  cudaFree(d_prim);
  cudaFree(d_grad);
  cudaFree(d_rec);
  if (e != cudaSuccess) return cuda_err(ctx, e, "pulse_render_backward");
  for (uint32_t m = 0; m < n_mat; ++m) {
    const float* g = h.data() + (size_t)m * pt::kGradStride;
    for (int c = 0; c < 3; ++c) {
      grads_out[m].base_color[c] = g[c];
      grads_out[m].emissive[c] = g[3 + c];
    }
    grads_out[m].roughness = g[6];
  }
  ctx->stats.kernel_launches += launches;
  ctx->stats.paths += 2 * paths;  // primal and adjoint replay
  return PULSE_OK;
}

// ------------------------------------------------------------ batched render
int32_t pulse_render_batch(PulseCtx* ctx, const PulseBatchItem* items, uint32_t n, const PulseRenderParams* p,
                           uint32_t flags) {
  if (!ctx) return PULSE_ERR_INVALID_ARG;
  if (!items || n == 0 || n > pt::kMaxBatch)
    return set_err(ctx, PULSE_ERR_INVALID_ARG, "pulse_render_batch: need 1 to 64 items");
  if (flags & ~PULSE_BATCH_NO_GRAPH) return set_err(ctx, PULSE_ERR_INVALID_ARG, "pulse_render_batch: unknown flags");
  if (int32_t rc = check_params(ctx, p)) return rc;
  std::vector<pt::WfScene> tab(n);
  uint64_t paths = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const PulseBatchItem& it = items[i];
    const std::string at = "pulse_render_batch: item " + std::to_string(i) + ": ";
    if (!it.scene || !it.target) return set_err(ctx, PULSE_ERR_INVALID_ARG, at + "scene or target is NULL");
    if (it.scene->ctx != ctx || it.target->ctx != ctx)
      return set_err(ctx, PULSE_ERR_INVALID_ARG, at + "belongs to another context");
    if (!it.scene->ready) return set_err(ctx, PULSE_ERR_NOT_READY, at + "scene has no buffers");
    if (it.max_depth > 4096) return set_err(ctx, PULSE_ERR_INVALID_ARG, at + "max_depth must be <= 4096");
    for (uint32_t j = 0; j < i; ++j)
      if (items[j].target == it.target) return set_err(ctx, PULSE_ERR_INVALID_ARG, at + "target repeated");
    pt::PathCfg pc = path_cfg(p);
    if (it.max_depth) pc.max_depth = it.max_depth;
    pc.seed = it.seed;
    target_write_fence(it.target);
    tab[i] = pt::wf_scene(it.scene->dev, pc, frame_cfg(&it.view, it.target, it.accumulation_count), it.target->image);
    paths += (uint64_t)it.target->W * it.target->H * p->spp;
  }
  if (paths >= (1ull << 31)) return set_err(ctx, PULSE_ERR_INVALID_ARG, "pulse_render_batch: over 2^31 paths");
  cudaSetDevice(ctx->device);
  quiesce(ctx);
  cudaError_t e = grow_wf(ctx, paths);
  if (e != cudaSuccess) return cuda_err(ctx, e, "pulse_render_batch: wavefront buffers");
  const pt::WfBuffers B = pt::wf_carve(ctx->wf.p, paths);
  e = pt::wf_prepare((int)p->nee_mode);
  if (e != cudaSuccess) return cuda_err(ctx, e, "pulse_render_batch: kernel attributes");
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(ctx->stream, &cap);
  if (e != cudaSuccess) return cuda_err(ctx, e, "pulse_render_batch: stream state");
  // Inside a caller's capture the kernels join the caller's graph directly.
  const bool graph = !(flags & PULSE_BATCH_NO_GRAPH) && cap == cudaStreamCaptureStatusNone;
  uint32_t launches = 0;
  if (!graph) {
    cudaEventRecord(ctx->ev0, ctx->stream);
    e = pt::wf_render((int)p->nee_mode, trace_cfg(p, items[0].scene->dev), tab.data(), n, p->wf_segments,
                      p->trace_blocks, B,
                      ctx->d_counters, nullptr, &launches, ctx->stream);
    cudaEventRecord(ctx->ev1, ctx->stream);
    ctx->timed = cap == cudaStreamCaptureStatusNone;
    if (e != cudaSuccess) return cuda_err(ctx, e, "pulse_render_batch");
  } else {
    e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_err(ctx, e, "pulse_render_batch: begin capture");
    const cudaError_t er = pt::wf_render((int)p->nee_mode, trace_cfg(p, items[0].scene->dev), tab.data(), n,
                                         p->wf_segments,
                                         p->trace_blocks, B, ctx->d_counters, nullptr, &launches, ctx->stream);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(ctx->stream, &g);
    if (er != cudaSuccess || e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return cuda_err(ctx, er != cudaSuccess ? er : e, "pulse_render_batch: capture");
    }
    if (ctx->batch_exec) {
      cudaGraphExecUpdateResultInfo info;
      if (cudaGraphExecUpdate(ctx->batch_exec, g, &info) != cudaSuccess) {
        cudaGetLastError();  // a changed topology: instantiate anew
        cudaGraphExecDestroy(ctx->batch_exec);
        ctx->batch_exec = nullptr;
      }
    }
    if (!ctx->batch_exec) e = cudaGraphInstantiate(&ctx->batch_exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      ctx->batch_exec = nullptr;
      return cuda_err(ctx, e, "pulse_render_batch: instantiate");
    }
    cudaEventRecord(ctx->ev0, ctx->stream);
    e = cudaGraphLaunch(ctx->batch_exec, ctx->stream);
    cudaEventRecord(ctx->ev1, ctx->stream);
    ctx->timed = true;
    if (e != cudaSuccess) return cuda_err(ctx, e, "pulse_render_batch: graph launch");
  }
  ctx->stats.kernel_launches += launches;
  ctx->stats.paths += paths;
  return PULSE_OK;
}

// ---------------------------------------------------------- no-alloc render
// pulse_render_forward_noalloc: the wavefront render with its path buffers in
// g_noalloc_paths, a file-scope device array, instead of the context's
// allocation.  Host code never uses the array's name as an address: each
// device's address comes from cudaGetSymbolAddress, looked up on the first
// call with that device current.
namespace {
constexpr size_t kNoAllocMaxPaths = 65536;
constexpr size_t kNoAllocBytes = kNoAllocMaxPaths * (64 + 16 + 64 + 4 + 4 + 4) + 9 * 256 + 32 * 1024 + 16 * 1024;
static_assert(pt::wf_bytes(kNoAllocMaxPaths) <= kNoAllocBytes, "the fixed path buffer must hold the wavefront layout");
static __device__ __align__(256) unsigned char g_noalloc_paths[kNoAllocBytes];
std::mutex g_noalloc_mu;
constexpr int kNoAllocDevices = 128;
void* g_noalloc_addr[kNoAllocDevices] = {};
}  // namespace

int32_t pulse_render_forward_noalloc(PulseScene* s, const PulseView* view, PulseTarget* t,
                                     uint32_t accumulation_count, const PulseRenderParams* p) {
  if (!s || !view || !t) return PULSE_ERR_INVALID_ARG;
  PulseCtx* ctx = s->ctx;
  if (t->ctx != ctx) return set_err(ctx, PULSE_ERR_INVALID_ARG, "target belongs to another context");
  if (int32_t rc = check_params(ctx, p)) return rc;
  if (!s->ready) return set_err(ctx, PULSE_ERR_NOT_READY, "scene has no buffers");
  const uint64_t paths = (uint64_t)t->W * t->H * p->spp;
  if (paths > kNoAllocMaxPaths)
    return set_err(ctx, PULSE_ERR_INVALID_ARG,
                   "pulse_render_forward_noalloc: width * height * spp = " + std::to_string(paths) +
                       " exceeds the fixed buffer's 65536 paths");
  if (ctx->device < 0 || ctx->device >= kNoAllocDevices)
    return set_err(ctx, PULSE_ERR_INVALID_ARG, "pulse_render_forward_noalloc: device index out of range");
  if (pt::wf_bytes(paths) > kNoAllocBytes) return set_err(ctx, PULSE_ERR_INVALID_ARG, "path buffer layout too large");
  cudaSetDevice(ctx->device);
  quiesce(ctx);
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[ctx->device]) {
      void* ptr = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_paths);
      if (e != cudaSuccess) return cuda_err(ctx, e, "pulse_render_forward_noalloc: device address of the path buffer");
      g_noalloc_addr[ctx->device] = ptr;
    }
    base = g_noalloc_addr[ctx->device];
  }
  const pt::WfBuffers B = pt::wf_carve(base, paths);
  const pt::FrameCfg fc = frame_cfg(view, t, accumulation_count);
  uint32_t launches = 0;
  const pt::WfScene one = pt::wf_scene(s->dev, path_cfg(p), fc, t->image);
  target_write_fence(t);
  cudaEventRecord(ctx->ev0, ctx->stream);
  const cudaError_t e = pt::wf_render((int)p->nee_mode, trace_cfg(p, s->dev), &one, 1, p->wf_segments,
                                      p->trace_blocks, B,
                                      ctx->d_counters, nullptr, &launches, ctx->stream);
  cudaEventRecord(ctx->ev1, ctx->stream);
  ctx->timed = true;
  if (e != cudaSuccess) return cuda_err(ctx, e, "pulse_render_forward_noalloc");
  ctx->stats.kernel_launches += launches;
  ctx->stats.paths += paths;
  return PULSE_OK;
}

}  // extern "C"
