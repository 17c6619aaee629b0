// api.cu -- the extern "C" entry points declared in include/pulse_cuda.h.
//
// Host side of the drop-in boundary: contexts, scenes (device copies of the
// scene bind group plus derived layouts), render targets, validation of
// untrusted scene buffers before any kernel reads them, and launches.
#include <algorithm>
#include <array>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pulse_cuda.h"
#include "kernels.h"

struct PulseCtx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  pt::Counters* d_counters = nullptr;
  PulseStats stats{};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
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

}  // namespace

struct PulseScene {
  PulseCtx* ctx = nullptr;
  bool ready = false;
  uint32_t counts[10] = {0};
  DevBuf primitives, triangle_data, triangle_indices, blas_nodes, tlas_nodes, instance_indices, instances,
      materials, strength_cdf, tri_cdfs, mesh_areas, light_indices, inst_light, tri_bvh;
  pt::DevScene dev{};

  void free_all() {
    for (DevBuf* b : {&primitives, &triangle_data, &triangle_indices, &blas_nodes, &tlas_nodes, &instance_indices,
                      &instances, &materials, &strength_cdf, &tri_cdfs, &mesh_areas, &light_indices, &inst_light,
                      &tri_bvh}) {
      if (b->p) cudaFree(b->p);
      b->p = nullptr;
      b->bytes = 0;
    }
    ready = false;
  }
};

struct PulseTarget {
  PulseCtx* ctx = nullptr;
  uint32_t W = 0, H = 0;
  float4* image = nullptr;
};

namespace {

cudaError_t upload(DevBuf& b, const void* host, size_t bytes, cudaStream_t st) {
  if (b.p) { cudaFree(b.p); b.p = nullptr; }
  b.bytes = bytes;
  const size_t alloc = bytes ? bytes : 16;
  cudaError_t e = cudaMalloc(&b.p, alloc);
  if (e != cudaSuccess) { b.p = nullptr; return e; }
  if (bytes) return cudaMemcpyAsync(b.p, host, bytes, cudaMemcpyHostToDevice, st);
  return cudaMemsetAsync(b.p, 0, alloc, st);
}

// ---------------------------------------------------------------- validation
// Checks that every index a kernel will follow stays inside its buffer and that
// every BVH reachable from a root is a tree (a node reached twice is rejected),
// so device traversal never leaves its buffers; its loops are additionally
// bounded by the iteration cap as in the reference.
std::string validate(const PulseSceneBuffers* b) {
  const uint32_t K = b->instance_count, L = b->light_count, P = b->primitive_count, TI = b->triangle_index_count,
                 BN = b->blas_node_count, TN = b->tlas_node_count, II = b->instance_index_count,
                 M = b->material_count, C = b->light_cdf_count;
  if (P && (!b->primitives || !b->triangle_data)) return "primitives/triangle_data missing";
  if (TI && !b->triangle_indices) return "triangle_indices missing";
  if (BN && !b->blas_nodes) return "blas_nodes missing";
  if (TN == 0 || !b->tlas_nodes) return "tlas_nodes missing (an empty scene still has the invalid root node)";
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
    std::vector<uint32_t> stack{0};
    while (!stack.empty()) {
      const uint64_t g = no + stack.back();
      stack.pop_back();
      if (g >= BN) return "mesh at node_offset " + std::to_string(no) + ": BLAS node out of range";
      if (mark[g] == walk) return "mesh at node_offset " + std::to_string(no) + ": BLAS is not a tree";
      mark[g] = walk;
      const PulseBvhNode& nd = b->blas_nodes[g];
      if (nd.count > 0) {
        if ((uint64_t)nd.a + nd.count > tc) return "mesh at node_offset " + std::to_string(no) + ": BLAS leaf out of range";
      } else {
        if (no + (uint64_t)nd.a + 1 >= BN) return "mesh at node_offset " + std::to_string(no) + ": BLAS child out of range";
        stack.push_back(nd.a + 1);
        stack.push_back(nd.a);
      }
    }
  }
  // TLAS.
  {
    std::vector<uint8_t> tseen(TN, 0);
    const PulseBvhNode& r = b->tlas_nodes[0];
    if (!(r.a == 0 && r.count == 0)) {
      std::vector<uint32_t> stack{0};
      while (!stack.empty()) {
        const uint64_t n = stack.back();
        stack.pop_back();
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
          stack.push_back(nd.a + 1);
          stack.push_back(nd.a);
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
  return PULSE_OK;
}

pt::TraceCfg trace_cfg(const PulseRenderParams* p) {
  pt::TraceCfg t;
  t.stack_depth = p->stack_depth;
  t.iter_cap = p->iter_cap;
  t.eps_tri = p->eps_tri;
  t.eps_par = p->eps_par;
  t.quirks = p->quirks != 0;
  return t;
}
pt::PathCfg path_cfg(const PulseRenderParams* p) {
  pt::PathCfg c;
  c.max_depth = p->max_depth;
  c.spp = p->spp;
  c.nee_mode = p->nee_mode;
  c.light_pick = p->light_pick;
  c.seed = p->seed;
  c.eps_origin = p->eps_origin;
  c.eps_shadow = p->eps_shadow;
  c.quirks = p->quirks != 0;
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
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&c->d_counters, sizeof(pt::Counters));
  if (e == cudaSuccess) e = cudaMemset(c->d_counters, 0, sizeof(pt::Counters));
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
  if (e != cudaSuccess) {
    if (c->stream) cudaStreamDestroy(c->stream);
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
  cudaStreamSynchronize(ctx->stream);
  cudaFree(ctx->d_counters);
  cudaEventDestroy(ctx->ev0);
  cudaEventDestroy(ctx->ev1);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return PULSE_OK;
}

const char* pulse_last_error(const PulseCtx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int32_t pulse_sync(PulseCtx* ctx) {
  if (!ctx) return PULSE_ERR_INVALID_ARG;
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? PULSE_OK : cuda_err(ctx, e, "sync");
}

int32_t pulse_get_stats(const PulseCtx* ctx, PulseStats* out) {
  if (!ctx || !out) return PULSE_ERR_INVALID_ARG;
  *out = ctx->stats;
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
  cudaStreamSynchronize(s->ctx->stream);
  s->free_all();
  delete s;
  return PULSE_OK;
}

int32_t pulse_scene_set_buffers(PulseScene* s, const PulseSceneBuffers* b) {
  if (!s || !b) return PULSE_ERR_INVALID_ARG;
  PulseCtx* ctx = s->ctx;
  const std::string why = validate(b);
  if (!why.empty()) return set_err(ctx, PULSE_ERR_INVALID_ARG, "scene buffers: " + why);
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  cudaStreamSynchronize(st);
  s->free_all();
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
  std::vector<int32_t> inst_light(K ? K : 1, -1);
  for (uint32_t l = 0; l < L; ++l) {
    const uint32_t ii = b->light_indices[l].mesh_instance_index;
    if (inst_light[ii] < 0) inst_light[ii] = (int32_t)l;
  }
  up(s->inst_light, inst_light.data(), inst_light.size() * 4);
  if (e == cudaSuccess) {
    s->tri_bvh.bytes = (size_t)b->triangle_index_count * 48;
    e = cudaMalloc(&s->tri_bvh.p, s->tri_bvh.bytes ? s->tri_bvh.bytes : 16);
    if (e != cudaSuccess) s->tri_bvh.p = nullptr;
  }
  if (e == cudaSuccess) {
    // One gather per distinct mesh range referenced by an instance.
    std::vector<uint64_t> done;
    for (uint32_t i = 0; i < K && e == cudaSuccess; ++i) {
      const PulseMeshInstance& in = b->instances[i];
      const uint64_t key = ((uint64_t)in.index_offset << 32) | in.triangle_offset;
      bool dup = false;
      for (uint64_t d : done) dup |= d == key;
      if (dup) continue;
      done.push_back(key);
      e = pt::launch_gather_tri_bvh((const float4*)s->primitives.p, (const uint32_t*)s->triangle_indices.p,
                                    (float4*)s->tri_bvh.p, in.triangle_offset, in.index_offset, in.triangle_count,
                                    st);
    }
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    s->free_all();
    return cuda_err(ctx, e, "scene upload");
  }
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
  d.instance_count = K;
  d.light_count = L;
  s->ready = true;
  return PULSE_OK;
}

int32_t pulse_target_create(PulseCtx* ctx, uint32_t W, uint32_t H, PulseTarget** out) {
  if (!ctx || !out || W == 0 || H == 0 || (uint64_t)W * H > (1ull << 31)) return PULSE_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  PulseTarget* t = new PulseTarget();
  t->ctx = ctx;
  t->W = W;
  t->H = H;
  cudaError_t e = cudaMalloc(&t->image, (size_t)W * H * 16);
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
  cudaStreamSynchronize(t->ctx->stream);
  cudaFree(t->image);
  delete t;
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
  cudaError_t e = cudaMemcpyAsync(host, t->image, (size_t)t->W * t->H * 16, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? PULSE_OK : cuda_err(ctx, e, "target download");
}

int32_t pulse_render_forward(PulseScene* s, const PulseView* view, PulseTarget* t, uint32_t accumulation_count,
                             const PulseRenderParams* p) {
  if (!s || !view || !t) return PULSE_ERR_INVALID_ARG;
  PulseCtx* ctx = s->ctx;
  if (t->ctx != ctx) return set_err(ctx, PULSE_ERR_INVALID_ARG, "target belongs to another context");
  if (int32_t rc = check_params(ctx, p)) return rc;
  if (!s->ready) return set_err(ctx, PULSE_ERR_NOT_READY, "scene has no buffers");
  cudaSetDevice(ctx->device);
  pt::FrameCfg fc;
  const float* m = view->inverse_view_proj;
  fc.ivp = pt::M4{make_float4(m[0], m[1], m[2], m[3]), make_float4(m[4], m[5], m[6], m[7]),
                  make_float4(m[8], m[9], m[10], m[11]), make_float4(m[12], m[13], m[14], m[15])};
  fc.eye = make_float3(view->world_position[0], view->world_position[1], view->world_position[2]);
  fc.W = t->W;
  fc.H = t->H;
  fc.acc = accumulation_count;
  cudaEventRecord(ctx->ev0, ctx->stream);
  cudaError_t e = pt::launch_render_mega(s->dev, trace_cfg(p), path_cfg(p), fc, t->image, ctx->d_counters,
                                         ctx->stream);
  cudaEventRecord(ctx->ev1, ctx->stream);
  if (e != cudaSuccess) return cuda_err(ctx, e, "render");
  ctx->stats.paths += (uint64_t)t->W * t->H * p->spp;
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
  void* d_rays = nullptr;
  void* d_hits = nullptr;
  cudaError_t e = cudaMalloc(&d_rays, (size_t)n * 24);
  if (e == cudaSuccess) e = cudaMalloc(&d_hits, (size_t)n * sizeof(pt::Hit));
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_rays, rays, (size_t)n * 24, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess)
    e = pt::launch_trace_rays(s->dev, trace_cfg(p), (const float*)d_rays, n, (pt::Hit*)d_hits, ctx->d_counters,
                              ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(hits, d_hits, (size_t)n * sizeof(pt::Hit), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d_rays);
  cudaFree(d_hits);
  if (e != cudaSuccess) return cuda_err(ctx, e, "trace");
  ctx->stats.rays += n;
  return read_counters(ctx);
}

}  // extern "C"
