/*
 * pulse_cuda.h -- C ABI of the B200 (sm_100a) path-tracing library that stands
 * in for the WGSL/wgpu hot path of rubengrim/pulse.
 *
 * The reference's Rust plugin systems keep their names and schedule; where they
 * built wgpu bind groups and dispatched WGSL they call these entry points.  Each
 * declaration names the reference interface it replaces (paths are relative to
 * the reference project).
 *
 * Conventions
 *   - Every entry point returns int32_t: PULSE_OK (0) or a negative PULSE_ERR_*.
 *     Nothing aborts or traps; pulse_last_error() gives a message.
 *   - Host pointers passed in are read during the call only (the library
 *     copies).  The library owns all device memory.
 *   - One PulseCtx per render thread, one CUDA stream per context (and two
 *     internal ones for pipelined frames, pulse_ctx_set_pipeline); calls are
 *     asynchronous on that stream except downloads and pulse_sync().
 *   - Struct layouts below are the std430 layouts of src/scene/types.wgsl:3-74
 *     (what encase writes for the Rust structs in src/scene/mod.rs), so Rust
 *     Vec<T> of the reference's types can be passed without conversion.
 */
#ifndef PULSE_CUDA_H
#define PULSE_CUDA_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define PULSE_API __attribute__((visibility("default")))
#else
#define PULSE_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
#define PULSE_OK 0
#define PULSE_ERR_INVALID_ARG -1
#define PULSE_ERR_CUDA -2
#define PULSE_ERR_OOM -3
#define PULSE_ERR_ITER_CAP -4
#define PULSE_ERR_STACK_OVERFLOW -5
#define PULSE_ERR_NOT_READY -6
#define PULSE_ERR_DEGENERATE -7
#define PULSE_ERR_NO_DEVICE -8

/* ------------------------------------------------------- std430 row types */
/* PulsePrimitive, src/scene/mod.rs:344-347 / types.wgsl:23-27 (48 B). */
typedef struct { float p0[3]; float pad0; float p1[3]; float pad1; float p2[3]; float pad2; } PulsePrimitive;
/* PulseTriangleData, src/scene/mod.rs:338-342 / types.wgsl:29-36 (80 B). */
typedef struct {
  float n0[3]; float pad0; float n1[3]; float pad1; float n2[3]; float pad2;
  float uv0[2]; float uv1[2]; float uv2[2]; float pad3[2];
} PulseTriangleData;
/* PulseBLASNode / PulseTLASNode, src/scene/blas.rs:5-13, src/scene/tlas.rs:4-10 (32 B).
 * count > 0: leaf over [a, a+count); count == 0: interior with children a, a+1. */
typedef struct { float aabb_min[3]; uint32_t a; float aabb_max[3]; uint32_t count; } PulseBvhNode;
/* PulseMeshInstance, src/scene/mod.rs:527-533 / types.wgsl:52-60 (160 B).
 * Matrices are column-major (glam / WGSL mat4x4f). */
typedef struct {
  float object_world[16];
  float world_object[16];
  uint32_t triangle_offset, triangle_count, index_offset, node_offset, material_index;
  uint32_t pad[3];
} PulseMeshInstance;
/* PulseMaterial, src/scene/mod.rs:240-247 / types.wgsl:62-68 (48 B). */
typedef struct {
  float base_color[4];
  float emissive[4];
  float perceptual_roughness, reflectance, metallic, pad;
} PulseMaterial;
/* PulseLightDataIndex, src/scene/mod.rs:547-551 (8 B). */
typedef struct { uint32_t cdf_offset, mesh_instance_index; } PulseLightDataIndex;

/* The scene bind group: SceneUniform + 13 storage buffers
 * (src/scene/bindings.wgsl:14-28, written by queue_scene_bind_group,
 * src/scene/mod.rs:911-1090).  Counts are in rows. */
typedef struct {
  uint32_t instance_count;          /* SceneUniform.instance_count; rows of instances      */
  uint32_t light_count;             /* SceneUniform.light_count; rows of the 3 light arrays */
  uint32_t primitive_count;         /* rows of primitives and triangle_data                 */
  uint32_t triangle_index_count;
  uint32_t blas_node_count;
  uint32_t tlas_node_count;
  uint32_t instance_index_count;
  uint32_t material_count;
  uint32_t light_cdf_count;         /* length of light_triangle_area_cdfs */
  uint32_t pad;
  const PulsePrimitive* primitives;
  const PulseTriangleData* triangle_data;
  const uint32_t* triangle_indices;
  const PulseBvhNode* blas_nodes;
  const PulseBvhNode* tlas_nodes;
  const uint32_t* instance_indices;
  const PulseMeshInstance* instances;
  const PulseMaterial* materials;
  const float* light_emission_strength_cdf;
  const float* light_triangle_area_cdfs;
  const float* light_mesh_areas;
  const PulseLightDataIndex* light_indices;
} PulseSceneBuffers;

/* Bevy's View uniform fields the tracer reads (path_tracer.wgsl:70-73). */
typedef struct {
  float inverse_view_proj[16]; /* column-major */
  float world_position[3];
  float pad;
} PulseView;

/* Render knobs; pulse_default_params() fills the reference's constants
 * (max_depth 5 path_tracer.wgsl:80, stack 32 / iteration cap 100000
 * utilities.wgsl:134-137, epsilons utilities.wgsl:437,452,518,523). */
typedef struct {
  uint32_t max_depth;   /* bounces (path_trace: traced segments)                         */
  uint32_t spp;         /* samples per pixel per call; sample index = acc*spp + s         */
  uint32_t nee_mode;    /* 0 path_trace (no NEE), 1 diffuse NEE estimator, 2 corrected NEE+MIS */
  uint32_t light_pick;  /* 0 uniform (reference), 1 emission-strength CDF                 */
  uint32_t seed;        /* added as seed*0x9E3779B9 to the RNG state; 0 = reference stream */
  uint32_t quirks;      /* 1 reproduce the reference's FP32 quirks, 0 fix them            */
  uint32_t stack_depth; /* traversal stack entries per level (<= 64)                      */
  uint32_t iter_cap;    /* traversal loop cap per level                                   */
  float eps_origin;     /* secondary-ray origin offset along the normal                   */
  float eps_tri;        /* ray/triangle t lower bound                                     */
  float eps_par;        /* ray/triangle parallel threshold                                */
  float eps_shadow;     /* shadow test slack                                              */
  uint32_t kernel;      /* 0 auto (wavefront), 1 megakernel, 2 wavefront                  */
  uint32_t block_size;  /* wavefront: threads per block of the persistent traversal
                           kernels, 0 auto (128) or 64 (same threads per SM, same
                           register budget)                                       */
  uint32_t min_blocks;  /* register budget: 0 auto, else 4, 6 or 8 resident blocks per SM */
  uint32_t wf_segments; /* wavefront: segments traced as separate kernels before one
                           persistent kernel finishes the remaining paths; 0 auto (3;
                           2 for pulse_render_gi),
                           0xffffffff: no separate segments (the persistent kernel
                           runs every path from its primary ray)                      */
  uint32_t trace_blocks; /* wavefront: resident traversal blocks per SM, 0 auto (8), <= 8 */
  uint32_t step_policy;  /* wavefront traversal: which action a warp's step performs.
                            0 auto; 1 every lane its own (divergent); else one weight
                            byte per action, node | tri << 8 | enter << 16 | leave << 24:
                            the action with the largest lane count x weight runs   */
  uint32_t no_roulette;  /* 1: no Russian roulette (paths end at max_depth or a miss; the
                            roulette's random number is still drawn, so the sample
                            stream is unchanged); makes the image a smooth function
                            of the material parameters for finite differences       */
  uint32_t ray_sort;     /* wavefront: 1 reorders each bounce's queue of live paths by
                            ray direction octant and origin cell before it is traced
                            (results unchanged), 0 keeps the shading order          */
} PulseRenderParams;

/* Binned-SAH build knobs; reference values {20, 8} for BLAS (src/scene/blas.rs:96, :193)
 * and {2, 1} for the TLAS (src/scene/tlas.rs:73, :192). */
typedef struct { uint32_t bins, max_leaf; } PulseBvhParams;

/* One world-space ray and its closest-hit record (RayHitRecord, types.wgsl:8-21). */
typedef struct { float origin[3]; float dir[3]; } PulseRay;
typedef struct { float t; uint32_t instance_index, triangle_index; float u, v; } PulseHitRecord;

typedef struct {
  uint64_t paths, rays, iter_cap_hits, stack_overflows;
  uint64_t kernel_launches; /* kernels this context has launched */
  uint64_t reserved;
  float last_render_ms, last_build_ms, last_upload_ms, pad;
} PulseStats;

/* Work of the reference algorithm during one render, counted by the device:
 * traced rays, TLAS interior visits, BLAS entries, BLAS interior visits,
 * triangle tests, closest hits shaded, NEE samples with a shadow ray, and the
 * algorithmic bytes they imply:
 *   per ray  32 (TLAS root) + 64 per TLAS interior visit (two child nodes)
 *            + 196 per BLAS entry (instance index 4, instance 160, BLAS root 32)
 *            + 64 per BLAS interior visit + 52 per triangle test (index 4, primitive 48)
 *   per hit  132 (triangle index 4, triangle data 80, material 48)
 *   per NEE  268 (light index 8, instance 160, primitive 48, area 4, material 48)
 *   per path 32  (accumulation texel read + write). */
typedef struct {
  uint64_t paths, rays, tlas_interior, blas_entries, blas_interior, tri_tests, hits, nee;
  uint64_t bytes;
  uint64_t reserved;
} PulseWorkCounters;

typedef struct PulseCtx PulseCtx;
typedef struct PulseScene PulseScene;
typedef struct PulseTarget PulseTarget;

/* ---------------------------------------------------------------- context */
/* Replaces the wgpu RenderDevice/RenderQueue pair the plugin renders through. */
PULSE_API int32_t pulse_ctx_create(int32_t device, PulseCtx** out);
PULSE_API int32_t pulse_ctx_destroy(PulseCtx* ctx);
PULSE_API const char* pulse_last_error(const PulseCtx* ctx);
PULSE_API int32_t pulse_sync(PulseCtx* ctx);
PULSE_API int32_t pulse_get_stats(const PulseCtx* ctx, PulseStats* out);
PULSE_API void pulse_default_params(PulseRenderParams* out);
/* Run this context's work on a caller-owned CUDA stream (a cudaStream_t; NULL
 * returns to the context's own stream).  No reference counterpart: wgpu owns
 * its queue; a CUDA host application passes its stream here. */
PULSE_API int32_t pulse_ctx_set_stream(PulseCtx* ctx, void* cuda_stream);
/* The CUDA stream this context's work is enqueued on (the caller's stream
 * given to pulse_ctx_set_stream, else the context's own non-blocking stream),
 * as a cudaStream_t in *out.  A caller that reads a target's device image on
 * another stream (a collective over pulse_target_device_ptr, for instance)
 * orders itself after the library's work through it: the stream waits, from
 * this call on, for the pipelined frames in flight as well
 * (pulse_ctx_set_pipeline).  No reference counterpart: wgpu orders its queue
 * itself. */
PULSE_API int32_t pulse_ctx_get_stream(const PulseCtx* ctx, void** out);
/* Frame pipelining (no reference counterpart: wgpu schedules its queue
 * itself).  depth 2: each wavefront pulse_render_forward (without work
 * counters) runs on one of two streams of the context, alternating, each with
 * its own path buffers, so frame k+1's first launches fill the SMs that frame
 * k's last, draining launches leave idle; accumulation into a target keeps the
 * frames' order, and images are those of depth 1 bit for bit.  The context's
 * stream does not wait for such a frame: every other call of the library
 * waits for the frames in flight first, except pulse_instances_set's
 * double-buffered update and pulse_target_download_async, which wait for
 * what they use only.  A consumer outside the library (a device pointer from
 * pulse_target_device_ptr) orders itself through pulse_ctx_get_stream, called
 * after the frames it reads were queued.  depth 1 (the default) queues every
 * frame on the context's stream. */
PULSE_API int32_t pulse_ctx_set_pipeline(PulseCtx* ctx, uint32_t depth);

/* Testing aid for hosts' out-of-memory handling (no reference counterpart):
 * the library's next n device allocations, in any context of the process,
 * fail as if the device were full -- the calls that make them return
 * PULSE_ERR_OOM after releasing what they hold, and every context stays
 * usable.  n = 0 disarms.  Nothing is allocated or faulted on the device. */
PULSE_API int32_t pulse_debug_fail_allocations(uint32_t n);

/* ------------------------------------------------------------------ scene */
PULSE_API int32_t pulse_scene_create(PulseCtx* ctx, PulseScene** out);
PULSE_API int32_t pulse_scene_destroy(PulseScene* scene);

/* Raw bind-group upload: replaces queue_scene_bind_group (src/scene/mod.rs:911-1090),
 * i.e. the 13 create_storage_buffer calls plus the SceneUniform.  The buffers are
 * validated (every index in range, trees acyclic) before they reach the GPU. */
PULSE_API int32_t pulse_scene_set_buffers(PulseScene* scene, const PulseSceneBuffers* buffers);

/* Scene-preparation path (the reference's prepare systems, src/scene/mod.rs:372-742,
 * run on the GPU).  Meshes are triangle-soup-extracted and their BLAS built on
 * upload; pulse_instances_set does the per-frame work of prepare_mesh_instances:
 * instance records with inverse transforms, world bounds, light CDFs, TLAS. */
typedef struct {
  float object_world[16];  /* column-major GlobalTransform::compute_matrix() */
  uint32_t mesh_id;        /* from pulse_mesh_upload                          */
  uint32_t material_index; /* row of the array given to pulse_materials_set   */
  uint32_t pad[2];
} PulseInstanceDesc;

/* build_blas (src/scene/blas.rs:44-87) as a device kernel: prims (n rows) ->
 * nodes (capacity 2n-1) + tri_indices (n), bit-identical to the CPU builder.
 * Host arrays in and out; PULSE_ERR_DEGENERATE where the reference's partition
 * loop would panic (blas.rs:114-121). */
PULSE_API int32_t pulse_build_blas(PulseCtx* ctx, const PulsePrimitive* prims, uint32_t n,
                                   const PulseBvhParams* params, PulseBvhNode* nodes_out, uint32_t* node_count,
                                   uint32_t* tri_indices_out);
/* build_tlas (src/scene/tlas.rs:29-65) over PulsePrimitiveMeshInstance
 * {bounds_min, bounds_max, center} (n x 9 floats, src/scene/mod.rs:535-539);
 * n == 0 gives the single invalid root node (tlas.rs:30-35). */
PULSE_API int32_t pulse_build_tlas(PulseCtx* ctx, const float* bounds9, uint32_t n, const PulseBvhParams* params,
                                   PulseBvhNode* nodes_out, uint32_t* node_count, uint32_t* instance_indices_out);

/* prepare_extracted_mesh_assets (src/scene/mod.rs:372-448) for one mesh:
 * POSITION f32x3, NORMAL f32x3, UV_0 f32x2 per vertex and a u32 index buffer.
 * A mesh has fewer than 2^29 triangles (and a scene fewer than 2^29
 * instances; pulse_scene_set_buffers checks the same), so every tree has
 * fewer than 2^30 nodes; PULSE_ERR_INVALID_ARG otherwise. */
PULSE_API int32_t pulse_mesh_upload(PulseScene* scene, const float* positions, const float* normals, const float* uvs,
                                    uint32_t vertex_count, const uint32_t* indices, uint32_t index_count,
                                    const PulseBvhParams* params, uint32_t* mesh_id);
PULSE_API int32_t pulse_mesh_remove(PulseScene* scene, uint32_t mesh_id);
/* prepare_material_data (src/scene/mod.rs:279-297).  On a scene prepared by
 * pulse_instances_set the instance records, light list and light CDFs are
 * rebuilt as well (they follow the materials' emission, src/scene/mod.rs:583-622);
 * if the last instances use a material index beyond the new list, the scene is
 * not ready until the next pulse_instances_set.  With pulse_scene_set_buffers
 * the light buffers stay the caller's and n must cover every material index
 * the instances use (PULSE_ERR_INVALID_ARG otherwise). */
PULSE_API int32_t pulse_materials_set(PulseScene* scene, const PulseMaterial* materials, uint32_t n);
/* prepare_mesh_instances (src/scene/mod.rs:561-697) + the TLAS build, every frame.
 * Returns once the new records, light CDFs and TLAS are on the device; from a
 * scene's second call on (no mesh, material or buffer change since the last
 * one, at most 1024 instances) they are written into a second buffer set on a
 * stream of the scene's own, so renders already queued keep reading the
 * previous set and may still be running when the call returns; renders queued
 * afterwards read the new one. */
PULSE_API int32_t pulse_instances_set(PulseScene* scene, const PulseInstanceDesc* instances, uint32_t n,
                                      const PulseBvhParams* tlas_params);
/* Incremental form of the per-frame rebuild of src/scene/mod.rs:561-697 for a
 * frame in which only transforms changed: instance indices[k] (rows of the
 * last pulse_instances_set) gets object_world[16k..16k+15] (column-major).
 * Only those records and bounds are recomputed; the light list and CDFs stay
 * (they are in object space, src/scene/mod.rs:700-742) and the TLAS is rebuilt
 * over all bounds with the last TLAS parameters, or tlas_params when given.
 * The scene equals, bit for bit, the one pulse_instances_set makes from the
 * updated list.  PULSE_ERR_NOT_READY unless the scene was prepared by
 * pulse_instances_set with no mesh upload or removal since;
 * PULSE_ERR_INVALID_ARG for an index out of range or repeated. */
PULSE_API int32_t pulse_instances_update(PulseScene* scene, const uint32_t* indices, const float* object_world,
                                         uint32_t n, const PulseBvhParams* tlas_params);
/* Row counts of the scene's 13 buffers (pointers in *out are set to NULL). */
PULSE_API int32_t pulse_scene_counts(PulseScene* scene, PulseSceneBuffers* out);
/* Blocking copy of the scene's buffers into host arrays: every non-NULL
 * pointer of *dst is a destination with room for the counts pulse_scene_counts
 * reports. */
PULSE_API int32_t pulse_scene_download(PulseScene* scene, const PulseSceneBuffers* dst);

/* ------------------------------------------------------------------ frame */
/* Render target of W x H rgba32float texels (PulsePathTracerRenderTarget,
 * src/path_tracer/mod.rs:120-166). */
PULSE_API int32_t pulse_target_create(PulseCtx* ctx, uint32_t width, uint32_t height, PulseTarget** out);
PULSE_API int32_t pulse_target_destroy(PulseTarget* target);
/* Device address of the float4 accumulation texels (row-major, W*H*16 bytes). */
PULSE_API int32_t pulse_target_device_ptr(const PulseTarget* target, void** out);
/* Upscaling hand-off (src/path_tracer/pt_upscaling/node.rs:29-96 reads this
 * texture): blocking copy of W*H*4 floats to host memory. */
PULSE_API int32_t pulse_target_download(PulseTarget* target, float* host_rgba);
/* The same copy without blocking (no reference counterpart: a real-time host
 * reads frame k back while frame k+1 traces): enqueued after the work already
 * on the context's stream, it runs on a copy stream of the target's own, and
 * host_rgba holds the texels once pulse_target_download_wait returns.  Only
 * the next write of the image waits for the copy -- for pulse_render_forward
 * with the wavefront kernels that is its last kernel (the accumulation), so
 * the copy overlaps the next frame's tracing.  host_rgba should be pinned
 * (cudaHostAlloc / cudaHostRegister) for the copy to run asynchronously, and
 * must not be read or reused before the wait. */
PULSE_API int32_t pulse_target_download_async(PulseTarget* target, float* host_rgba);
PULSE_API int32_t pulse_target_download_wait(PulseTarget* target);
/* Resume of an accumulation (no reference counterpart: the reference keeps it
 * in a cached texture and restarts on motion, src/path_tracer/mod.rs:107-118):
 * blocking copy of W*H*4 floats from host memory into the target.  A frame
 * saved with pulse_target_download and its accumulation count continues with
 * pulse_render_forward(..., count, ...) exactly as if never interrupted. */
PULSE_API int32_t pulse_target_upload(PulseTarget* target, const float* host_rgba);
/* The upscaling pass itself (pt_upscaling.wgsl:40-50 with wgpu's default
 * sampler, node.rs:70-77): the target resampled to out_w x out_h RGBA16F texels
 * (8 bytes each, row-major), output texel (x, y) sampling the target at
 * ((x + 0.5) / out_w, (y + 0.5) / out_h); filter 0 nearest (the reference's
 * sampler), 1 bilinear (clamp to edge).  dst is device memory (stream-ordered,
 * no synchronisation) or, with dst_on_host = 1, host memory (blocking; the
 * target keeps a staging buffer).  The raster blit is replaced by this kernel:
 * no graphics API is involved. */
PULSE_API int32_t pulse_target_resample(PulseTarget* target, uint32_t out_w, uint32_t out_h, uint32_t filter,
                                        void* dst, uint32_t dst_on_host);

/* One PulsePathTracerNode::run (src/path_tracer/node.rs:40-119): the
 * path_trace dispatch (path_tracer.wgsl:58-124) for every texel of the target,
 * with the running-mean accumulation; accumulation_count == 0 resets. */
PULSE_API int32_t pulse_render_forward(PulseScene* scene, const PulseView* view, PulseTarget* target,
                             uint32_t accumulation_count, const PulseRenderParams* params);

/* pulse_render_forward with the device counting the reference algorithm's work
 * (same image result; a separate, slower kernel instantiation). */
PULSE_API int32_t pulse_render_count(PulseScene* scene, const PulseView* view, PulseTarget* target,
                                     uint32_t accumulation_count, const PulseRenderParams* params,
                                     PulseWorkCounters* out);

/* pulse_render_forward for callers that cannot allocate device memory: the
 * same wavefront render, with its path buffers in a fixed static device array
 * instead of memory the library allocates.  No counterpart in the reference.
 * Meant for hosts that reserve all GPU memory up front -- a game engine with a
 * fixed memory budget, or a real-time frame loop where cudaMalloc/cudaFree
 * would synchronize the device and stall the frame.
 *   - Limit: W * H * spp <= 65536 paths per call (e.g. 256 x 256 at 1 spp);
 *     larger calls return PULSE_ERR_INVALID_ARG.  The array (about 10 MB) is
 *     held on every GPU that loads the library until the process exits.
 *   - The first call on a device looks up the array's device address; make
 *     that first call before any stream capture.
 *   - Every call uses the same array: calls whose GPU work overlaps (other
 *     streams, other contexts on the same device) race; serialize them.
 *   - params->kernel is ignored (always the wavefront kernels). */
PULSE_API int32_t pulse_render_forward_noalloc(PulseScene* scene, const PulseView* view, PulseTarget* target,
                                               uint32_t accumulation_count, const PulseRenderParams* params);

/* One scene of a batched frame: its camera, target and accumulation count,
 * its bounce limit and its RNG seed (both as in PulseRenderParams). */
typedef struct {
  PulseScene* scene;
  PulseTarget* target;
  PulseView view;
  uint32_t accumulation_count;
  uint32_t max_depth; /* 0 = params->max_depth */
  uint32_t seed;
  uint32_t pad;
} PulseBatchItem;

#define PULSE_BATCH_MAX 64
#define PULSE_BATCH_NO_GRAPH 1u /* flags: enqueue the kernels directly, no CUDA graph */

/* Renders n <= PULSE_BATCH_MAX scenes of one context in one wavefront frame:
 * the paths of all items share the same launches (one id space, each kernel
 * finds a path's scene in a table), so small scenes fill the GPU together and
 * the long path tails of every scene overlap.  The frame is captured as a CUDA
 * graph and replayed; the context keeps the instantiated graph and updates it
 * in place while the batch's composition (item count, bounce limits) stays the
 * same.  Each item's image is bit-identical to pulse_render_forward of that
 * item alone with max_depth and seed taken from the item.  Every target
 * appears at most once.  No reference counterpart: the reference renders one
 * camera per render-graph node run (src/path_tracer/node.rs:40-119). */
PULSE_API int32_t pulse_render_batch(PulseCtx* ctx, const PulseBatchItem* items, uint32_t n,
                                     const PulseRenderParams* params, uint32_t flags);

/* Gradient of a loss with respect to one material's parameters (the fields of
 * PulseMaterial: base_color rgb, emissive rgb, perceptual_roughness). */
typedef struct {
  float base_color[3];
  float emissive[3];
  float roughness;
  float pad;
} PulseMaterialGrad;

/* Path-replay adjoint of the corrected estimator (params->nee_mode 2): given
 * dloss/dimage (host, float4 per texel, width x height) of the image that is
 * the mean of sample_count samples per texel -- the image pulse_render_forward
 * accumulates over frames 0 .. F-1 at spp s has sample_count F*s, with the same
 * view and params -- writes the gradient of the loss for every material of the
 * scene to grads_out (material_count rows).  Every path is computed twice from
 * its RNG seed: the primal frame (its radiance is all that is kept, 16 bytes
 * per path in the context's path buffers) and the adjoint replay; sampling is
 * detached, so the result is an unbiased estimate of the gradient of the
 * expected image's loss.  params->no_roulette 1 makes the seeded estimator a
 * smooth function of the albedos (for finite-difference checks).  No
 * reference counterpart (the reference renders only); it is the
 * differentiable addition of this library. */
PULSE_API int32_t pulse_render_backward(PulseScene* scene, const PulseView* view, uint32_t width, uint32_t height,
                                        uint32_t sample_count, const PulseRenderParams* params,
                                        const float* dloss_dimage, PulseMaterialGrad* grads_out);

/* ------------------------------------------------------------ realtime GI */
/* One texel of the G-buffer the realtime GI pass reads: the PbrInput fields
 * src/pulse/gi.wgsl:67-83 uses (world position, world normal, base color,
 * emissive), decoded.  64 bytes; a device array is 16-byte aligned. */
typedef struct {
  float world_position[3];
  uint32_t valid; /* 0: no surface at this texel (its GI output is 0) */
  float world_normal[3];
  float pad0;
  float base_color[3];
  float pad1;
  float emissive[3];
  float pad2;
} PulseGBufferTexel;

/* Our own primary-hit buffer in place of Bevy's deferred G-buffer
 * (src/pulse/gi.wgsl:61-67 reads prepass depth + deferred texture): the closest
 * hit of each texel's camera ray (src/path_tracer/path_tracer.wgsl:63-75) with
 * the interpolated world normal and its material's colors
 * (path_tracer.wgsl:89-100); a miss gives valid 0.  dst holds w*h texels in
 * device memory (dst_on_host 0) or host memory (1). */
PULSE_API int32_t pulse_gbuffer_primary(PulseScene* scene, const PulseView* view, uint32_t w, uint32_t h,
                                        const PulseRenderParams* params, PulseGBufferTexel* dst,
                                        uint32_t dst_on_host);
/* The realtime GI pass (src/pulse/node.rs:24-127 dispatching
 * src/pulse/gi.wgsl:56-135) into the target (the reference's gi_output):
 * for texel (x, y) of the W x H target, params->spp samples of the diffuse
 * estimator start at G-buffer texel (u32(x / W * gw), u32(y / H * gh)): a
 * cosine-sampled bounce, the direct light there, then up to params->max_depth
 * diffuse bounces with NEE and Russian roulette.  The samples share one random
 * state seeded pixel * 5817321 (+ params->seed * 0x9E3779B9); the texel is
 * overwritten with (mean, 1).  The reference's pass is spp 2, max_depth 5,
 * light_pick 0 (pulse_default_gi_params); nee_mode is not read (the pass has
 * its own estimator).  gbuffer: gw*gh texels in device memory
 * (gbuffer_on_host 0) or host memory (1). */
PULSE_API int32_t pulse_render_gi(PulseScene* scene, const PulseGBufferTexel* gbuffer, uint32_t gw, uint32_t gh,
                                  uint32_t gbuffer_on_host, PulseTarget* target, const PulseRenderParams* params);
/* pulse_default_params with the realtime GI pass's constants
 * (src/pulse/gi.wgsl:68, :81): spp 2, max_depth 5, uniform light pick. */
PULSE_API void pulse_default_gi_params(PulseRenderParams* out);

/* Closest-hit query of world rays (trace_ray, src/utilities.wgsl:112-114):
 * host arrays in and out, n rays. */
PULSE_API int32_t pulse_trace(PulseScene* scene, const PulseRay* rays, uint32_t n, const PulseRenderParams* params,
                    PulseHitRecord* hits_out);

#ifdef __cplusplus
}
#endif
#endif /* PULSE_CUDA_H */
