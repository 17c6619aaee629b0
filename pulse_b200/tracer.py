"""Python front end of the C ABI: contexts, scenes, render targets.

These classes are thin owners of the library's handles; every call goes through
``libpulse_cuda.so``.  Errors become ``PulseError`` carrying the library's
status code and message.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _ffi
from .layout import INSTANCE_WORDS, NODE_WORDS, Instance, Material, Mesh, SceneBuffers

DEFAULTS = dict(max_depth=5, spp=1, nee_mode=0, light_pick=0, seed=0, quirks=1, stack_depth=32,
                iter_cap=100000, eps_origin=0.001, eps_tri=0.001, eps_par=1e-4, eps_shadow=0.005,
                kernel=0, block_size=0, min_blocks=0, wf_segments=0, trace_blocks=0, step_policy=0, no_roulette=0,
                ray_sort=0)


class PulseError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ffi.ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


def render_params(**kw) -> _ffi.RenderParams:
    p = _ffi.RenderParams()
    _ffi.load().pulse_default_params(C.byref(p))
    for k, v in kw.items():
        if k in DEFAULTS:
            setattr(p, k, v)
    return p


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Context:
    def __init__(self, device: int = 0):
        self.lib = _ffi.load()
        h = C.c_void_p()
        rc = self.lib.pulse_ctx_create(device, C.byref(h))
        if rc != 0:
            raise PulseError(rc, f"pulse_ctx_create(device={device})")
        self.h = h

    def check(self, rc: int, what: str):
        if rc != 0:
            msg = self.lib.pulse_last_error(self.h)
            raise PulseError(rc, f"{what}: {msg.decode() if msg else ''}")

    def sync(self):
        self.check(self.lib.pulse_sync(self.h), "pulse_sync")

    def set_stream(self, cuda_stream_ptr: int | None):
        """Launch on a caller's cudaStream_t (e.g. torch.cuda.Stream().cuda_stream); None = own stream."""
        self.check(self.lib.pulse_ctx_set_stream(self.h, cuda_stream_ptr or None), "pulse_ctx_set_stream")

    def set_pipeline(self, depth: int):
        """1: every frame on the context's stream; 2: consecutive wavefront
        frames overlap on two streams of the context (pulse_ctx_set_pipeline)."""
        self.check(self.lib.pulse_ctx_set_pipeline(self.h, depth), "pulse_ctx_set_pipeline")

    def stream_ptr(self) -> int:
        """The cudaStream_t the context's work is enqueued on (as an int)."""
        h = C.c_void_p()
        self.check(self.lib.pulse_ctx_get_stream(self.h, C.byref(h)), "pulse_ctx_get_stream")
        return h.value or 0

    def stats(self) -> dict:
        s = _ffi.Stats()
        self.check(self.lib.pulse_get_stats(self.h, C.byref(s)), "pulse_get_stats")
        return s.as_dict()

    def build_blas(self, prims, bins: int = 20, max_leaf: int = 8):
        """Device build_blas: prims (n, 12) f32 -> (nodes (N, 8) u32, tri_indices (n,) u32)."""
        prims = np.ascontiguousarray(prims, dtype=np.float32).reshape(-1, 12)
        n = prims.shape[0]
        nodes = np.zeros((max(2 * n - 1, 1), NODE_WORDS), np.uint32)
        idx = np.zeros(n, np.uint32)
        cnt = C.c_uint32(0)
        bp = _ffi.BvhParams(bins, max_leaf)
        self.check(self.lib.pulse_build_blas(self.h, _ptr(prims), n, C.byref(bp), _ptr(nodes), C.byref(cnt),
                                             _ptr(idx)), "pulse_build_blas")
        return nodes[:cnt.value].copy(), idx

    def build_tlas(self, bounds, bins: int = 2, max_leaf: int = 1):
        """Device build_tlas: bounds (k, 9) f32 -> (nodes, instance_indices)."""
        bounds = np.ascontiguousarray(bounds, dtype=np.float32).reshape(-1, 9)
        k = bounds.shape[0]
        nodes = np.zeros((max(2 * k - 1, 1), NODE_WORDS), np.uint32)
        idx = np.zeros(max(k, 1), np.uint32)
        cnt = C.c_uint32(0)
        bp = _ffi.BvhParams(bins, max_leaf)
        self.check(self.lib.pulse_build_tlas(self.h, _ptr(bounds) if k else None, k, C.byref(bp), _ptr(nodes),
                                             C.byref(cnt), _ptr(idx) if k else None), "pulse_build_tlas")
        return nodes[:cnt.value].copy(), idx[:k].copy()

    def close(self):
        if getattr(self, "h", None):
            self.lib.pulse_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Scene:
    def __init__(self, ctx: Context):
        self.ctx = ctx
        h = C.c_void_p()
        ctx.check(ctx.lib.pulse_scene_create(ctx.h, C.byref(h)), "pulse_scene_create")
        self.h = h

    def set_buffers(self, sb: SceneBuffers):
        arrs = [np.ascontiguousarray(a) for a in sb.arrays()]
        prim, tdata, tidx, blas, tlas, iidx, inst, mats, scdf, tcdf, areas, lidx = arrs
        b = _ffi.SceneBuffersC(
            sb.instance_count, sb.light_count, prim.shape[0] if prim.ndim else 0, tidx.size, blas.shape[0],
            tlas.shape[0], iidx.size, mats.shape[0], tcdf.size, 0,
            *[a.ctypes.data if a.size else None for a in arrs])
        self.ctx.check(self.ctx.lib.pulse_scene_set_buffers(self.h, C.byref(b)), "pulse_scene_set_buffers")

    def upload_mesh(self, mesh: Mesh, bins: int = 20, max_leaf: int = 8) -> int:
        """prepare_extracted_mesh_assets on the device: soup + BLAS; returns the mesh id."""
        mid = C.c_uint32(0)
        bp = _ffi.BvhParams(bins, max_leaf)
        self.ctx.check(self.ctx.lib.pulse_mesh_upload(self.h, _ptr(mesh.positions), _ptr(mesh.normals),
                                                      _ptr(mesh.uvs), mesh.positions.shape[0], _ptr(mesh.indices),
                                                      mesh.indices.size, C.byref(bp), C.byref(mid)),
                       "pulse_mesh_upload")
        return mid.value

    def remove_mesh(self, mesh_id: int):
        self.ctx.check(self.ctx.lib.pulse_mesh_remove(self.h, mesh_id), "pulse_mesh_remove")

    def set_materials(self, materials):
        rows = np.ascontiguousarray(np.stack([m.to_words() for m in materials]) if len(materials)
                                    else np.zeros((0, 12), np.float32), dtype=np.float32)
        self.ctx.check(self.ctx.lib.pulse_materials_set(self.h, _ptr(rows) if rows.size else None, rows.shape[0]),
                       "pulse_materials_set")

    def set_instances(self, instances, mesh_ids, tlas_bins: int = 2, tlas_leaf: int = 1):
        """prepare_mesh_instances + TLAS build on the device.  ``instances`` are
        layout.Instance whose ``mesh`` indexes ``mesh_ids``."""
        arr = (_ffi.InstanceDesc * max(len(instances), 1))()
        for i, inst in enumerate(instances):
            arr[i].object_world[:] = [float(x) for x in inst.columns()]
            arr[i].mesh_id = mesh_ids[inst.mesh]
            arr[i].material_index = inst.material
        bp = _ffi.BvhParams(tlas_bins, tlas_leaf)
        self.ctx.check(self.ctx.lib.pulse_instances_set(self.h, arr, len(instances), C.byref(bp)),
                       "pulse_instances_set")

    def update_instances(self, indices, object_world, tlas_bins: int | None = None, tlas_leaf: int = 1):
        """Move instances ``indices`` (rows of the last ``set_instances``) to
        the column-major 4x4 transforms ``object_world`` (k x 16); records,
        bounds and TLAS are rebuilt on the device, the light list is kept."""
        idx = np.ascontiguousarray(indices, dtype=np.uint32).reshape(-1)
        mats = np.ascontiguousarray(object_world, dtype=np.float32).reshape(idx.size, 16)
        bp = _ffi.BvhParams(tlas_bins, tlas_leaf) if tlas_bins is not None else None
        self.ctx.check(self.ctx.lib.pulse_instances_update(self.h, _ptr(idx) if idx.size else None,
                                                           _ptr(mats) if idx.size else None, idx.size,
                                                           C.byref(bp) if bp is not None else None),
                       "pulse_instances_update")

    def counts(self) -> dict:
        b = _ffi.SceneBuffersC()
        self.ctx.check(self.ctx.lib.pulse_scene_counts(self.h, C.byref(b)), "pulse_scene_counts")
        return {n: getattr(b, n) for n, t in b._fields_ if t is C.c_uint32}

    def download(self) -> SceneBuffers:
        """The scene's 13 bind-group buffers, copied to host arrays."""
        c = self.counts()
        sb = SceneBuffers(
            instance_count=c["instance_count"], light_count=c["light_count"],
            primitives=np.zeros((c["primitive_count"], 12), np.float32),
            triangle_data=np.zeros((c["primitive_count"], 20), np.float32),
            triangle_indices=np.zeros(c["triangle_index_count"], np.uint32),
            blas_nodes=np.zeros((c["blas_node_count"], NODE_WORDS), np.uint32),
            tlas_nodes=np.zeros((c["tlas_node_count"], NODE_WORDS), np.uint32),
            instance_indices=np.zeros(c["instance_index_count"], np.uint32),
            instances=np.zeros((c["instance_count"], INSTANCE_WORDS), np.uint32),
            materials=np.zeros((c["material_count"], 12), np.float32),
            light_emission_strength_cdf=np.zeros(c["light_count"], np.float32),
            light_triangle_area_cdfs=np.zeros(c["light_cdf_count"], np.float32),
            light_mesh_areas=np.zeros(c["light_count"], np.float32),
            light_indices=np.zeros((c["light_count"], 2), np.uint32))
        b = _ffi.SceneBuffersC(c["instance_count"], c["light_count"], c["primitive_count"],
                               c["triangle_index_count"], c["blas_node_count"], c["tlas_node_count"],
                               c["instance_index_count"], c["material_count"], c["light_cdf_count"], 0,
                               *[a.ctypes.data if a.size else None for a in sb.arrays()])
        self.ctx.check(self.ctx.lib.pulse_scene_download(self.h, C.byref(b)), "pulse_scene_download")
        return sb

    def trace(self, rays, **params) -> np.ndarray:
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
        out = np.zeros(rays.shape[0], dtype=_ffi.HIT_DTYPE)
        p = render_params(**params)
        self.ctx.check(self.ctx.lib.pulse_trace(self.h, _ptr(rays), rays.shape[0], C.byref(p), _ptr(out)),
                       "pulse_trace")
        return out

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.pulse_scene_destroy(self.h)
            self.h = None


class Target:
    def __init__(self, ctx: Context, width: int, height: int):
        self.ctx = ctx
        self.width, self.height = width, height
        h = C.c_void_p()
        ctx.check(ctx.lib.pulse_target_create(ctx.h, width, height, C.byref(h)), "pulse_target_create")
        self.h = h

    def download(self, out=None) -> np.ndarray:
        if out is None:
            out = np.empty((self.height, self.width, 4), dtype=np.float32)
        self.ctx.check(self.ctx.lib.pulse_target_download(self.h, _ptr(out)), "pulse_target_download")
        return out

    def upload(self, image: np.ndarray):
        """Restore the target's texels (H, W, 4) float32, e.g. a saved accumulation."""
        img = np.ascontiguousarray(image, dtype=np.float32)
        assert img.shape == (self.height, self.width, 4)
        self.ctx.check(self.ctx.lib.pulse_target_upload(self.h, _ptr(img)), "pulse_target_upload")

    def resample(self, out_w: int, out_h: int, filter: int = 0) -> np.ndarray:
        """pulse_target_resample to host memory: (out_h, out_w, 4) float16."""
        out = np.empty((out_h, out_w, 4), dtype=np.float16)
        self.ctx.check(self.ctx.lib.pulse_target_resample(self.h, out_w, out_h, filter, _ptr(out), 1),
                       "pulse_target_resample")
        return out

    def device_ptr(self) -> int:
        p = C.c_void_p()
        self.ctx.check(self.ctx.lib.pulse_target_device_ptr(self.h, C.byref(p)), "pulse_target_device_ptr")
        return p.value

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.pulse_target_destroy(self.h)
            self.h = None


def make_view(view) -> _ffi.ViewC:
    v = _ffi.ViewC()
    v.inverse_view_proj[:] = [float(x) for x in np.asarray(view.inverse_view_proj, dtype=np.float32)]
    v.world_position[:] = [float(x) for x in np.asarray(view.world_position, dtype=np.float32)]
    return v


def render_count(scene: Scene, view, target: Target, accumulation_count: int = 0, **params) -> dict:
    """render_forward in the counting instantiation: returns the device-counted work."""
    v = make_view(view)
    p = render_params(**params)
    w = _ffi.WorkCounters()
    ctx = scene.ctx
    ctx.check(ctx.lib.pulse_render_count(scene.h, C.byref(v), target.h, accumulation_count, C.byref(p), C.byref(w)),
              "pulse_render_count")
    return w.as_dict()


def render_forward(scene: Scene, view, target: Target, accumulation_count: int = 0, **params):
    v = make_view(view)
    p = render_params(**params)
    ctx = scene.ctx
    ctx.check(ctx.lib.pulse_render_forward(scene.h, C.byref(v), target.h, accumulation_count, C.byref(p)),
              "pulse_render_forward")


def gi_params(**kw) -> _ffi.RenderParams:
    """pulse_default_gi_params (the realtime GI pass's spp 2, max_depth 5,
    uniform light pick) with the given overrides."""
    p = _ffi.RenderParams()
    _ffi.load().pulse_default_gi_params(C.byref(p))
    for k, v in kw.items():
        if k in DEFAULTS:
            setattr(p, k, v)
    return p


def gbuffer_primary(scene: Scene, view, width: int, height: int, out=None, **params):
    """The primary-hit G-buffer of ``view``: a (height, width, 16) float32
    host array, or written into ``out`` (a CUDA tensor of that many floats)."""
    v = make_view(view)
    p = render_params(**params)
    ctx = scene.ctx
    if out is None:
        host = np.zeros((height, width, 16), np.float32)
        ctx.check(ctx.lib.pulse_gbuffer_primary(scene.h, C.byref(v), width, height, C.byref(p), _ptr(host), 1),
                  "pulse_gbuffer_primary")
        return host
    assert out.numel() >= width * height * 16 and out.is_cuda
    ctx.check(ctx.lib.pulse_gbuffer_primary(scene.h, C.byref(v), width, height, C.byref(p),
                                            C.c_void_p(out.data_ptr()), 0), "pulse_gbuffer_primary")
    return out


def render_gi(scene: Scene, gbuffer, target: Target, gw: int | None = None, gh: int | None = None, **params):
    """The realtime GI pass into ``target`` from ``gbuffer``: a (gh, gw, 16)
    float32 host array, or a CUDA tensor with gw and gh given."""
    p = gi_params(**params)
    ctx = scene.ctx
    if isinstance(gbuffer, np.ndarray):
        gb = np.ascontiguousarray(gbuffer, dtype=np.float32)
        gh, gw = gb.shape[0], gb.shape[1]
        rc = ctx.lib.pulse_render_gi(scene.h, _ptr(gb), gw, gh, 1, target.h, C.byref(p))
    else:
        rc = ctx.lib.pulse_render_gi(scene.h, C.c_void_p(gbuffer.data_ptr()), gw, gh, 0, target.h, C.byref(p))
    ctx.check(rc, "pulse_render_gi")


class BatchItem:
    """One scene of a batched frame (see render_batch)."""

    def __init__(self, scene: Scene, view, target: Target, accumulation_count: int = 0, max_depth: int = 0,
                 seed: int = 0):
        self.scene, self.view, self.target = scene, view, target
        self.accumulation_count, self.max_depth, self.seed = accumulation_count, max_depth, seed


def render_batch(ctx: Context, items, graph: bool = True, **params):
    """pulse_render_batch: every item's scene rendered into its target in one
    wavefront frame (a CUDA graph unless graph=False).  Item max_depth 0 takes
    params' max_depth; the item seed replaces params' seed."""
    items = list(items)
    arr = (_ffi.BatchItem * max(1, len(items)))()
    for a, it in zip(arr, items):
        a.scene = it.scene.h
        a.target = it.target.h
        a.view = make_view(it.view)
        a.accumulation_count = it.accumulation_count
        a.max_depth = it.max_depth
        a.seed = it.seed
    p = render_params(**params)
    flags = 0 if graph else _ffi.PULSE_BATCH_NO_GRAPH
    ctx.check(ctx.lib.pulse_render_batch(ctx.h, arr, len(items), C.byref(p), flags), "pulse_render_batch")


def render_backward(scene: Scene, view, width: int, height: int, sample_count: int, dloss_dimage, **params):
    """pulse_render_backward: (material_count, 7) float32 gradients
    [base rgb, emissive rgb, roughness] of the loss whose dloss/dimage
    (H x W x 4 float32) is given, for the image that is the mean of
    sample_count samples per texel (nee_mode 2)."""
    g = np.ascontiguousarray(np.asarray(dloss_dimage, dtype=np.float32).reshape(height, width, 4))
    n_mat = scene.counts()["material_count"]
    out = (_ffi.MaterialGrad * max(1, n_mat))()
    p = render_params(**dict(params, nee_mode=2))
    v = make_view(view)
    ctx = scene.ctx
    ctx.check(ctx.lib.pulse_render_backward(scene.h, C.byref(v), width, height, sample_count, C.byref(p),
                                            g.ctypes.data_as(C.c_void_p), out), "pulse_render_backward")
    arr = np.frombuffer(out, dtype=np.float32).reshape(-1, 8)[:n_mat, :7]
    return arr.copy()
