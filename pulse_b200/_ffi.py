"""ctypes bindings of ``include/pulse_cuda.h`` (the library's C ABI).

The shared library is built in-tree (``pulse_b200/libpulse_cuda.so``) by
``pulse_b200.build``; importing this module without it raises, there is no
fallback path.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libpulse_cuda.so"

PULSE_OK = 0
PULSE_ERR_INVALID_ARG = -1
PULSE_ERR_CUDA = -2
PULSE_ERR_OOM = -3
PULSE_ERR_ITER_CAP = -4
PULSE_ERR_STACK_OVERFLOW = -5
PULSE_ERR_NOT_READY = -6
PULSE_ERR_DEGENERATE = -7
PULSE_ERR_NO_DEVICE = -8

ERROR_NAMES = {0: "PULSE_OK", -1: "PULSE_ERR_INVALID_ARG", -2: "PULSE_ERR_CUDA", -3: "PULSE_ERR_OOM",
               -4: "PULSE_ERR_ITER_CAP", -5: "PULSE_ERR_STACK_OVERFLOW", -6: "PULSE_ERR_NOT_READY",
               -7: "PULSE_ERR_DEGENERATE", -8: "PULSE_ERR_NO_DEVICE"}


class RenderParams(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("max_depth", "spp", "nee_mode", "light_pick", "seed", "quirks",
                                          "stack_depth", "iter_cap")] + \
               [(n, C.c_float) for n in ("eps_origin", "eps_tri", "eps_par", "eps_shadow")] + \
               [(n, C.c_uint32) for n in ("kernel", "block_size", "min_blocks", "wf_segments", "trace_blocks",
                                          "step_policy", "no_roulette", "ray_sort")]


class BvhParams(C.Structure):
    _fields_ = [("bins", C.c_uint32), ("max_leaf", C.c_uint32)]


class SceneBuffersC(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("instance_count", "light_count", "primitive_count",
                                          "triangle_index_count", "blas_node_count", "tlas_node_count",
                                          "instance_index_count", "material_count", "light_cdf_count", "pad")] + \
               [(n, C.c_void_p) for n in ("primitives", "triangle_data", "triangle_indices", "blas_nodes",
                                          "tlas_nodes", "instance_indices", "instances", "materials",
                                          "light_emission_strength_cdf", "light_triangle_area_cdfs",
                                          "light_mesh_areas", "light_indices")]


class InstanceDesc(C.Structure):
    _fields_ = [("object_world", C.c_float * 16), ("mesh_id", C.c_uint32), ("material_index", C.c_uint32),
                ("pad", C.c_uint32 * 2)]


class ViewC(C.Structure):
    _fields_ = [("inverse_view_proj", C.c_float * 16), ("world_position", C.c_float * 3), ("pad", C.c_float)]


class BatchItem(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("target", C.c_void_p), ("view", ViewC), ("accumulation_count", C.c_uint32),
                ("max_depth", C.c_uint32), ("seed", C.c_uint32), ("pad", C.c_uint32)]


class MaterialGrad(C.Structure):
    _fields_ = [("base_color", C.c_float * 3), ("emissive", C.c_float * 3), ("roughness", C.c_float),
                ("pad", C.c_float)]


PULSE_BATCH_MAX = 64
PULSE_BATCH_NO_GRAPH = 1


class Stats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("paths", "rays", "iter_cap_hits", "stack_overflows", "kernel_launches",
                                          "reserved")] + \
               [(n, C.c_float) for n in ("last_render_ms", "last_build_ms", "last_upload_ms", "pad")]

    def as_dict(self):
        return {n: (getattr(self, n)) for n, _ in self._fields_ if n not in ("pad", "reserved")}


class WorkCounters(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("paths", "rays", "tlas_interior", "blas_entries", "blas_interior",
                                          "tri_tests", "hits", "nee", "bytes", "reserved")]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n, _ in self._fields_ if n != "reserved"}


HIT_DTYPE = [("t", "<f4"), ("instance_index", "<u4"), ("triangle_index", "<u4"), ("u", "<f4"), ("v", "<f4")]

# Every entry point of include/pulse_cuda.h with its ctypes signature.
P = C.c_void_p
SIGNATURES = {
    "pulse_ctx_create": (C.c_int32, [C.c_int32, C.POINTER(C.c_void_p)]),
    "pulse_ctx_destroy": (C.c_int32, [P]),
    "pulse_last_error": (C.c_char_p, [P]),
    "pulse_sync": (C.c_int32, [P]),
    "pulse_get_stats": (C.c_int32, [P, C.POINTER(Stats)]),
    "pulse_default_params": (None, [C.POINTER(RenderParams)]),
    "pulse_ctx_set_stream": (C.c_int32, [P, P]),
    "pulse_ctx_get_stream": (C.c_int32, [P, C.POINTER(C.c_void_p)]),
    "pulse_ctx_set_pipeline": (C.c_int32, [P, C.c_uint32]),
    "pulse_debug_fail_allocations": (C.c_int32, [C.c_uint32]),
    "pulse_scene_create": (C.c_int32, [P, C.POINTER(C.c_void_p)]),
    "pulse_scene_destroy": (C.c_int32, [P]),
    "pulse_scene_set_buffers": (C.c_int32, [P, C.POINTER(SceneBuffersC)]),
    "pulse_target_create": (C.c_int32, [P, C.c_uint32, C.c_uint32, C.POINTER(C.c_void_p)]),
    "pulse_target_destroy": (C.c_int32, [P]),
    "pulse_target_device_ptr": (C.c_int32, [P, C.POINTER(C.c_void_p)]),
    "pulse_target_download": (C.c_int32, [P, P]),
    "pulse_target_download_async": (C.c_int32, [P, P]),
    "pulse_target_download_wait": (C.c_int32, [P]),
    "pulse_target_upload": (C.c_int32, [P, P]),
    "pulse_target_resample": (C.c_int32, [P, C.c_uint32, C.c_uint32, C.c_uint32, P, C.c_uint32]),
    "pulse_render_forward": (C.c_int32, [P, C.POINTER(ViewC), P, C.c_uint32, C.POINTER(RenderParams)]),
    "pulse_render_count": (C.c_int32, [P, C.POINTER(ViewC), P, C.c_uint32, C.POINTER(RenderParams),
                                       C.POINTER(WorkCounters)]),
    "pulse_render_forward_noalloc": (C.c_int32, [P, C.POINTER(ViewC), P, C.c_uint32, C.POINTER(RenderParams)]),
    "pulse_render_batch": (C.c_int32, [P, C.POINTER(BatchItem), C.c_uint32, C.POINTER(RenderParams), C.c_uint32]),
    "pulse_render_backward": (C.c_int32, [P, C.POINTER(ViewC), C.c_uint32, C.c_uint32, C.c_uint32,
                                          C.POINTER(RenderParams), P, P]),
    "pulse_trace": (C.c_int32, [P, P, C.c_uint32, C.POINTER(RenderParams), P]),
    "pulse_gbuffer_primary": (C.c_int32, [P, C.POINTER(ViewC), C.c_uint32, C.c_uint32, C.POINTER(RenderParams), P,
                                          C.c_uint32]),
    "pulse_render_gi": (C.c_int32, [P, P, C.c_uint32, C.c_uint32, C.c_uint32, P, C.POINTER(RenderParams)]),
    "pulse_default_gi_params": (None, [C.POINTER(RenderParams)]),
    "pulse_build_blas": (C.c_int32, [P, P, C.c_uint32, C.POINTER(BvhParams), P, C.POINTER(C.c_uint32), P]),
    "pulse_build_tlas": (C.c_int32, [P, P, C.c_uint32, C.POINTER(BvhParams), P, C.POINTER(C.c_uint32), P]),
    "pulse_mesh_upload": (C.c_int32, [P, P, P, P, C.c_uint32, P, C.c_uint32, C.POINTER(BvhParams),
                                      C.POINTER(C.c_uint32)]),
    "pulse_mesh_remove": (C.c_int32, [P, C.c_uint32]),
    "pulse_materials_set": (C.c_int32, [P, P, C.c_uint32]),
    "pulse_instances_set": (C.c_int32, [P, P, C.c_uint32, C.POINTER(BvhParams)]),
    "pulse_instances_update": (C.c_int32, [P, P, P, C.c_uint32, C.POINTER(BvhParams)]),
    "pulse_scene_counts": (C.c_int32, [P, C.POINTER(SceneBuffersC)]),
    "pulse_scene_download": (C.c_int32, [P, C.POINTER(SceneBuffersC)]),
}

_lib = None


def load():
    """Load the library and bind every declared entry point (raises if absent)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m pulse_b200.build`")
        lib = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib
