"""Python front end of the C ABI: contexts, scenes, render targets.

These classes are thin owners of the library's handles; every call goes through
``libpulse_cuda.so``.  Errors become ``PulseError`` carrying the library's
status code and message.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _ffi
from .layout import SceneBuffers

DEFAULTS = dict(max_depth=5, spp=1, nee_mode=0, light_pick=0, seed=0, quirks=1, stack_depth=32,
                iter_cap=100000, eps_origin=0.001, eps_tri=0.001, eps_par=1e-4, eps_shadow=0.005,
                kernel=0, block_size=0)


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

    def stats(self) -> dict:
        s = _ffi.Stats()
        self.check(self.lib.pulse_get_stats(self.h, C.byref(s)), "pulse_get_stats")
        return s.as_dict()

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


def render_forward(scene: Scene, view, target: Target, accumulation_count: int = 0, **params):
    v = make_view(view)
    p = render_params(**params)
    ctx = scene.ctx
    ctx.check(ctx.lib.pulse_render_forward(scene.h, C.byref(v), target.h, accumulation_count, C.byref(p)),
              "pulse_render_forward")
