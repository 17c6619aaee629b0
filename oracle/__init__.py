"""ctypes front end of the CPU oracle (``oracle/pulse_oracle.cpp``).

Test infrastructure only: imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline / reference legs of ``bench.py`` as the checker, never by
the product library.

The reference (a Rust/WGSL Bevy plugin) cannot be built or run here, so every
result is "parity unpinned" against the reference's own outputs; the oracle is
pinned by hand-derived known answers instead (tests/test_oracle_kat.py).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from pulse_b200.layout import (INSTANCE_WORDS, NODE_WORDS, Mesh, SceneBuffers, triangle_soup)

HERE = Path(__file__).resolve().parent
SRC = HERE / "pulse_oracle.cpp"
LIB = HERE / "liboracle.so"
CXXFLAGS = ["-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared"]


def build(force: bool = False) -> Path:
    """Compile the oracle with g++ (FP contraction off, IEEE math)."""
    if force or not LIB.exists() or LIB.stat().st_mtime < SRC.stat().st_mtime:
        tmp = LIB.with_suffix(".so.tmp")
        subprocess.check_call(["g++", *CXXFLAGS, "-o", str(tmp), str(SRC)])
        os.replace(tmp, LIB)
    return LIB


class Params(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("max_depth", "spp", "nee_mode", "light_pick", "seed", "quirks",
                                          "stack_depth", "iter_cap")] + \
               [(n, C.c_float) for n in ("eps_origin", "eps_tri", "eps_par", "eps_shadow")] + \
               [(n, C.c_uint32) for n in ("kernel", "block_size", "min_blocks", "wf_segments", "trace_blocks",
                                          "step_policy", "no_roulette")]


# Reference values of every knob (src/path_tracer/path_tracer.wgsl:80, src/utilities.wgsl:137,
# :134, :437, :452, :518, :523).
DEFAULTS = dict(max_depth=5, spp=1, nee_mode=0, light_pick=0, seed=0, quirks=1, stack_depth=32,
                iter_cap=100000, eps_origin=0.001, eps_tri=0.001, eps_par=1e-4, eps_shadow=0.005,
                kernel=0, block_size=0, min_blocks=0, wf_segments=0, trace_blocks=0, step_policy=0, no_roulette=0)


def make_params(**kw) -> Params:
    d = dict(DEFAULTS)
    for k, v in kw.items():
        if k in d:
            d[k] = v
    d["stack_depth"] = min(int(d["stack_depth"]), 256)
    return Params(**d)


class Scene(C.Structure):
    _fields_ = [("instance_count", C.c_uint32), ("light_count", C.c_uint32)] + \
               [(n, C.c_void_p) for n in ("primitives", "triangle_data", "triangle_indices", "blas_nodes",
                                          "tlas_nodes", "instance_indices", "instances", "materials",
                                          "light_emission_strength_cdf", "light_triangle_area_cdfs",
                                          "light_mesh_areas", "light_indices")]


class Stats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("rays", "tlas_interior", "blas_entries", "blas_interior",
                                          "tri_tests", "hits", "nee", "cdf_reads", "iter_cap_hits",
                                          "stack_overflows", "paths")]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


_lib = None


def lib():
    global _lib
    if _lib is None:
        if SRC.exists():
            build()
        L = C.CDLL(str(LIB))
        P = C.c_void_p
        L.oracle_build_blas.argtypes = [P, C.c_uint32, C.c_uint32, C.c_uint32, P, P, P]
        L.oracle_build_tlas.argtypes = [P, C.c_uint32, C.c_uint32, C.c_uint32, P, P, P]
        L.oracle_prepare_instances.argtypes = [C.c_uint32, P, P, P, P, C.c_uint32, P, P, P, P, P, P, P, P, P]
        L.oracle_trace.argtypes = [P, P, C.c_uint32, P, P, P, P, P, P, P, C.c_int]
        L.oracle_render.argtypes = [P, P, P, C.c_uint32, C.c_uint32, C.c_uint32, P, C.c_int, P, C.c_uint32, P, P,
                                    C.c_int]
        L.oracle_gbuffer_primary.argtypes = [P, P, P, C.c_uint32, C.c_uint32, P, P, C.c_int]
        L.oracle_render_gi.argtypes = [P, P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, P, P, C.c_uint32, P, P,
                                       C.c_int]
        L.oracle_render_mean64.argtypes = [P, P, P, C.c_uint32, C.c_uint32, C.c_uint32, P, P, C.c_uint32, P,
                                           C.c_int, P, C.c_int]
        L.oracle_path_log.argtypes = [P, P, P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, P, P,
                                      C.c_uint32, P, P]
        L.oracle_backward.argtypes = [P, P, P, C.c_uint32, C.c_uint32, C.c_uint32, P, P, C.c_uint32, P, C.c_int]
        L.oracle_eval_g_grad.argtypes = [P, P, P, P, P]
        L.oracle_rand_u.argtypes = [P]
        L.oracle_rand_u.restype = C.c_uint32
        L.oracle_rand_f.argtypes = [P]
        L.oracle_rand_f.restype = C.c_float
        L.oracle_sincos.argtypes = [C.c_float, P, P]
        L.oracle_cdf_walk.argtypes = [P, C.c_uint32, C.c_uint32, C.c_float]
        L.oracle_cdf_walk.restype = C.c_uint32
        L.oracle_ray_aabb.argtypes = [P, P, P, P, C.c_float]
        L.oracle_ray_aabb.restype = C.c_float
        L.oracle_ray_triangle.argtypes = [P, P, P, P]
        L.oracle_inverse4.argtypes = [P, P]
        L.oracle_importance_sample.argtypes = [P, P, P, P, C.c_int, P, P]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


# ------------------------------------------------------------------ build --
def build_blas(prims, bins: int = 20, max_leaf: int = 8):
    """src/scene/blas.rs:44 -> (nodes (N,8) u32, tri_indices (n,) u32)."""
    prims = _c(prims, np.float32)
    n = prims.shape[0]
    nodes = np.zeros((max(2 * n - 1, 1), NODE_WORDS), dtype=np.uint32)
    idx = np.zeros(n, dtype=np.uint32)
    cnt = np.zeros(1, dtype=np.uint32)
    rc = lib().oracle_build_blas(_p(prims), n, bins, max_leaf, _p(nodes), _p(cnt), _p(idx))
    if rc != 0:
        raise RuntimeError(f"oracle_build_blas failed: {rc}")
    return nodes[:cnt[0]].copy(), idx


def build_tlas(bounds, bins: int = 2, max_leaf: int = 1):
    """src/scene/tlas.rs:29; bounds (k, 9) = bounds_min, bounds_max, center."""
    bounds = _c(bounds, np.float32).reshape(-1, 9)
    k = bounds.shape[0]
    nodes = np.zeros((max(2 * k - 1, 1), NODE_WORDS), dtype=np.uint32)
    idx = np.zeros(max(k, 1), dtype=np.uint32)
    cnt = np.zeros(1, dtype=np.uint32)
    rc = lib().oracle_build_tlas(_p(bounds), k, bins, max_leaf, _p(nodes), _p(cnt), _p(idx))
    if rc != 0:
        raise RuntimeError(f"oracle_build_tlas failed: {rc}")
    return nodes[:cnt[0]].copy(), idx[:k].copy()


def inverse4(cols16):
    src = _c(cols16, np.float32).reshape(16)
    dst = np.zeros(16, dtype=np.float32)
    lib().oracle_inverse4(_p(src), _p(dst))
    return dst


def prepare_instances(object_world_cols, mesh_index, material_index, materials, primitives, blas_nodes,
                      tlas_bins: int = 2, tlas_leaf: int = 1):
    """src/scene/mod.rs:561-697: instances, light arrays, world bounds, TLAS."""
    ow = _c(object_world_cols, np.float32).reshape(-1, 16)
    k = ow.shape[0]
    mi = _c(mesh_index, np.uint32).reshape(-1, 4)
    mat = _c(material_index, np.uint32).reshape(-1)
    mats = _c(materials, np.float32).reshape(-1, 12)
    prims = _c(primitives, np.float32)
    nodes = _c(blas_nodes, np.uint32)
    inst = np.zeros((k, INSTANCE_WORDS), dtype=np.uint32)
    bounds = np.zeros((k, 9), dtype=np.float32)
    lidx = np.zeros((max(k, 1), 2), dtype=np.uint32)
    scdf = np.zeros(max(k, 1), dtype=np.float32)
    areas = np.zeros(max(k, 1), dtype=np.float32)
    total_tris = int(mi[:, 1].sum()) if k else 0
    tcdf = np.zeros(max(total_tris, 1), dtype=np.float32)
    counts = np.zeros(2, dtype=np.uint32)
    rc = lib().oracle_prepare_instances(k, _p(ow), _p(mi), _p(mat), _p(mats), mats.shape[0], _p(prims), _p(nodes),
                                        _p(inst), _p(bounds), _p(lidx), _p(scdf), _p(areas), _p(tcdf), _p(counts))
    if rc != 0:
        raise RuntimeError(f"oracle_prepare_instances failed: {rc}")
    L, CL = int(counts[0]), int(counts[1])
    tlas_nodes, inst_idx = build_tlas(bounds, tlas_bins, tlas_leaf)
    return dict(instances=inst, bounds=bounds, light_indices=lidx[:L].copy(), strength_cdf=scdf[:L].copy(),
                mesh_areas=areas[:L].copy(), tri_cdfs=tcdf[:CL].copy(), tlas_nodes=tlas_nodes,
                instance_indices=inst_idx)


def assemble(meshes, materials, instances, bins: int = 20, max_leaf: int = 8, tlas_bins: int = 2,
             tlas_leaf: int = 1) -> SceneBuffers:
    """Whole scene preparation on the CPU (the reference's prepare systems,
    src/scene/mod.rs:372-510, :561-742), mesh order = list order."""
    prims_l, tdata_l, idx_l, nodes_l, mesh_index = [], [], [], [], []
    tri_off = node_off = 0
    for m in meshes:
        prims, tdata = triangle_soup(m)
        nodes, tri_idx = build_blas(prims, bins, max_leaf)
        mesh_index.append((tri_off, prims.shape[0], tri_off, node_off))
        prims_l.append(prims); tdata_l.append(tdata); idx_l.append(tri_idx); nodes_l.append(nodes)
        tri_off += prims.shape[0]
        node_off += nodes.shape[0]
    mesh_index = np.array(mesh_index, dtype=np.uint32).reshape(-1, 4)
    primitives = np.concatenate(prims_l) if prims_l else np.zeros((0, 12), np.float32)
    tdata = np.concatenate(tdata_l) if tdata_l else np.zeros((0, 20), np.float32)
    tri_idx = np.concatenate(idx_l) if idx_l else np.zeros(0, np.uint32)
    blas = np.concatenate(nodes_l) if nodes_l else np.zeros((0, 8), np.uint32)
    mats = np.stack([m.to_words() for m in materials]) if materials else np.zeros((0, 12), np.float32)
    ow = np.stack([i.columns() for i in instances]) if instances else np.zeros((0, 16), np.float32)
    mi = mesh_index[[i.mesh for i in instances]] if instances else np.zeros((0, 4), np.uint32)
    mat_idx = np.array([i.material for i in instances], dtype=np.uint32)
    prep = prepare_instances(ow, mi, mat_idx, mats, primitives, blas, tlas_bins, tlas_leaf)
    return SceneBuffers(
        instance_count=len(instances), light_count=prep["light_indices"].shape[0],
        primitives=primitives, triangle_data=tdata, triangle_indices=tri_idx, blas_nodes=blas,
        tlas_nodes=prep["tlas_nodes"], instance_indices=prep["instance_indices"], instances=prep["instances"],
        materials=mats, light_emission_strength_cdf=prep["strength_cdf"],
        light_triangle_area_cdfs=prep["tri_cdfs"], light_mesh_areas=prep["mesh_areas"],
        light_indices=prep["light_indices"], mesh_index=mesh_index)


def assemble_desc(desc) -> SceneBuffers:
    p = desc.params
    return assemble(desc.meshes, desc.materials, desc.instances, p.get("bins", 20), p.get("max_leaf", 8))


# ----------------------------------------------------------------- render --
class _Bound:
    """Keeps the numpy arrays of a SceneBuffers alive behind a ctypes Scene."""

    def __init__(self, sb: SceneBuffers):
        self.arrs = [np.ascontiguousarray(a) if a is not None and a.size else np.zeros(16, np.uint32)
                     for a in sb.arrays()]
        self.s = Scene(sb.instance_count, sb.light_count, *[a.ctypes.data for a in self.arrs])

    def ptr(self):
        return C.byref(self.s)


def trace(sb: SceneBuffers, rays, nthreads: int = 0, **params):
    """Closest-hit query for world rays (n,6) -> dict of t, instance, triangle (BVH slot), u, v."""
    rays = _c(rays, np.float32).reshape(-1, 6)
    n = rays.shape[0]
    out = dict(t=np.zeros(n, np.float32), instance=np.zeros(n, np.uint32), triangle=np.zeros(n, np.uint32),
               u=np.zeros(n, np.float32), v=np.zeros(n, np.float32))
    b = _Bound(sb)
    st = Stats()
    p = make_params(**params)
    lib().oracle_trace(b.ptr(), _p(rays), n, C.byref(p), _p(out["t"]), _p(out["instance"]), _p(out["triangle"]),
                       _p(out["u"]), _p(out["v"]), C.byref(st), nthreads)
    out["stats"] = st.as_dict()
    return out


def render(sb: SceneBuffers, view, width: int, height: int, accumulation_count: int = 0, image=None,
           pixels=None, precision: int = 32, nthreads: int = 0, **params):
    """One path_trace dispatch (running-mean accumulation into ``image``)."""
    if image is None:
        image = np.zeros((height, width, 4), dtype=np.float32)
    assert image.dtype == np.float32 and image.flags.c_contiguous
    pix = None if pixels is None else _c(pixels, np.uint32)
    b = _Bound(sb)
    st = Stats()
    p = make_params(**params)
    ivp = _c(view.inverse_view_proj, np.float32)
    wp = _c(view.world_position, np.float32)
    lib().oracle_render(b.ptr(), _p(ivp), _p(wp), width, height, accumulation_count, C.byref(p), precision,
                        _p(pix), 0 if pix is None else pix.size, _p(image), C.byref(st), nthreads)
    return image, st.as_dict()


def gbuffer_primary(sb: SceneBuffers, view, width: int, height: int, nthreads: int = 0, **params) -> np.ndarray:
    """Primary-hit G-buffer (H, W, 16) f32: position + valid bits, normal,
    base color, emissive per texel (valid bits 0 on a miss)."""
    out = np.zeros((height, width, 16), dtype=np.float32)
    b = _Bound(sb)
    p = make_params(**params)
    ivp = _c(view.inverse_view_proj, np.float32)
    wp = _c(view.world_position, np.float32)
    lib().oracle_gbuffer_primary(b.ptr(), _p(ivp), _p(wp), width, height, C.byref(p), _p(out), nthreads)
    return out


def render_gi(sb: SceneBuffers, gbuffer, width: int, height: int, pixels=None, nthreads: int = 0, **params):
    """The realtime GI pass (src/pulse/gi.wgsl:56-135) over ``gbuffer``
    (gh, gw, 16) into a (height, width, 4) image (texels not in ``pixels`` 0)."""
    gb = _c(np.asarray(gbuffer, dtype=np.float32), np.float32)
    gh, gw = gb.shape[0], gb.shape[1]
    image = np.zeros((height, width, 4), dtype=np.float32)
    pix = None if pixels is None else _c(pixels, np.uint32)
    b = _Bound(sb)
    st = Stats()
    p = make_params(**params)
    lib().oracle_render_gi(b.ptr(), _p(gb), gw, gh, width, height, C.byref(p), _p(pix), 0 if pix is None else pix.size,
                           _p(image), C.byref(st), nthreads)
    return image, st.as_dict()


def render_mean64(sb: SceneBuffers, view, width: int, height: int, spp_total: int, pixels=None,
                  nthreads: int = 0, eval_materials=None, precision: int = 64, **params):
    """Mean radiance over sample indices 0..spp_total-1 (float64 array),
    every path in double precision with quirks off (precision 64), or in the
    float arithmetic the GPU matches bit for bit (precision 32).

    eval_materials (nee_mode 2): (material_count, 12) rows whose BSDF values
    and emissions weight the paths while the scene's materials still make
    every sampling decision (the detached-sampling estimator)."""
    pix = None if pixels is None else _c(pixels, np.uint32)
    n = width * height if pix is None else pix.size
    out = np.zeros((n, 3), dtype=np.float64)
    b = _Bound(sb)
    p = make_params(**params)
    ivp = _c(view.inverse_view_proj, np.float32)
    wp = _c(view.world_position, np.float32)
    em = None
    if eval_materials is not None:
        em = _c(eval_materials, np.float32).reshape(-1, 12)
        assert em.shape == np.asarray(sb.materials).reshape(-1, 12).shape
    lib().oracle_render_mean64(b.ptr(), _p(ivp), _p(wp), width, height, spp_total, C.byref(p), _p(pix),
                               0 if pix is None else pix.size, _p(out), nthreads, _p(em), int(precision))
    return out


def detached_fd(sb: SceneBuffers, view, width: int, height: int, n_samples: int, weights, materials_at, x0,
                eps: float = 1e-3, pixels=None, nthreads: int = 0, **params) -> np.ndarray:
    """Central differences, in every parameter of x0, of sum(weights . I)
    where I is the detached-sampling image: paths sampled with the scene's
    materials in the float arithmetic the GPU matches bit for bit (so they are
    the GPU's paths; double-precision paths would take other directions where
    rounding flips a decision), weighted by the materials materials_at(x) returns
    ((material_count, 12) rows) at x0 +/- eps in one parameter; the step is
    taken in float32 (the parameters' type), and the difference quotient
    divides by the float32 step actually taken.  weights: (H, W, 4)
    dloss/dimage (alpha ignored); only texels in pixels (all if None) are
    rendered, so weights should be zero elsewhere."""
    w = np.asarray(weights, dtype=np.float64).reshape(-1, 4)[:, :3]
    pix = np.arange(width * height, dtype=np.uint32) if pixels is None else _c(pixels, np.uint32)
    wp = w[pix]
    x0 = np.asarray(x0, dtype=np.float64)
    out = np.zeros_like(x0)
    p = dict(params, nee_mode=2)
    for k in range(x0.size):
        v = []
        for sgn in (1.0, -1.0):
            x = x0.copy()
            x[k] += sgn * eps
            img = render_mean64(sb, view, width, height, n_samples, pixels=pix, nthreads=nthreads,
                                eval_materials=materials_at(x), precision=32, **p)
            v.append(float(np.sum(wp * img)))
        step = float(np.float32(x0[k] + eps)) - float(np.float32(x0[k] - eps))
        out[k] = (v[0] - v[1]) / step
    return out


def path_log(sb: SceneBuffers, view, width: int, height: int, x: int, y: int, sample: int = 0, max_rays: int = 4096,
             **params):
    """Every ray one FP32 sample of texel (x, y) traces, in order (camera,
    bounces, shadow rays), as (rays (n, 6) origin + direction, hits dict of t,
    instance, triangle, u, v), and the sample's radiance.  For finding the
    first ray on which another tracer (pulse_trace) disagrees."""
    out = np.zeros((max_rays, 11), np.float32)
    n = np.zeros(1, np.uint32)
    rgb = np.zeros(3, np.float32)
    b = _Bound(sb)
    p = make_params(**params)
    ivp = _c(view.inverse_view_proj, np.float32)
    wp = _c(view.world_position, np.float32)
    lib().oracle_path_log(b.ptr(), _p(ivp), _p(wp), width, height, x, y, sample, C.byref(p), _p(out), max_rays,
                          _p(n), _p(rgb))
    k = min(int(n[0]), max_rays)
    rows = out[:k]
    hits = dict(t=rows[:, 6].copy(), instance=rows[:, 7].view(np.uint32).copy(),
                triangle=rows[:, 8].view(np.uint32).copy(), u=rows[:, 9].copy(), v=rows[:, 10].copy())
    return np.ascontiguousarray(rows[:, :6]), hits, rgb


def backward(sb: SceneBuffers, view, width: int, height: int, n_samples: int, dloss_dimage, nthreads: int = 0,
             **params) -> np.ndarray:
    """FP64 path-replay adjoint (nee_mode 2): (material_count, 8) gradients
    [base rgb, emissive rgb, roughness, 0] of the loss whose dloss/dimage
    (H x W x 4) is given, for the mean of n_samples samples per texel."""
    img = _c(np.asarray(dloss_dimage, dtype=np.float32).reshape(height * width * 4), np.float32)
    n_mat = int(sb.materials.shape[0])
    out = np.zeros((n_mat, 8), dtype=np.float64)
    b = _Bound(sb)
    p = make_params(**dict(params, nee_mode=2))
    ivp = _c(view.inverse_view_proj, np.float32)
    wp = _c(view.world_position, np.float32)
    rc = lib().oracle_backward(b.ptr(), _p(ivp), _p(wp), width, height, n_samples, C.byref(p), _p(img), n_mat,
                               _p(out), nthreads)
    if rc != 0:
        raise ValueError("oracle_backward: nee_mode must be 2")
    return out


def eval_g_grad(n, wo, wi, material_row) -> np.ndarray:
    """(3, 3) rows: eval_g rgb, d/dbase rgb, d/droughness rgb, in double."""
    a = [_c(np.asarray(x, dtype=np.float64), np.float64) for x in (n, wo, wi)]
    m = _c(np.asarray(material_row, dtype=np.float32), np.float32)
    out = np.zeros(9, dtype=np.float64)
    lib().oracle_eval_g_grad(_p(a[0]), _p(a[1]), _p(a[2]), _p(m), _p(out))
    return out.reshape(3, 3)


def primary_rays(view, width: int, height: int, pixels=None):
    """The primary rays of path_trace (path_tracer.wgsl:63-73) in float32 with the
    oracle's operation order, as (n, 6) origin + direction rows."""
    m = np.asarray(view.inverse_view_proj, dtype=np.float32).reshape(4, 4)  # m[c][r]
    pix = np.arange(width * height, dtype=np.uint32) if pixels is None else _c(pixels, np.uint32)
    x = (pix % width).astype(np.float32)
    y = (pix // width).astype(np.float32)
    ux = x / np.float32(width)
    uy = y / np.float32(height)
    cx = ux * np.float32(2) - np.float32(1)
    cy = -(uy * np.float32(2) - np.float32(1))
    h = [((m[0, r] * cx + m[1, r] * cy) + m[2, r] * np.float32(1)) + m[3, r] * np.float32(1) for r in range(4)]
    tgt = np.stack([h[0] / h[3], h[1] / h[3], h[2] / h[3]], 1).astype(np.float32)
    d = tgt - np.asarray(view.world_position, dtype=np.float32)
    ln = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])
    d = d / ln[:, None]
    o = np.broadcast_to(np.asarray(view.world_position, dtype=np.float32), d.shape)
    return np.ascontiguousarray(np.concatenate([o, d], 1), dtype=np.float32)
