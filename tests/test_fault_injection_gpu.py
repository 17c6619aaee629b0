"""Malformed and degenerate inputs, made on the host: the library must reject
them with a status code (or render them exactly as the oracle does) and stay
usable.  Nothing here faults the GPU: rejected buffers never reach it, and the
allocation failures are simulated by the library's own hook before any
cudaMalloc.

  * pulse_scene_set_buffers with out-of-range indices (triangle, BLAS child,
    TLAS leaf and instance index, material, light instance and CDF offset,
    instance triangle range), a mesh of 2^29 triangles (the limit of a tree)
    and with cyclic trees: PULSE_ERR_INVALID_ARG,
    the scene keeps its previous buffers;
  * meshes with NaN vertices: built and rendered exactly as the oracle does;
  * an emissive mesh whose triangles all have zero area: Heron's formula
    gives 0 for every triangle, so the area CDF is 0/0 as in the reference
    (src/scene/mod.rs:702-721); the light is never hit (a zero-area triangle
    fails the ray/triangle parallel test) and its NEE samples contribute
    nothing, so images stay finite and equal to the oracle's;
  * meshes without indices (the reference logs an error and skips them,
    src/scene/mod.rs:403-407): PULSE_ERR_INVALID_ARG, like other malformed
    index buffers;
  * allocation failures (pulse_debug_fail_allocations) in target creation,
    mesh upload, instance preparation and the first render of a larger frame:
    PULSE_ERR_OOM, and the same calls succeed afterwards.
"""
import ctypes as C
import dataclasses

import numpy as np
import pytest

import oracle
from pulse_b200 import _ffi, scenes
from pulse_b200.layout import (INST_MATERIAL_INDEX, INST_TRIANGLE_COUNT, Instance, Material, Mesh)
from pulse_b200.tracer import PulseError, Scene, Target, render_forward

pytestmark = pytest.mark.gpu

PARAMS = dict(max_depth=4, nee_mode=2, light_pick=1, quirks=0)


@pytest.fixture(scope="module")
def cornell():
    d = scenes.cornell(48, 32)
    return d, oracle.assemble(d.meshes, d.materials, d.instances, 16, 4)


def _copy(sb):
    return dataclasses.replace(sb, **{f.name: np.array(getattr(sb, f.name), copy=True)
                                      for f in dataclasses.fields(sb)
                                      if isinstance(getattr(sb, f.name), np.ndarray)})


def _interior(nodes, start=0):
    """Index of the first interior node at or after start."""
    for i in range(start, nodes.shape[0]):
        if nodes[i, 7] == 0:
            return i
    raise AssertionError("no interior node")


def _mutations(sb):
    K = sb.instance_count
    out = {}
    b = _copy(sb); b.triangle_indices[0] = 10 ** 6; out["triangle index"] = b
    b = _copy(sb); i = _interior(b.blas_nodes); b.blas_nodes[i, 3] = b.blas_nodes.shape[0]; out["BLAS child"] = b
    b = _copy(sb); i = _interior(b.blas_nodes); b.blas_nodes[i, 3] = 0; out["BLAS cycle"] = b
    b = _copy(sb); b.instance_indices[0] = K; out["TLAS instance index"] = b
    # (the root itself with a = 0 and count 0 is the empty scene's marker)
    b = _copy(sb); i = _interior(b.tlas_nodes, 1); b.tlas_nodes[i, 3] = 0; out["TLAS cycle"] = b
    b = _copy(sb)
    leaf = next(i for i in range(b.tlas_nodes.shape[0]) if b.tlas_nodes[i, 7] > 0)
    b.tlas_nodes[leaf, 3] = b.instance_indices.size
    out["TLAS leaf range"] = b
    b = _copy(sb); b.instances[0, INST_MATERIAL_INDEX] = b.materials.shape[0]; out["material index"] = b
    b = _copy(sb); b.instances[0, INST_TRIANGLE_COUNT] = b.primitives.shape[0] + 1; out["instance triangles"] = b
    # trees are limited to fewer than 2^29 elements (stack entries tag node indices)
    b = _copy(sb); b.instances[0, INST_TRIANGLE_COUNT] = 1 << 29; out["mesh of 2^29 triangles"] = b
    b = _copy(sb); b.light_indices[0, 1] = K; out["light instance"] = b
    b = _copy(sb); b.light_indices[0, 0] = b.light_triangle_area_cdfs.size; out["light CDF offset"] = b
    return out


def test_set_buffers_rejects_malformed_buffers(ctx, cornell):
    desc, sb = cornell
    W, H = desc.width, desc.height
    sc = Scene(ctx)
    sc.set_buffers(sb)
    tg = Target(ctx, W, H)
    render_forward(sc, desc.view, tg, 0, **PARAMS)
    good = tg.download()
    for name, bad in _mutations(sb).items():
        try:
            sc.set_buffers(bad)
            code = 0
        except PulseError as e:
            code = e.code
        assert code == _ffi.PULSE_ERR_INVALID_ARG, (name, code)
        # the scene keeps its buffers: the same frame renders the same bits
        render_forward(sc, desc.view, tg, 0, **PARAMS)
        assert np.array_equal(tg.download().view(np.uint32), good.view(np.uint32)), name
    ref, _ = oracle.render(sb, desc.view, W, H, 0, **PARAMS)
    assert np.array_equal(good.view(np.uint32), ref.view(np.uint32))
    tg.close()
    sc.close()


def _with_extra_mesh(desc, mesh, material):
    meshes = list(desc.meshes) + [mesh]
    materials = list(desc.materials) + [material]
    instances = list(desc.instances) + [Instance(len(meshes) - 1, len(materials) - 1)]
    return dataclasses.replace(desc, meshes=meshes, materials=materials, instances=instances)


def _device_scene(ctx, d):
    sc = Scene(ctx)
    ids = [sc.upload_mesh(m, d.params["bins"], d.params["max_leaf"]) for m in d.meshes]
    sc.set_materials(d.materials)
    sc.set_instances(d.instances, ids)
    return sc


def _same_bits_or_both_nan(a, b):
    a = np.asarray(a).reshape(-1)
    b = np.asarray(b).reshape(-1)
    if a.dtype.kind == "f":
        both_nan = np.isnan(a) & np.isnan(b)
        return a.shape == b.shape and np.array_equal(a.view(np.uint32)[~both_nan], b.view(np.uint32)[~both_nan])
    return np.array_equal(a, b)


def _render_both(ctx, sc, sb, d, params):
    W, H = d.width, d.height
    tg = Target(ctx, W, H)
    ref = np.zeros((H, W, 4), np.float32)
    for acc in range(2):
        oracle.render(sb, d.view, W, H, acc, image=ref, **params)
        render_forward(sc, d.view, tg, acc, **params)
    got = tg.download()
    tg.close()
    return got, ref


def test_nan_vertices_render_like_the_oracle(ctx, cornell):
    desc, _ = cornell
    # a quad in front of the back wall with one vertex NaN, one triangle intact
    pos = np.array([[-0.5, -0.5, -0.5], [0.5, -0.5, -0.5], [0.5, 0.5, -0.5], [np.nan, 0.5, -0.5]], np.float32)
    mesh = Mesh(pos, np.tile([0.0, 0.0, 1.0], (4, 1)), np.zeros((4, 2)), np.array([0, 1, 2, 0, 2, 3]))
    d = _with_extra_mesh(desc, mesh, Material((0.5, 0.5, 0.5, 1), (0, 0, 0, 1), 0.5, 0.5, 0.0))
    sb = oracle.assemble_desc(d)
    sc = _device_scene(ctx, d)
    got_sb = sc.download()
    for name in ("primitives", "blas_nodes", "tlas_nodes", "instance_indices", "instances"):
        assert _same_bits_or_both_nan(getattr(got_sb, name), getattr(sb, name)), name
    for mode in (0, 1, 2):
        params = dict(PARAMS, nee_mode=mode, light_pick=1 if mode == 2 else 0)
        got, ref = _render_both(ctx, sc, sb, d, params)
        assert np.isfinite(got).all()
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), mode
    sc.close()


def test_zero_area_emissive_mesh(ctx, cornell):
    desc, _ = cornell
    # two triangles of collinear vertices: Heron's formula gives exactly 0
    pos = np.array([[-0.4, 0.9, 0.0], [0.0, 0.9, 0.0], [0.4, 0.9, 0.0], [0.8, 0.9, 0.0]], np.float32)
    mesh = Mesh(pos, np.tile([0.0, -1.0, 0.0], (4, 1)), np.zeros((4, 2)), np.array([0, 1, 2, 1, 2, 3]))
    d = _with_extra_mesh(desc, mesh, Material((0.8, 0.8, 0.8, 1), (5.0, 5.0, 5.0, 1), 1.0, 0.5, 0.0))
    sb = oracle.assemble_desc(d)
    assert sb.light_count == 2
    k = int(np.nonzero(sb.light_mesh_areas == 0)[0][0])  # the zero-area light
    sc = _device_scene(ctx, d)
    got_sb = sc.download()
    assert got_sb.light_mesh_areas[k] == 0.0
    off = int(sb.light_indices[k, 0])
    assert np.isnan(got_sb.light_triangle_area_cdfs[off:off + 2]).all()  # 0/0, as the reference
    for name in ("light_emission_strength_cdf", "light_triangle_area_cdfs", "light_mesh_areas", "light_indices"):
        assert _same_bits_or_both_nan(getattr(got_sb, name), getattr(sb, name)), name
    for mode, pick in ((0, 0), (1, 0), (1, 1), (2, 0), (2, 1)):
        params = dict(PARAMS, nee_mode=mode, light_pick=pick)
        got, ref = _render_both(ctx, sc, sb, d, params)
        assert np.isfinite(got).all(), (mode, pick)
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), (mode, pick)
    sc.close()


def test_meshes_without_valid_indices_are_rejected(ctx, cornell):
    desc, sb = cornell
    sc = Scene(ctx)
    lib = ctx.lib
    m = desc.meshes[0]
    bp = _ffi.BvhParams(16, 4)
    mid = C.c_uint32(0)
    P = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    nv = m.positions.shape[0]
    cases = {
        "no index buffer": (None, 0),
        "no index buffer, count 6": (None, 6),
        "empty index buffer": (m.indices, 0),
        "count not a multiple of 3": (m.indices, 5),
        "index beyond the vertices": (np.array([0, 1, nv], np.uint32), 3),
    }
    for name, (idx, count) in cases.items():
        rc = lib.pulse_mesh_upload(sc.h, P(m.positions), P(m.normals), P(m.uvs), nv,
                                   None if idx is None else P(idx), count, C.byref(bp), C.byref(mid))
        assert rc == _ffi.PULSE_ERR_INVALID_ARG, name
    # the scene still takes meshes and renders them
    sc.close()
    sc = _device_scene(ctx, desc)
    got, ref = _render_both(ctx, sc, sb, desc, PARAMS)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    sc.close()


def _arm(ctx, n):
    ctx.lib.pulse_debug_fail_allocations(n)


def test_allocation_failures_return_oom_and_recover(ctx, cornell):
    desc, sb = cornell
    try:
        _arm(ctx, 1)
        with pytest.raises(PulseError) as e:
            Target(ctx, 64, 64)
        assert e.value.code == _ffi.PULSE_ERR_OOM
        for k in (1, 2, 3, 5):  # the k-th allocation of a mesh upload fails
            sc = Scene(ctx)
            _arm(ctx, 0)
            _arm(ctx, k)
            try:
                sc.upload_mesh(desc.meshes[5], 16, 4)
                failed = False
            except PulseError as err:
                assert err.code == _ffi.PULSE_ERR_OOM, k
                failed = True
            _arm(ctx, 0)
            assert failed or k > 3
            sc.close()
        # instance preparation: the first frame's buffers
        sc = Scene(ctx)
        ids = [sc.upload_mesh(m, 16, 4) for m in desc.meshes]
        sc.set_materials(desc.materials)
        _arm(ctx, 1)
        with pytest.raises(PulseError) as e:
            sc.set_instances(desc.instances, ids)
        assert e.value.code == _ffi.PULSE_ERR_OOM
        _arm(ctx, 0)
        sc.set_instances(desc.instances, ids)
        # the wavefront buffers of a frame larger than any before
        W, H = 3000, 2000
        tg = Target(ctx, W, H)
        _arm(ctx, 1)
        with pytest.raises(PulseError) as e:
            render_forward(sc, desc.view, tg, 0, **PARAMS)
        assert e.value.code == _ffi.PULSE_ERR_OOM
        _arm(ctx, 0)
        tg.close()
        # everything works again and renders the oracle's bits
        got, ref = _render_both(ctx, sc, sb, desc, PARAMS)
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
        sc.close()
    finally:
        _arm(ctx, 0)


def test_double_buffered_update_allocation_failure_recovers(ctx, cornell):
    """From a scene's second pulse_instances_set on, the update writes the
    other of two buffer sets; a frame with more instances grows that set.  An
    allocation failure there returns PULSE_ERR_OOM, and the next call (in
    place, on the context's stream) and the one after it (double-buffered
    again, growing the other set) prepare the larger scene exactly as the
    oracle does."""
    desc, _ = cornell
    sc = Scene(ctx)
    ids = [sc.upload_mesh(m, 16, 4) for m in desc.meshes]
    sc.set_materials(desc.materials)
    sc.set_instances(desc.instances, ids)  # in place
    sc.set_instances(desc.instances, ids)  # double-buffered: the second set
    big = dataclasses.replace(desc, instances=list(desc.instances) * 4)
    sb = oracle.assemble(big.meshes, big.materials, big.instances, 16, 4)
    try:
        _arm(ctx, 1)
        with pytest.raises(PulseError) as e:
            sc.set_instances(big.instances, ids)
        assert e.value.code == _ffi.PULSE_ERR_OOM
    finally:
        _arm(ctx, 0)
    for _ in range(2):
        sc.set_instances(big.instances, ids)
        got, ref = _render_both(ctx, sc, sb, big, PARAMS)
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    sc.close()
