"""Device BVH build and scene preparation against the CPU builders.

Bar: node arrays, tri_indices and every scene buffer bit-identical to the
restated reference (src/scene/blas.rs, src/scene/tlas.rs, src/scene/mod.rs).
"""
import numpy as np
import pytest

import oracle
from pulse_b200 import scenes
from pulse_b200.layout import triangle_soup
from pulse_b200.tracer import PulseError, Scene

pytestmark = pytest.mark.gpu


def _rand_prims(seed, n, spread=5.0, snap=False):
    rng = np.random.default_rng(seed)
    c = rng.normal(size=(n, 1, 3)) * spread
    v = (c + rng.normal(size=(n, 3, 3)) * 0.3).astype(np.float32)
    if snap:
        v[: n // 3] = np.round(v[: n // 3])
    prims = np.zeros((n, 12), np.float32)
    for k in range(3):
        prims[:, 4 * k:4 * k + 3] = v[:, k]
    return prims


def _check_blas(ctx, prims, bins, leaf):
    rn, ri = oracle.build_blas(prims, bins, leaf)
    gn, gi = ctx.build_blas(prims, bins, leaf)
    assert np.array_equal(gi, ri)
    assert gn.shape == rn.shape
    assert np.array_equal(gn, rn)


@pytest.mark.parametrize("n", [1, 2, 8, 9, 17, 100, 1023, 1024, 1025, 5000, 70000])
@pytest.mark.parametrize("bins,leaf", [(20, 8), (16, 4), (32, 4), (2, 1)])
def test_blas_random(ctx, n, bins, leaf):
    _check_blas(ctx, _rand_prims(n + bins, n, snap=(n % 2 == 0)), bins, leaf)


def test_blas_nine_triangles(ctx):
    from tests.test_oracle_kat import nine_triangles
    _check_blas(ctx, nine_triangles(), 20, 8)


@pytest.mark.parametrize("level", [3, 5, 6])
def test_blas_icosphere(ctx, level):
    prims, _ = triangle_soup(scenes.displaced_icosphere(level, 0.1, 0))
    _check_blas(ctx, prims, 20, 8)
    _check_blas(ctx, prims, 32, 4)


def test_blas_grid_terrain(ctx):
    prims, _ = triangle_soup(scenes.fbm_grid(160, 40.0, 2.0, 1))
    _check_blas(ctx, prims, 32, 4)


def test_blas_large_terrain(ctx):
    """2,093,058 triangles (the large workload's terrain at 1024^2 vertices;
    bench.py --large --large-check runs the full 4096^2 one)."""
    prims, _ = triangle_soup(scenes.fbm_grid(1024, 400.0, 12.0, 0))
    _check_blas(ctx, prims, 32, 4)


def test_blas_degenerate_reported(ctx):
    prims = np.zeros((12, 12), np.float32)
    prims[:, 4] = 1.0
    prims[:, 9] = 1.0
    with pytest.raises(PulseError) as ei:
        ctx.build_blas(prims, 20, 8)
    assert ei.value.code == -7
    prims[:, 0:11:4] -= 5.0
    _check_blas(ctx, prims, 20, 8)


def test_blas_failed_split_rotation(ctx):
    # Some nodes whose split leaves one side empty keep the reference's rotated order.
    rng = np.random.default_rng(5)
    prims = _rand_prims(7, 600)
    prims[300:] = prims[300]  # 300 identical triangles
    prims[300:, 0:11:4] += np.float32(3.0)
    _check_blas(ctx, prims, 20, 8)
    del rng


@pytest.mark.parametrize("k", [1, 2, 3, 64, 1500, 4097])
def test_tlas_random(ctx, k):
    rng = np.random.default_rng(k)
    lo = rng.uniform(-20, 20, (k, 3)).astype(np.float32)
    hi = (lo + rng.uniform(0.1, 3, (k, 3))).astype(np.float32)
    ce = (lo + np.float32(0.5) * (hi - lo)).astype(np.float32)
    b = np.concatenate([lo, hi, ce], 1)
    rn, ri = oracle.build_tlas(b, 2, 1)
    gn, gi = ctx.build_tlas(b, 2, 1)
    assert np.array_equal(gi, ri) and np.array_equal(gn, rn)


def test_tlas_empty(ctx):
    gn, gi = ctx.build_tlas(np.zeros((0, 9), np.float32))
    assert gn.shape == (1, 8) and not gn.any()


def _managed(ctx, desc):
    p = desc.params
    sc = Scene(ctx)
    ids = [sc.upload_mesh(m, p.get("bins", 20), p.get("max_leaf", 8)) for m in desc.meshes]
    sc.set_materials(desc.materials)
    sc.set_instances(desc.instances, ids)
    return sc


@pytest.mark.parametrize("name", ["cornell", "spheres"])
def test_scene_preparation_bit_exact(ctx, name):
    desc = scenes.cornell(32, 32) if name == "cornell" else scenes.spheres_1080p(level=4, n_instances=24)
    ref = oracle.assemble_desc(desc)
    sc = _managed(ctx, desc)
    got = sc.download()
    sc.close()
    for field in ("primitives", "triangle_data", "triangle_indices", "blas_nodes", "tlas_nodes", "instance_indices",
                  "instances", "materials", "light_emission_strength_cdf", "light_triangle_area_cdfs",
                  "light_mesh_areas", "light_indices"):
        a, b = getattr(got, field), getattr(ref, field)
        assert a.shape == b.shape, field
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), field
    assert got.instance_count == ref.instance_count and got.light_count == ref.light_count


def test_managed_scene_renders_like_oracle(ctx):
    from pulse_b200.tracer import Target, render_forward
    desc = scenes.cornell(48, 48)
    ref_sb = oracle.assemble_desc(desc)
    sc = _managed(ctx, desc)
    tg = Target(ctx, 48, 48)
    params = dict(max_depth=4, nee_mode=2, light_pick=1)
    render_forward(sc, desc.view, tg, 0, **params)
    got = tg.download()
    ref, _ = oracle.render(ref_sb, desc.view, 48, 48, 0, **params)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    tg.close()
    sc.close()


def test_instances_update_per_frame(ctx):
    """prepare_mesh_instances runs every frame: moving an instance rebuilds the TLAS."""
    desc = scenes.spheres_1080p(level=3, n_instances=10)
    sc = _managed(ctx, desc)
    rng = np.random.default_rng(9)
    for _ in range(3):
        for inst in desc.instances[:10]:
            inst.object_world = scenes.trs(rng.uniform(-10, 10, 3), scenes.random_rotation(rng))
        sc.set_instances(desc.instances, list(range(len(desc.meshes))))
        ref = oracle.assemble_desc(desc)
        got = sc.download()
        assert np.array_equal(got.tlas_nodes, ref.tlas_nodes)
        assert np.array_equal(got.instances, ref.instances)
    sc.close()


def test_instances_set_overlaps_the_previous_frame(ctx):
    """pulse_instances_set prepares the next frame's instances and TLAS in the
    other of two buffer sets while the previous frame still traces.  Frames
    issued back to back (full updates, an incremental update and a material
    change among them, no host wait between the calls) equal the same frames
    rendered one at a time, and the last frame equals the oracle's render of
    the oracle's assembly."""
    from pulse_b200.tracer import Target, render_forward
    desc = scenes.spheres_1080p(level=3, n_instances=24)
    sc = _managed(ctx, desc)
    ids = list(range(len(desc.meshes)))
    rng = np.random.default_rng(33)
    W, H, frames = 64, 48, 7
    params = dict(max_depth=8, nee_mode=2, light_pick=1)
    poses = [[scenes.trs(rng.uniform(-10, 10, 3), scenes.random_rotation(rng)) for _ in desc.instances]
             for _ in range(frames)]
    moved = rng.choice(len(desc.instances), size=5, replace=False).astype(np.uint32)
    emissive = [i for i, m in enumerate(desc.materials) if max(m.emissive[:3]) > 0][0]

    def step(f):
        for inst, pose in zip(desc.instances, poses[f]):
            inst.object_world = pose
        if f == 3:  # an incremental update between two full ones
            sc.update_instances(moved, np.stack([desc.instances[i].columns() for i in moved]))
            for i in set(range(len(desc.instances))) - set(moved.tolist()):
                desc.instances[i].object_world = poses[f - 1][i]
        else:
            if f == 5:  # a material change: the next update must read the new emission
                em = desc.materials[emissive].emissive
                desc.materials[emissive].emissive = tuple(e * 2.0 for e in em[:3]) + tuple(em[3:])
                sc.set_materials(desc.materials)
            sc.set_instances(desc.instances, ids)

    tgs = [Target(ctx, W, H) for _ in range(frames)]
    saved = [inst.object_world for inst in desc.instances]  # replaced, never changed in place
    mats0 = [m.emissive for m in desc.materials]
    for f in range(frames):
        step(f)
        render_forward(sc, desc.view, tgs[f], 0, **params)
    back_to_back = [t.download() for t in tgs]
    for t in tgs:
        t.close()
    sc.close()

    for inst, w in zip(desc.instances, saved):
        inst.object_world = w
    for m, e in zip(desc.materials, mats0):
        m.emissive = e
    sc = _managed(ctx, desc)
    tg = Target(ctx, W, H)
    for f in range(frames):
        step(f)
        render_forward(sc, desc.view, tg, 0, **params)
        img = tg.download()  # the host waits for this frame before the next update
        assert np.array_equal(img.view(np.uint32), back_to_back[f].view(np.uint32)), f
    ref, _ = oracle.render(oracle.assemble_desc(desc), desc.view, W, H, 0, **params)
    assert np.array_equal(back_to_back[-1].view(np.uint32), ref.view(np.uint32))
    tg.close()
    sc.close()


_SCENE_FIELDS = ("primitives", "triangle_data", "triangle_indices", "blas_nodes", "tlas_nodes", "instance_indices",
                 "instances", "materials", "light_emission_strength_cdf", "light_triangle_area_cdfs",
                 "light_mesh_areas", "light_indices")


def test_instances_incremental_update(ctx):
    """Moving a few instances through pulse_instances_update gives the scene
    the full per-frame rebuild (src/scene/mod.rs:561-697) makes, bit for bit,
    and the same image."""
    from pulse_b200.tracer import Target, render_forward
    desc = scenes.spheres_1080p(level=3, n_instances=24)
    sc = _managed(ctx, desc)
    rng = np.random.default_rng(21)
    tg = Target(ctx, 64, 48)
    params = dict(max_depth=4, nee_mode=2, light_pick=1)
    for frame in range(4):
        k = int(rng.integers(1, 9))
        idx = rng.choice(len(desc.instances), size=k, replace=False).astype(np.uint32)
        for i in idx:
            desc.instances[i].object_world = scenes.trs(rng.uniform(-10, 10, 3), scenes.random_rotation(rng))
        bins = 8 if frame >= 2 else 2  # frame 2 switches the TLAS parameters, frame 3 keeps them
        sc.update_instances(idx, np.stack([desc.instances[i].columns() for i in idx]),
                            tlas_bins=8 if frame == 2 else None)
        got = sc.download()
        p = desc.params
        ref = oracle.assemble(desc.meshes, desc.materials, desc.instances, p.get("bins", 20), p.get("max_leaf", 8),
                              tlas_bins=bins)
        for field in _SCENE_FIELDS:
            a, b = getattr(got, field), getattr(ref, field)
            assert a.shape == b.shape, (frame, field)
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (frame, field)
        full = Scene(ctx)
        ids = [full.upload_mesh(m, p.get("bins", 20), p.get("max_leaf", 8)) for m in desc.meshes]
        full.set_materials(desc.materials)
        full.set_instances(desc.instances, ids, tlas_bins=bins)
        render_forward(sc, desc.view, tg, 0, **params)
        img = tg.download()
        render_forward(full, desc.view, tg, 0, **params)
        assert np.array_equal(img.view(np.uint32), tg.download().view(np.uint32)), frame
        full.close()
    tg.close()
    sc.close()


def test_instances_update_rejects(ctx):
    from pulse_b200 import _ffi
    desc = scenes.spheres_1080p(level=2, n_instances=6)
    sc = _managed(ctx, desc)
    eye = np.eye(4, dtype=np.float32).reshape(1, 16)
    with pytest.raises(PulseError) as e:
        sc.update_instances([len(desc.instances)], eye)
    assert e.value.code == _ffi.PULSE_ERR_INVALID_ARG
    with pytest.raises(PulseError) as e:
        sc.update_instances([2, 2], np.repeat(eye, 2, 0))
    assert e.value.code == _ffi.PULSE_ERR_INVALID_ARG
    sc.update_instances([], np.zeros((0, 16), np.float32))  # no-op: the TLAS is rebuilt unchanged
    before = sc.download()
    assert np.array_equal(before.tlas_nodes, oracle.assemble_desc(desc).tlas_nodes)
    sc.upload_mesh(desc.meshes[0], 20, 8)  # a mesh change needs the full pulse_instances_set
    with pytest.raises(PulseError) as e:
        sc.update_instances([0], eye)
    assert e.value.code == _ffi.PULSE_ERR_NOT_READY
    sc.close()
