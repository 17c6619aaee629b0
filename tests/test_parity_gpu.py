"""GPU parity: the CUDA path against the CPU oracle on the same seeded inputs.

Bit-exact is the bar for closest-hit IDs, t, u, v and for per-pixel radiance:
both sides evaluate the same IEEE binary32 operations in the same order
(no fused multiply-add except where written explicitly on both sides).
"""
import numpy as np
import pytest

import oracle
from pulse_b200 import scenes
from pulse_b200.tracer import Scene, Target, render_forward

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cornell_sb():
    d = scenes.cornell(64, 64)
    return d, oracle.assemble(d.meshes, d.materials, d.instances, 16, 4)


@pytest.fixture(scope="module")
def spheres_sb():
    d = scenes.spheres_1080p(level=4, n_instances=16, width=96, height=54)
    return d, oracle.assemble(d.meshes, d.materials, d.instances, 20, 8)


@pytest.fixture(scope="module")
def dense_sb():
    """Heavily overlapping instances (24 spheres of radius 1 in a 6^3 box): many
    BLAS entries per ray, the case the cross-BLAS culling acts on."""
    d = scenes.spheres_1080p(level=4, n_instances=24, width=80, height=45, box=3.0)
    return d, oracle.assemble(d.meshes, d.materials, d.instances, 20, 8)


def _random_rays(view, n, rng):
    o = np.asarray(view.world_position, dtype=np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([np.broadcast_to(o, (n, 3)), d], 1).astype(np.float32)


@pytest.mark.parametrize("which", ["cornell_sb", "spheres_sb", "dense_sb"])
@pytest.mark.parametrize("quirks", [1, 0])
def test_trace_bit_exact(ctx, request, which, quirks):
    desc, sb = request.getfixturevalue(which)
    rng = np.random.default_rng(1)
    rays = np.concatenate([oracle.primary_rays(desc.view, desc.width, desc.height),
                           _random_rays(desc.view, 4096, rng)])
    ref = oracle.trace(sb, rays, quirks=quirks)
    sc = Scene(ctx)
    sc.set_buffers(sb)
    got = sc.trace(rays, quirks=quirks)
    sc.close()
    assert np.array_equal(got["t"].view(np.uint32), ref["t"].view(np.uint32))
    assert np.array_equal(got["instance_index"], ref["instance"])
    assert np.array_equal(got["triangle_index"], ref["triangle"])
    assert np.array_equal(got["u"].view(np.uint32), ref["u"].view(np.uint32))
    assert np.array_equal(got["v"].view(np.uint32), ref["v"].view(np.uint32))


@pytest.mark.parametrize("which", ["cornell_sb", "spheres_sb", "dense_sb"])
@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("kernel,min_blocks,wf_segments", [(1, 4, 0), (1, 6, 0), (1, 8, 0), (2, 0, 0), (2, 0, 1),
                                                        (2, 0, 9)])
def test_render_bit_exact(ctx, request, which, mode, kernel, min_blocks, wf_segments):
    desc, sb = request.getfixturevalue(which)
    params = dict(max_depth=5, nee_mode=mode, light_pick=1 if mode == 2 else 0, quirks=1, min_blocks=min_blocks,
                  kernel=kernel, wf_segments=wf_segments)
    W, H = desc.width, desc.height
    ref = np.zeros((H, W, 4), np.float32)
    sc = Scene(ctx)
    sc.set_buffers(sb)
    tg = Target(ctx, W, H)
    for acc in range(3):
        oracle.render(sb, desc.view, W, H, acc, image=ref, **params)
        render_forward(sc, desc.view, tg, acc, **params)
    if kernel == 2:  # spp > 1 in one call: sample index acc*spp + s
        oracle.render(sb, desc.view, W, H, 1, image=ref, **dict(params, spp=3))
        render_forward(sc, desc.view, tg, 1, **dict(params, spp=3))
    got = tg.download()
    tg.close()
    sc.close()
    assert np.isfinite(ref).any()
    diff = got.view(np.uint32) != ref.view(np.uint32)
    assert not diff.any(), f"{diff.any(axis=2).sum()} of {W*H} texels differ"


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("kernel", [1, 2])
def test_work_counters_match_oracle(ctx, spheres_sb, mode, kernel):
    """The device's tallies of the reference algorithm's work (the roofline's
    algorithmic bytes) equal the oracle's on the same frame."""
    from pulse_b200.tracer import render_count
    desc, sb = spheres_sb
    params = dict(max_depth=8, nee_mode=mode, light_pick=1 if mode == 2 else 0)
    W, H = desc.width, desc.height
    _, ref = oracle.render(sb, desc.view, W, H, 0, **params)
    params["kernel"] = kernel
    sc = Scene(ctx)
    sc.set_buffers(sb)
    tg = Target(ctx, W, H)
    got = render_count(sc, desc.view, tg, 0, **params)
    tg.close()
    sc.close()
    for k in ("rays", "tlas_interior", "blas_entries", "blas_interior", "tri_tests", "hits", "nee"):
        assert got[k] == ref[k], (k, got[k], ref[k])
    assert got["paths"] == W * H


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("kernel", [1, 2])
def test_render_no_roulette_bit_exact(ctx, cornell_sb, mode, kernel):
    """Russian roulette off: paths run to max_depth (or a miss), same draws."""
    desc, sb = cornell_sb
    params = dict(max_depth=6, nee_mode=mode, light_pick=1 if mode == 2 else 0, quirks=0, no_roulette=1,
                  kernel=kernel)
    W, H = desc.width, desc.height
    ref = np.zeros((H, W, 4), np.float32)
    sc = Scene(ctx)
    sc.set_buffers(sb)
    tg = Target(ctx, W, H)
    for acc in range(2):
        oracle.render(sb, desc.view, W, H, acc, image=ref, **params)
        render_forward(sc, desc.view, tg, acc, **params)
    got = tg.download()
    tg.close()
    sc.close()
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
