"""Edge cases of the render against the oracle, bit for bit, with both
kernels and every estimator: stacks smaller than the trees (pushes dropped as
in the reference, counted), a binding iteration cap, a scene without emissive
material (NEE with no light), a scene without instances, tiny and odd image
sizes with several samples per texel, and zero or one bounce."""
import dataclasses

import numpy as np
import pytest

import oracle
from pulse_b200 import scenes
from pulse_b200.layout import Material
from pulse_b200.tracer import Scene, Target, render_forward

pytestmark = pytest.mark.gpu

MODES = [(0, 1), (0, 2), (1, 1), (1, 2), (2, 1), (2, 2)]  # (nee_mode, kernel)


def _check(ctx, sb, view, W, H, frames=2, counters=False, **params):
    ref = np.zeros((H, W, 4), np.float32)
    sc = Scene(ctx)
    sc.set_buffers(sb)
    tg = Target(ctx, W, H)
    s0 = ctx.stats()
    ost = {"stack_overflows": 0, "iter_cap_hits": 0}
    for acc in range(frames):
        _, st = oracle.render(sb, view, W, H, acc, image=ref, **params)
        for k in ost:
            ost[k] += st[k]
        render_forward(sc, view, tg, acc, **params)
    got = tg.download()
    s1 = ctx.stats()
    tg.close()
    sc.close()
    diff = got.view(np.uint32) != ref.view(np.uint32)
    assert not diff.any(), f"{diff.any(axis=2).sum()} of {W * H} texels differ"
    if counters:
        for k, v in ost.items():
            assert s1[k] - s0[k] == v, (k, s1[k] - s0[k], v)
    return ost


@pytest.fixture(scope="module")
def dense():
    d = scenes.spheres_1080p(level=4, n_instances=24, width=64, height=36, box=3.0)
    return d, oracle.assemble(d.meshes, d.materials, d.instances, 20, 8)


@pytest.fixture(scope="module")
def cornell():
    d = scenes.cornell(40, 30)
    return d, oracle.assemble(d.meshes, d.materials, d.instances, 16, 4)


@pytest.mark.parametrize("mode,kernel", MODES)
@pytest.mark.parametrize("quirks", [1, 0])
def test_stack_overflow_dropped_like_reference(ctx, dense, mode, kernel, quirks):
    d, sb = dense
    ost = _check(ctx, sb, d.view, d.width, d.height, counters=True, max_depth=4, nee_mode=mode, kernel=kernel,
                 light_pick=1 if mode == 2 else 0, quirks=quirks, stack_depth=3)
    assert ost["stack_overflows"] > 0


@pytest.mark.parametrize("mode,kernel", MODES)
def test_iteration_cap_binds_like_reference(ctx, dense, mode, kernel):
    d, sb = dense
    ost = _check(ctx, sb, d.view, d.width, d.height, counters=True, max_depth=3, nee_mode=mode, kernel=kernel,
                 light_pick=1 if mode == 2 else 0, quirks=0, iter_cap=12)
    assert ost["iter_cap_hits"] > 0


@pytest.mark.parametrize("mode,kernel", MODES)
def test_no_emissive_material(ctx, cornell, mode, kernel):
    d, _ = cornell
    mats = [dataclasses.replace(m, emissive=(0.0, 0.0, 0.0, 1.0)) for m in d.materials]
    sb = oracle.assemble(d.meshes, mats, d.instances, 16, 4)
    assert sb.light_count == 0
    _check(ctx, sb, d.view, d.width, d.height, max_depth=4, nee_mode=mode, kernel=kernel,
           light_pick=1 if mode == 2 else 0)


@pytest.mark.parametrize("mode,kernel", MODES)
def test_scene_without_instances(ctx, cornell, mode, kernel):
    d, _ = cornell
    sb = oracle.assemble(d.meshes, d.materials, [], 16, 4)
    assert sb.instance_count == 0
    _check(ctx, sb, d.view, d.width, d.height, max_depth=4, nee_mode=mode, kernel=kernel)


@pytest.mark.parametrize("size", [(1, 1), (7, 3), (17, 9), (33, 1)])
@pytest.mark.parametrize("mode,kernel", MODES)
def test_tiny_and_odd_images(ctx, cornell, size, mode, kernel):
    d, sb = cornell
    W, H = size
    _check(ctx, sb, d.view, W, H, frames=3, max_depth=4, nee_mode=mode, kernel=kernel, spp=3,
           light_pick=1 if mode == 2 else 0)


@pytest.mark.parametrize("depth", [0, 1])
@pytest.mark.parametrize("mode,kernel", MODES)
def test_zero_and_one_bounce(ctx, cornell, depth, mode, kernel):
    d, sb = cornell
    _check(ctx, sb, d.view, d.width, d.height, max_depth=depth, nee_mode=mode, kernel=kernel,
           light_pick=1 if mode == 2 else 0)
