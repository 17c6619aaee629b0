"""Bit-exact parity on the benchmark's own scene and settings.

The 1080p benchmark traces 64 instances of the subdivision-7 displaced
icosphere (327,680 triangles, a 20-level BLAS) with the corrected estimator
(nee_mode 2), the power light CDF, quirks off, 8 bounces and the reference's
stack of 32 entries.  Its trees fit the stack (19 pushes deep at most), so the
exact box-skipping shortcuts of the traversal are on, as in the benchmark;
the small-scene parity tests run level-4 spheres.  Here the same scene at
192 x 108 texels, prepared on the device exactly as the benchmark prepares it
(mesh upload with the device BVH build, instances with the device TLAS), is
rendered for three accumulated frames and compared bit for bit with the CPU
oracle, which builds its own trees.
"""
import numpy as np
import pytest

import oracle
from pulse_b200 import scenes
from pulse_b200.tracer import Scene, Target, render_forward

pytestmark = pytest.mark.gpu

PARAMS = dict(max_depth=8, nee_mode=2, light_pick=1, quirks=0, spp=1, stack_depth=32)


@pytest.fixture(scope="module")
def headline():
    d = scenes.spheres_1080p(level=7, width=192, height=108)
    return d, oracle.assemble_desc(d)


@pytest.fixture(scope="module")
def device_scene(ctx, headline):
    d, _ = headline
    sc = Scene(ctx)
    ids = [sc.upload_mesh(m, d.params["bins"], d.params["max_leaf"]) for m in d.meshes]
    sc.set_materials(d.materials)
    sc.set_instances(d.instances, ids)
    yield sc
    sc.close()


def test_device_scene_equals_oracle_scene(headline, device_scene):
    _, sb = headline
    got = device_scene.download()
    for name in ("primitives", "triangle_data", "triangle_indices", "blas_nodes", "tlas_nodes", "instance_indices",
                 "instances", "materials", "light_emission_strength_cdf", "light_triangle_area_cdfs",
                 "light_mesh_areas", "light_indices"):
        a, b = np.asarray(getattr(got, name)), np.asarray(getattr(sb, name))
        assert a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32)), name


@pytest.mark.parametrize("seed,wf_segments,knobs", [(0, 0, {}), (1, 0, {}), (0, 1, {}), (0, 0xffffffff, {}),
                                                     (0, 0, dict(ray_sort=1)), (0, 0, dict(block_size=64)),
                                                     (0, 4, dict(ray_sort=1, block_size=64, trace_blocks=6))])
def test_headline_frames_bit_exact(ctx, headline, device_scene, seed, wf_segments, knobs):
    """Every launch-shape knob of the autotuner renders the same bits."""
    d, sb = headline
    W, H = d.width, d.height
    params = dict(PARAMS, seed=seed)
    g0 = ctx.stats()
    ref = np.zeros((H, W, 4), np.float32)
    tg = Target(ctx, W, H)
    for acc in range(3):
        oracle.render(sb, d.view, W, H, acc, image=ref, **params)
        render_forward(device_scene, d.view, tg, acc, kernel=2, wf_segments=wf_segments, **params, **knobs)
    got = tg.download()
    tg.close()
    g1 = ctx.stats()
    assert g1["stack_overflows"] == g0["stack_overflows"] and g1["iter_cap_hits"] == g0["iter_cap_hits"]
    assert np.isfinite(ref).all() and ref[..., :3].max() > 0
    diff = np.any(got.view(np.uint32) != ref.view(np.uint32), axis=2)
    assert not diff.any(), f"{int(diff.sum())} of {W * H} texels differ"
