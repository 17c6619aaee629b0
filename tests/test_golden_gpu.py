"""The CUDA library against the committed golden fixtures (tests/golden),
with no oracle at run time: BVH builds, the preparation path's scene buffers,
closest hits and accumulated images, bit for bit."""
import numpy as np
import pytest

from golden_util import H, RENDER_CASES, SCENE_FIELDS, W, load, same_bits, scene_buffers
from pulse_b200 import scenes
from pulse_b200.tracer import Scene, Target, render_forward

pytestmark = pytest.mark.gpu


def test_builds(ctx):
    g = load("icosphere_bvh.npz")
    nodes, idx = ctx.build_blas(g["prims"], 20, 8)
    assert same_bits(nodes, g["blas_nodes"]) and same_bits(idx, g["blas_indices"])
    tn, ti = ctx.build_tlas(g["tlas_bounds"], 2, 1)
    assert same_bits(tn, g["tlas_nodes"]) and same_bits(ti, g["tlas_indices"])


def test_prepared_scene(ctx):
    desc = scenes.cornell(W, H)
    sc = Scene(ctx)
    ids = [sc.upload_mesh(m, 16, 4) for m in desc.meshes]
    sc.set_materials(desc.materials)
    sc.set_instances(desc.instances, ids)
    got = sc.download()
    sc.close()
    g = load("cornell_scene.npz")
    for f in SCENE_FIELDS:
        assert same_bits(np.asarray(getattr(got, f)), g[f]), f


@pytest.mark.parametrize("quirks", [1, 0])
def test_hits(ctx, quirks):
    g = load("cornell_hits.npz")
    sc = Scene(ctx)
    sc.set_buffers(scene_buffers())
    h = sc.trace(g["rays"], quirks=quirks)
    sc.close()
    for k, gk in (("t", "t"), ("instance_index", "instance"), ("triangle_index", "triangle"), ("u", "u"), ("v", "v")):
        assert same_bits(h[k], g[f"q{quirks}_{gk}"]), k


@pytest.mark.parametrize("kernel", [1, 2])
@pytest.mark.parametrize("case", sorted(RENDER_CASES))
def test_render(ctx, case, kernel):
    desc = scenes.cornell(W, H)
    sc = Scene(ctx)
    sc.set_buffers(scene_buffers())
    tg = Target(ctx, W, H)
    for acc in range(2):
        render_forward(sc, desc.view, tg, acc, kernel=kernel, **RENDER_CASES[case])
    img = tg.download()
    tg.close()
    sc.close()
    assert same_bits(img, load("cornell_render.npz")[case])
