"""The CPU oracle against the committed golden fixtures (tests/golden): any
change of the oracle's arithmetic shows up here bit for bit."""
import numpy as np
import pytest

import oracle
from golden_util import H, RENDER_CASES, SCENE_FIELDS, W, load, same_bits, scene_buffers
from pulse_b200 import scenes
from pulse_b200.layout import triangle_soup


@pytest.fixture(scope="module")
def cornell():
    d = scenes.cornell(W, H)
    return d, oracle.assemble(d.meshes, d.materials, d.instances, 16, 4)


def test_scene_buffers(cornell):
    _, sb = cornell
    g = load("cornell_scene.npz")
    for f in SCENE_FIELDS:
        assert same_bits(np.asarray(getattr(sb, f)), g[f]), f
    assert (sb.instance_count, sb.light_count) == tuple(int(x) for x in g["counts"])


@pytest.mark.parametrize("quirks", [1, 0])
def test_hits(quirks):
    g = load("cornell_hits.npz")
    h = oracle.trace(scene_buffers(), g["rays"], quirks=quirks)
    for k in ("t", "instance", "triangle", "u", "v"):
        assert same_bits(h[k], g[f"q{quirks}_{k}"]), k


@pytest.mark.parametrize("case", sorted(RENDER_CASES))
def test_render(cornell, case):
    desc, _ = cornell
    img = np.zeros((H, W, 4), np.float32)
    sb = scene_buffers()
    for acc in range(2):
        oracle.render(sb, desc.view, W, H, acc, image=img, **RENDER_CASES[case])
    assert same_bits(img, load("cornell_render.npz")[case])


def test_icosphere_bvh():
    g = load("icosphere_bvh.npz")
    prims, _ = triangle_soup(scenes.displaced_icosphere(3, 0.1, 3))
    assert same_bits(prims, g["prims"])
    nodes, idx = oracle.build_blas(prims, 20, 8)
    assert same_bits(nodes, g["blas_nodes"]) and same_bits(idx, g["blas_indices"])
    tn, ti = oracle.build_tlas(g["tlas_bounds"], 2, 1)
    assert same_bits(tn, g["tlas_nodes"]) and same_bits(ti, g["tlas_indices"])
