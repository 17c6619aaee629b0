"""Loading of the golden fixtures (tests/golden, written by make_golden.py)."""
import os

import numpy as np

from pulse_b200.layout import SceneBuffers

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
W, H = 32, 24
SCENE_FIELDS = ("primitives", "triangle_data", "triangle_indices", "blas_nodes", "tlas_nodes", "instance_indices",
                "instances", "materials", "light_emission_strength_cdf", "light_triangle_area_cdfs",
                "light_mesh_areas", "light_indices")
RENDER_CASES = {
    "m0_q1": dict(max_depth=5, nee_mode=0, light_pick=0, quirks=1),
    "m1_q1": dict(max_depth=5, nee_mode=1, light_pick=0, quirks=1),
    "m2_q0": dict(max_depth=6, nee_mode=2, light_pick=1, quirks=0),
    "m2_q0_norr": dict(max_depth=6, nee_mode=2, light_pick=1, quirks=0, no_roulette=1),
}


def load(name):
    with np.load(os.path.join(GOLDEN, name)) as z:
        return {k: z[k] for k in z.files}


def scene_buffers() -> SceneBuffers:
    g = load("cornell_scene.npz")
    return SceneBuffers(int(g["counts"][0]), int(g["counts"][1]), *[np.ascontiguousarray(g[f]) for f in SCENE_FIELDS])


def same_bits(a, b) -> bool:
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.shape == b.shape and a.tobytes() == b.tobytes()
