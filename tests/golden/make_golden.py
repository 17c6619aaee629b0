"""Writes the golden fixtures of this directory from the CPU oracle.

    python tests/golden/make_golden.py

Every fixture is a seeded, small workload with the oracle's output:
  cornell_scene.npz   the 13 scene buffers of the Cornell box (36 triangles,
                      BLAS bins 16 / leaf 4, TLAS 2 / 1) as the preparation
                      path builds them (BVHs, instance records, light CDFs);
  cornell_hits.npz    closest hits (t, instance, BVH slot, u, v) of the 32x24
                      primary rays plus 1024 seeded random rays, quirks on and off;
  cornell_render.npz  32x24 images after 2 accumulated frames of 1 sample:
                      estimator modes 0 and 1 with the reference's quirks,
                      mode 2 without, Russian roulette on and off;
  icosphere_bvh.npz   BLAS of a displaced icosphere (subdivision 3, 1280
                      triangles, bins 20 / leaf 8) and the TLAS over 64 seeded
                      instance boxes (bins 2 / leaf 1).
The tests compare the oracle (CPU) and the CUDA library (GPU) with these bit
for bit, so a change of either side's arithmetic shows up against a fixed file.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from pulse_b200 import scenes  # noqa: E402
from pulse_b200.layout import triangle_soup  # noqa: E402

W, H = 32, 24
SCENE_FIELDS = ("primitives", "triangle_data", "triangle_indices", "blas_nodes", "tlas_nodes", "instance_indices",
                "instances", "materials", "light_emission_strength_cdf", "light_triangle_area_cdfs",
                "light_mesh_areas", "light_indices")
RENDER_CASES = {  # name: params
    "m0_q1": dict(max_depth=5, nee_mode=0, light_pick=0, quirks=1),
    "m1_q1": dict(max_depth=5, nee_mode=1, light_pick=0, quirks=1),
    "m2_q0": dict(max_depth=6, nee_mode=2, light_pick=1, quirks=0),
    "m2_q0_norr": dict(max_depth=6, nee_mode=2, light_pick=1, quirks=0, no_roulette=1),
}


def cornell():
    d = scenes.cornell(W, H)
    return d, oracle.assemble(d.meshes, d.materials, d.instances, 16, 4)


def random_rays(view, n, seed=1):
    rng = np.random.default_rng(seed)
    o = np.asarray(view.world_position, dtype=np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([np.broadcast_to(o, (n, 3)), d], 1).astype(np.float32)


def hit_rays(desc):
    return np.concatenate([oracle.primary_rays(desc.view, W, H), random_rays(desc.view, 1024)]).astype(np.float32)


def render_case(sb, desc, params):
    img = np.zeros((H, W, 4), np.float32)
    for acc in range(2):
        oracle.render(sb, desc.view, W, H, acc, image=img, **params)
    return img


def icosphere_case():
    mesh = scenes.displaced_icosphere(3, 0.1, 3)
    prims, _ = triangle_soup(mesh)
    nodes, idx = oracle.build_blas(prims, 20, 8)
    rng = np.random.default_rng(4)
    lo = rng.uniform(-10, 10, (64, 3)).astype(np.float32)
    hi = (lo + rng.uniform(0.1, 3.0, (64, 3))).astype(np.float32)
    bounds = np.concatenate([lo, hi, lo + np.float32(0.5) * (hi - lo)], 1).astype(np.float32)
    tnodes, tidx = oracle.build_tlas(bounds, 2, 1)
    return dict(prims=prims, blas_nodes=nodes, blas_indices=idx, tlas_bounds=bounds, tlas_nodes=tnodes,
                tlas_indices=tidx)


def main():
    oracle.build()
    desc, sb = cornell()
    np.savez_compressed(os.path.join(HERE, "cornell_scene.npz"),
                        **{f: np.asarray(getattr(sb, f)) for f in SCENE_FIELDS},
                        counts=np.array([sb.instance_count, sb.light_count], np.uint32))
    rays = hit_rays(desc)
    out = dict(rays=rays)
    for q in (1, 0):
        h = oracle.trace(sb, rays, quirks=q)
        for k in ("t", "instance", "triangle", "u", "v"):
            out[f"q{q}_{k}"] = h[k]
    np.savez_compressed(os.path.join(HERE, "cornell_hits.npz"), **out)
    np.savez_compressed(os.path.join(HERE, "cornell_render.npz"),
                        **{name: render_case(sb, desc, p) for name, p in RENDER_CASES.items()})
    np.savez_compressed(os.path.join(HERE, "icosphere_bvh.npz"), **icosphere_case())
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")


if __name__ == "__main__":
    main()
