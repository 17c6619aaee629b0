"""The realtime GI restatement (oracle.render_gi, src/pulse/gi.wgsl:56-135) on
the CPU, pinned to the path tracer's diffuse estimator (nee_mode 1,
src/path_tracer/path_tracer.wgsl:127-192), which the golden fixtures pin.

The GI pass at texel P seeds P * 5817321 (+ seed * 0x9E3779B9); the path
tracer seeds P * 1235243 + acc * 5817321 + seed * 0x9E3779B9.  With the path
tracer's seed chosen so both states agree at P, one GI sample from the
primary-hit G-buffer is the path tracer's mode-1 sample at P, bit for bit.
"""
import numpy as np
import pytest

import oracle
from pulse_b200 import scenes

K = 0x9E3779B9
K_INV = pow(K, -1, 1 << 32)


def _matching_seed(pixel: int, gi_seed: int = 0) -> int:
    want = (pixel * 5817321 + gi_seed * K) & 0xFFFFFFFF
    return ((want - pixel * 1235243) * K_INV) & 0xFFFFFFFF


@pytest.fixture(scope="module")
def cornell():
    d = scenes.cornell(32, 24)
    return d, oracle.assemble(d.meshes, d.materials, d.instances, 16, 4)


@pytest.mark.parametrize("light_pick,no_roulette", [(0, 0), (1, 0), (0, 1)])
def test_gi_sample_is_the_diffuse_estimator(cornell, light_pick, no_roulette):
    d, sb = cornell
    W, H = 32, 24
    gb = oracle.gbuffer_primary(sb, d.view, W, H)
    assert (gb[..., 3].view(np.uint32) == 1).sum() > W * H // 2
    rng = np.random.default_rng(3)
    pixels = rng.choice(W * H, size=24, replace=False)
    gi, _ = oracle.render_gi(sb, gb, W, H, spp=1, max_depth=5, light_pick=light_pick, no_roulette=no_roulette)
    for p in pixels:
        ref, _ = oracle.render(sb, d.view, W, H, 0, pixels=[p], spp=1, max_depth=5, nee_mode=1,
                               light_pick=light_pick, no_roulette=no_roulette, seed=_matching_seed(int(p)))
        y, x = divmod(int(p), W)
        assert np.array_equal(gi[y, x].view(np.uint32), ref[y, x].view(np.uint32)), p


def test_gi_samples_share_one_random_state(cornell):
    """The first of two samples is the one-sample pass's sample: mean =
    c0 * 0.5 + c1 * 0.5 with c0 from the one-sample image."""
    d, sb = cornell
    W, H = 32, 24
    gb = oracle.gbuffer_primary(sb, d.view, W, H)
    one, _ = oracle.render_gi(sb, gb, W, H, spp=1)
    two, st = oracle.render_gi(sb, gb, W, H, spp=2)
    assert st["paths"] == 2 * W * H
    c1 = (two[..., :3] - one[..., :3] * np.float32(0.5)) * 2
    assert np.all(np.isfinite(c1)) and np.all(c1 >= -1e-4)
    assert not np.array_equal(c1, one[..., :3])  # the second sample continues the state
    assert np.all(two[..., 3] == 1.0)


def test_gi_invalid_texels_and_texel_mapping(cornell):
    d, sb = cornell
    gw, gh = 8, 6
    gb = np.zeros((gh, gw, 16), np.float32)
    gb[2, 3, 0:3] = [0.0, 1.0, 0.0]
    gb[2, 3, 3] = np.uint32(1).view(np.float32)
    gb[2, 3, 4:7] = [0.0, -1.0, 0.0]
    gb[2, 3, 8:11] = [0.5, 0.5, 0.5]
    gb[2, 3, 12:15] = [0.25, 0.5, 1.0]
    W, H = 40, 30  # texel (x, y) reads (u32(x / 40 * 8), u32(y / 30 * 6))
    img, st = oracle.render_gi(sb, gb, W, H, spp=2)
    xs = [x for x in range(W) if int(np.float32(x) / np.float32(W) * np.float32(gw)) == 3]
    ys = [y for y in range(H) if int(np.float32(y) / np.float32(H) * np.float32(gh)) == 2]
    mask = np.zeros((H, W), bool)
    mask[np.ix_(ys, xs)] = True
    assert np.all(img[~mask][:, :3] == 0) and np.all(img[..., 3] == 1)
    assert np.all(img[mask][:, :3] >= np.array([0.25, 0.5, 1.0], np.float32))  # emission + non-negative light
    assert st["paths"] == 2 * W * H


def test_gbuffer_primary_matches_trace(cornell):
    d, sb = cornell
    W, H = 32, 24
    gb = oracle.gbuffer_primary(sb, d.view, W, H)
    valid = gb[..., 3].view(np.uint32)
    assert set(np.unique(valid)) <= {0, 1}
    n = np.linalg.norm(gb[..., 4:7], axis=-1)
    assert np.allclose(n[valid == 1], 1.0, atol=1e-5)
    assert np.all(gb[valid == 0] == 0)
