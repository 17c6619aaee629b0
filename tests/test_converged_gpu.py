"""Converged images against the FP64 CPU oracle.

The GPU accumulates N frames of 1 sample (FP32 paths, running mean in FP32);
the oracle averages the same N sample indices with every path computed in
double precision.  Both follow the same random numbers, so a path only
changes where rounding flips one of its discrete decisions (a Russian-roulette
draw, a lobe choice, a triangle edge); such a path is an independent sample,
and in a scene with bright small lights it can be a firefly worth hundreds of
times a texel's value.  The stated bounds are therefore:
  * RMSE over the 99% of texels with the smallest difference <= 1e-3 x the
    image mean (every texel whose paths all agree matches to rounding);
  * at least 98.5% of texels within 1e-3 relative (1e-5 absolute floor);
the full RMSE is printed beside them.
"""
import numpy as np
import pytest

import oracle
from pulse_b200 import scenes
from pulse_b200.tracer import Scene, Target, render_forward

pytestmark = pytest.mark.gpu

TRIMMED_REL_RMSE = 1e-3
CLOSE_FRACTION = 0.985


def _gpu_mean(ctx, sb, desc, frames, params):
    sc = Scene(ctx)
    sc.set_buffers(sb)
    tg = Target(ctx, desc.width, desc.height)
    for acc in range(frames):
        render_forward(sc, desc.view, tg, acc, **params)
    img = tg.download()
    tg.close()
    sc.close()
    return img[..., :3].reshape(-1, 3).astype(np.float64)


@pytest.mark.parametrize("which,mode", [("cornell", 2), ("cornell", 0), ("cornell", 1), ("spheres", 2)])
def test_converged_rmse_vs_fp64(ctx, which, mode):
    if which == "cornell":
        desc = scenes.cornell(48, 36)
        sb = oracle.assemble(desc.meshes, desc.materials, desc.instances, 16, 4)
    else:
        desc = scenes.spheres_1080p(level=4, n_instances=16, width=64, height=36)
        sb = oracle.assemble(desc.meshes, desc.materials, desc.instances, 20, 8)
    params = dict(max_depth=6, nee_mode=mode, light_pick=1 if mode == 2 else 0, quirks=0)
    frames = 64
    got = _gpu_mean(ctx, sb, desc, frames, params)
    ref = oracle.render_mean64(sb, desc.view, desc.width, desc.height, frames, **params)
    d = np.abs(got - ref)
    worst = d.max(axis=1)
    keep = worst <= np.quantile(worst, 0.99)
    trimmed = float(np.sqrt(np.mean(d[keep] ** 2)))
    close = float(np.mean(worst <= np.maximum(1e-3 * ref.max(axis=1), 1e-5)))
    mean = float(np.mean(ref))
    print(f"{which} mode {mode}: rmse {np.sqrt(np.mean(d ** 2)):.3e}, trimmed {trimmed:.3e}, mean {mean:.3e}, "
          f"close {close:.4f}")
    assert mean > 0
    assert trimmed <= TRIMMED_REL_RMSE * mean
    assert close >= CLOSE_FRACTION
