"""pulse_render_forward_noalloc: the render for callers that cannot allocate
device memory (engines that reserve all GPU memory up front, frame loops where
an allocation would synchronize the device).  Its path buffers live in a fixed
static device array; this checks, through the C ABI, that it produces exactly
the images of pulse_render_forward (wavefront kernels, same parameters) on two
calls in a row, and that it refuses frames beyond its 65536-path limit.

Collected last on purpose: its first call on a device performs the one-time
address lookup of the static array, and it must work both in a fresh process
and after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from pulse_b200 import scenes
from pulse_b200.tracer import PulseError, Scene, Target, make_view, render_forward, render_params

pytestmark = pytest.mark.gpu


def _noalloc(ctx, scene, view, target, acc, **params):
    v = make_view(view)
    p = render_params(**params)
    ctx.check(ctx.lib.pulse_render_forward_noalloc(scene.h, C.byref(v), target.h, acc, C.byref(p)),
              "pulse_render_forward_noalloc")


def test_noalloc_matches_render_forward(ctx):
    desc = scenes.cornell(96, 64)
    sb = oracle.assemble(desc.meshes, desc.materials, desc.instances, 16, 4)
    sc = Scene(ctx)
    sc.set_buffers(sb)
    ref_t = Target(ctx, 96, 64)
    got_t = Target(ctx, 96, 64)
    params = dict(max_depth=4, nee_mode=2, light_pick=1, kernel=2)
    for acc in range(2):  # two calls in a row, the second accumulating onto the first
        render_forward(sc, desc.view, ref_t, acc, **params)
        _noalloc(ctx, sc, desc.view, got_t, acc, **params)
        ref = ref_t.download()
        got = got_t.download()
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), f"call {acc}"
        assert np.isfinite(got).all() and got[..., :3].max() > 0
    ref_t.close()
    got_t.close()
    sc.close()


def test_noalloc_rejects_frames_beyond_the_fixed_buffer(ctx):
    desc = scenes.cornell(257, 256)  # 65792 paths > 65536
    sb = oracle.assemble(desc.meshes, desc.materials, desc.instances, 16, 4)
    sc = Scene(ctx)
    sc.set_buffers(sb)
    tg = Target(ctx, 257, 256)
    with pytest.raises(PulseError) as ei:
        _noalloc(ctx, sc, desc.view, tg, 0, max_depth=2)
    assert ei.value.code == -1 and "65536" in str(ei.value)
    tg.close()
    sc.close()
