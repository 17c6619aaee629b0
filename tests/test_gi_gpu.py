"""The realtime GI mode on the GPU (pulse_gbuffer_primary + pulse_render_gi)
against the oracle's restatement of src/pulse/gi.wgsl:56-135, bit for bit:
the primary-hit G-buffer, the GI image from host and device G-buffers, G-buffers
of another resolution than the output, invalid (sky) texels, every launch shape."""
import numpy as np
import pytest

import oracle
from pulse_b200 import _ffi, scenes
from pulse_b200.tracer import PulseError, Scene, Target, gbuffer_primary, render_gi

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cornell_sb():
    d = scenes.cornell(48, 40)
    return d, oracle.assemble(d.meshes, d.materials, d.instances, 16, 4)


@pytest.fixture(scope="module")
def spheres_sb():
    d = scenes.spheres_1080p(level=4, n_instances=16, width=96, height=54)
    return d, oracle.assemble(d.meshes, d.materials, d.instances, 20, 8)


def _same(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


@pytest.mark.parametrize("which", ["cornell_sb", "spheres_sb"])
@pytest.mark.parametrize("quirks", [1, 0])
def test_gbuffer_primary_bit_exact(ctx, request, which, quirks):
    d, sb = request.getfixturevalue(which)
    sc = Scene(ctx)
    sc.set_buffers(sb)
    got = gbuffer_primary(sc, d.view, d.width, d.height, quirks=quirks)
    sc.close()
    ref = oracle.gbuffer_primary(sb, d.view, d.width, d.height, quirks=quirks)
    assert _same(got, ref)


@pytest.mark.parametrize("which", ["cornell_sb", "spheres_sb"])
@pytest.mark.parametrize("params", [dict(), dict(light_pick=1), dict(no_roulette=1, max_depth=3),
                                    dict(seed=7, spp=3), dict(spp=1, max_depth=0), dict(quirks=0)])
def test_render_gi_bit_exact(ctx, request, which, params):
    d, sb = request.getfixturevalue(which)
    W, H = d.width, d.height
    gb = oracle.gbuffer_primary(sb, d.view, W, H, **params)
    ref, _ = oracle.render_gi(sb, gb, W, H, **{"spp": 2, "max_depth": 5, **params})
    sc = Scene(ctx)
    sc.set_buffers(sb)
    tg = Target(ctx, W, H)
    render_gi(sc, gb, tg, **params)
    got = tg.download()
    tg.close()
    sc.close()
    assert _same(got, ref)


@pytest.mark.parametrize("gsize", [(2.0, 2.0), (0.5, 0.5), (1.37, 0.73)])
def test_render_gi_other_gbuffer_resolution(ctx, spheres_sb, gsize):
    d, sb = spheres_sb
    W, H = d.width, d.height
    gw, gh = max(1, int(W * gsize[0])), max(1, int(H * gsize[1]))
    gb = oracle.gbuffer_primary(sb, d.view, gw, gh)
    ref, _ = oracle.render_gi(sb, gb, W, H, spp=2, max_depth=5)
    sc = Scene(ctx)
    sc.set_buffers(sb)
    tg = Target(ctx, W, H)
    render_gi(sc, gb, tg)
    got = tg.download()
    tg.close()
    sc.close()
    assert _same(got, ref)


def test_render_gi_device_gbuffer_and_launch_shapes(ctx, spheres_sb):
    import torch
    d, sb = spheres_sb
    W, H = d.width, d.height
    sc = Scene(ctx)
    sc.set_buffers(sb)
    dev = torch.zeros(H * W * 16, dtype=torch.float32, device="cuda")
    gbuffer_primary(sc, d.view, W, H, out=dev)
    torch.cuda.synchronize()
    host = dev.cpu().numpy().reshape(H, W, 16)
    assert _same(host, oracle.gbuffer_primary(sb, d.view, W, H))
    ref, _ = oracle.render_gi(sb, host, W, H, spp=2, max_depth=5)
    assert (host[..., 3].view(np.uint32) == 0).any()  # the sky: invalid texels
    tg = Target(ctx, W, H)
    for shape in [dict(), dict(wf_segments=1), dict(wf_segments=6), dict(wf_segments=0xFFFFFFFF),
                  dict(trace_blocks=3), dict(trace_blocks=8, step_policy=1), dict(stack_depth=24)]:
        render_gi(sc, dev, tg, gw=W, gh=H, **shape)
        assert _same(tg.download(), ref), shape
    tg.close()
    sc.close()


def test_render_gi_rejects(ctx, cornell_sb):
    import torch
    d, sb = cornell_sb
    sc = Scene(ctx)
    tg = Target(ctx, 8, 8)
    gb = np.zeros((8, 8, 16), np.float32)
    with pytest.raises(PulseError) as e:
        render_gi(sc, gb, tg)
    assert e.value.code == _ffi.PULSE_ERR_NOT_READY
    sc.set_buffers(sb)
    dev = torch.zeros(8 * 8 * 16 + 1, dtype=torch.float32, device="cuda")
    with pytest.raises(PulseError) as e:
        render_gi(sc, dev[1:], tg, gw=8, gh=8)  # 4-byte offset: not 16-byte aligned
    assert e.value.code == _ffi.PULSE_ERR_INVALID_ARG
    with pytest.raises(PulseError) as e:
        render_gi(sc, np.zeros((0, 8, 16), np.float32), tg)
    assert e.value.code == _ffi.PULSE_ERR_INVALID_ARG
    tg.close()
    sc.close()
