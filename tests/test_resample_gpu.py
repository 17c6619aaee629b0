"""The upscaling hand-off (pulse_target_resample) against a NumPy restatement
of the same float32 arithmetic and float16 rounding, bit for bit."""
import numpy as np
import pytest

from pulse_b200 import scenes
from pulse_b200.tracer import Scene, Target, render_forward

pytestmark = pytest.mark.gpu


def resample_ref(src: np.ndarray, out_w: int, out_h: int, filt: int) -> np.ndarray:
    """src (H, W, 4) float32 -> (out_h, out_w, 4) float16; see resample.cu."""
    H, W = src.shape[:2]
    f32 = np.float32
    u = (np.arange(out_w, dtype=f32) + f32(0.5)) / f32(out_w)
    v = (np.arange(out_h, dtype=f32) + f32(0.5)) / f32(out_h)
    if filt == 0:
        sx = np.minimum(np.floor(u * f32(W)).astype(np.int64), W - 1)
        sy = np.minimum(np.floor(v * f32(H)).astype(np.int64), H - 1)
        out = src[sy[:, None], sx[None, :]]
    else:
        px = u * f32(W) - f32(0.5)
        py = v * f32(H) - f32(0.5)
        fx0, fy0 = np.floor(px), np.floor(py)
        fx, fy = (px - fx0).astype(f32), (py - fy0).astype(f32)
        ix, iy = fx0.astype(np.int64), fy0.astype(np.int64)
        x0, x1 = np.clip(ix, 0, W - 1), np.clip(ix + 1, 0, W - 1)
        y0, y1 = np.clip(iy, 0, H - 1), np.clip(iy + 1, 0, H - 1)
        a, b = src[y0[:, None], x0[None, :]], src[y0[:, None], x1[None, :]]
        c, d = src[y1[:, None], x0[None, :]], src[y1[:, None], x1[None, :]]
        FX, FY = fx[None, :, None], fy[:, None, None]
        one = f32(1.0)
        w00, w10, w01, w11 = (one - FX) * (one - FY), FX * (one - FY), (one - FX) * FY, FX * FY
        out = ((a * w00 + b * w10) + c * w01) + d * w11
    return out.astype(np.float32).astype(np.float16)


@pytest.fixture(scope="module")
def rendered(ctx):
    desc = scenes.cornell(37, 23)  # odd sizes: non-integer scale factors
    sc = Scene(ctx)
    ids = [sc.upload_mesh(m, 16, 4) for m in desc.meshes]
    sc.set_materials(desc.materials)
    sc.set_instances(desc.instances, ids)
    tg = Target(ctx, desc.width, desc.height)
    for acc in range(2):
        render_forward(sc, desc.view, tg, acc, max_depth=4, nee_mode=2, light_pick=1, quirks=0)
    yield tg, tg.download()
    tg.close()
    sc.close()


@pytest.mark.parametrize("filt", [0, 1])
@pytest.mark.parametrize("size", [(37, 23), (74, 46), (100, 61), (16, 9), (1, 1)])
def test_resample_bit_exact(rendered, filt, size):
    tg, img = rendered
    got = tg.resample(size[0], size[1], filt)
    ref = resample_ref(img, size[0], size[1], filt)
    assert np.array_equal(got.view(np.uint16), ref.view(np.uint16))


def test_resample_identity_nearest(rendered):
    tg, img = rendered
    got = tg.resample(img.shape[1], img.shape[0], 0)
    assert np.array_equal(got.view(np.uint16), img.astype(np.float16).view(np.uint16))


def test_resample_rejects(ctx, rendered):
    from pulse_b200.tracer import PulseError
    tg, _ = rendered
    with pytest.raises(PulseError):
        tg.resample(8, 8, 2)
    with pytest.raises(PulseError):
        tg.resample(0, 8, 0)


def test_accumulation_checkpoint_resume(ctx):
    """Frames 0-2, download + count (the checkpoint), a fresh target restored
    with pulse_target_upload, frames 3-5: the image of six uninterrupted frames."""
    d = scenes.cornell(48, 32)
    import oracle
    sb = oracle.assemble_desc(d)
    sc = Scene(ctx)
    sc.set_buffers(sb)
    params = dict(max_depth=5, nee_mode=2, light_pick=1, quirks=0)
    tg = Target(ctx, 48, 32)
    for k in range(6):
        render_forward(sc, d.view, tg, k, **params)
    straight = tg.download()
    for k in range(3):
        render_forward(sc, d.view, tg, k, **params)
    saved, count = tg.download(), 3
    tg.close()
    tg2 = Target(ctx, 48, 32)
    tg2.upload(saved)
    for k in range(count, 6):
        render_forward(sc, d.view, tg2, k, **params)
    resumed = tg2.download()
    tg2.close()
    sc.close()
    assert np.array_equal(resumed.view(np.uint32), straight.view(np.uint32))


def test_async_download_overlaps_the_next_frame(ctx):
    """pulse_target_download_async of frame k returns frame k's texels even
    though frame k+1 is enqueued before the wait (its accumulation waits for
    the copy), and frame k+1 is the two-frame running mean."""
    import ctypes as C

    import torch

    import oracle
    d = scenes.cornell(320, 240)
    sb = oracle.assemble_desc(d)
    sc = Scene(ctx)
    sc.set_buffers(sb)
    tg = Target(ctx, 320, 240)
    params = dict(max_depth=4, nee_mode=2, light_pick=1, quirks=0, spp=16)
    host = torch.empty((240, 320, 4), dtype=torch.float32, pin_memory=True)
    lib = ctx.lib
    render_forward(sc, d.view, tg, 0, **params)
    assert lib.pulse_target_download_async(tg.h, C.c_void_p(host.data_ptr())) == 0
    render_forward(sc, d.view, tg, 1, **params)
    assert lib.pulse_target_download_wait(tg.h) == 0
    frame0 = host.numpy().copy()
    frame1 = tg.download()
    ref0, _ = oracle.render(sb, d.view, 320, 240, 0, **params)
    ref1 = ref0.copy()
    oracle.render(sb, d.view, 320, 240, 1, image=ref1, **params)
    assert np.array_equal(frame0.view(np.uint32), ref0.view(np.uint32))
    assert np.array_equal(frame1.view(np.uint32), ref1.view(np.uint32))
    tg.close()
    sc.close()
