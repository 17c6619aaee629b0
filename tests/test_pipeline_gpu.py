"""Pipelined frames (pulse_ctx_set_pipeline(ctx, 2)): consecutive wavefront
frames run on two streams of the context and overlap.  The images must be
those of depth 1 bit for bit: every frame accumulates into its target after
the previous one, a scene update reaches the frames queued after it and no
frame queued before it, and every other call of the library waits for the
frames in flight.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from pulse_b200 import scenes
from pulse_b200.tracer import Context, Scene, Target, render_count, render_forward

pytestmark = pytest.mark.gpu

PARAMS = dict(max_depth=8, nee_mode=2, light_pick=1, quirks=0)


def _scene(ctx, desc):
    p = desc.params
    sc = Scene(ctx)
    ids = [sc.upload_mesh(m, p.get("bins", 20), p.get("max_leaf", 8)) for m in desc.meshes]
    sc.set_materials(desc.materials)
    sc.set_instances(desc.instances, ids)
    return sc, ids


def _run(depth, frames=7, wait_each=False):
    """Per frame: move every instance (pulse_instances_set), render with the
    running accumulation into one target, read the image back asynchronously
    into pinned memory; frame 3 moves a few instances with
    pulse_instances_update instead and frame 5 reads the image with a blocking
    download as well.  Returns every frame's image."""
    import torch
    ctx = Context(0)
    ctx.set_pipeline(depth)
    desc = scenes.spheres_1080p(level=3, n_instances=24)
    W, H = 96, 64
    sc, ids = _scene(ctx, desc)
    rng = np.random.default_rng(41)
    tg = Target(ctx, W, H)
    host = [torch.empty((H, W, 4), dtype=torch.float32, pin_memory=True) for _ in range(frames)]
    blocking = None
    for f in range(frames):
        for inst in desc.instances:
            inst.object_world = scenes.trs(rng.uniform(-10, 10, 3), scenes.random_rotation(rng))
        if f == 3:
            idx = np.array([0, 5, 9], np.uint32)
            sc.update_instances(idx, np.stack([desc.instances[i].columns() for i in idx]))
        else:
            sc.set_instances(desc.instances, ids)
        render_forward(sc, desc.view, tg, f, **PARAMS)
        if wait_each and f > 0:  # the previous frame's copy, with this frame already queued
            ctx.check(ctx.lib.pulse_target_download_wait(tg.h), "download wait")
        ctx.check(ctx.lib.pulse_target_download_async(tg.h, C.c_void_p(host[f].data_ptr())), "download")
        if f == 5:
            blocking = tg.download()
    ctx.check(ctx.lib.pulse_target_download_wait(tg.h), "download wait")
    imgs = [h.numpy().copy() for h in host]
    tg.close()
    sc.close()
    ctx.close()
    return imgs, blocking


def test_pipelined_frames_equal_serial_frames():
    serial, b1 = _run(1)
    piped, b2 = _run(2)
    for f, (a, b) in enumerate(zip(serial, piped)):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), f
    assert np.array_equal(b1.view(np.uint32), b2.view(np.uint32))
    assert np.array_equal(b2.view(np.uint32), piped[5].view(np.uint32))


def test_pipelined_frames_with_a_copy_wait_per_frame():
    """The real-time loop: frame k queued, then the wait for frame k-1's copy,
    then frame k's copy."""
    serial, _ = _run(1, wait_each=True)
    piped, _ = _run(2, wait_each=True)
    for f, (a, b) in enumerate(zip(serial, piped)):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), f


def test_pipelined_frames_into_several_targets():
    """Frames into three targets in turn (lanes and targets out of step), a
    counting render (which waits for the frames in flight) between them."""
    res = {}
    for depth in (1, 2):
        ctx = Context(0)
        ctx.set_pipeline(depth)
        desc = scenes.cornell(40, 32)
        sc, _ = _scene(ctx, desc)
        tgs = [Target(ctx, 40, 32) for _ in range(3)]
        for f in range(9):
            render_forward(sc, desc.view, tgs[f % 3], f // 3, **PARAMS)
            if f == 4:
                render_count(sc, desc.view, tgs[1], 1, **PARAMS)
                render_forward(sc, desc.view, tgs[1], 1, **PARAMS)  # accumulates over the counting frame's
        res[depth] = [t.download() for t in tgs]
        for t in tgs:
            t.close()
        sc.close()
        ctx.close()
    for a, b in zip(res[1], res[2]):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    # target 0 holds frames 0, 3 and 6 of the oracle's accumulation
    sb = oracle.assemble_desc(scenes.cornell(40, 32))
    ref = np.zeros((32, 40, 4), np.float32)
    for acc in range(3):
        oracle.render(sb, scenes.cornell(40, 32).view, 40, 32, acc, image=ref, **PARAMS)
    assert np.array_equal(res[2][0].view(np.uint32), ref.view(np.uint32))


def test_pipeline_depth_is_checked():
    from pulse_b200.tracer import PulseError
    ctx = Context(0)
    with pytest.raises(PulseError):
        ctx.set_pipeline(3)
    ctx.set_pipeline(2)
    ctx.set_pipeline(1)
    ctx.close()


def test_pipelined_frame_seen_through_target_view():
    """A torch consumer of the target's device image (multigpu.target_view,
    ordered through pulse_ctx_get_stream) reads the pipelined frame it follows."""
    import torch

    from pulse_b200 import multigpu
    ctx = Context(0)
    ctx.set_pipeline(2)
    desc = scenes.cornell(64, 48)
    sc, _ = _scene(ctx, desc)
    tg = Target(ctx, 64, 48)
    views = []
    for f in range(4):
        render_forward(sc, desc.view, tg, f, **PARAMS)
        views.append(multigpu.target_view(tg).clone())  # on torch's stream, after the frame
    torch.cuda.synchronize()
    final = tg.download()
    assert np.array_equal(views[-1].cpu().numpy().view(np.uint32), final.view(np.uint32))
    ref = np.zeros((48, 64, 4), np.float32)
    sb = oracle.assemble_desc(desc)
    for f in range(4):
        oracle.render(sb, desc.view, 64, 48, f, image=ref, **PARAMS)
        assert np.array_equal(views[f].cpu().numpy().view(np.uint32), ref.view(np.uint32)), f
    tg.close()
    sc.close()
    ctx.close()
