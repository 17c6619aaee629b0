"""The multi-GPU helpers on one B200: the zero-copy view of a target's device
image, and broadcast_scene / combine_images over an NCCL group of one rank
(in a child process), whose scene renders like the source's."""
import os
import socket
import subprocess
import sys
import textwrap

import numpy as np
import pytest

import oracle
from pulse_b200 import scenes
from pulse_b200.tracer import Scene, Target, render_forward

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PARAMS = dict(max_depth=4, nee_mode=2, light_pick=1, quirks=0)


def test_target_view_is_the_device_image(ctx):
    import torch
    from pulse_b200.multigpu import target_view
    d = scenes.cornell(40, 24)
    sc = Scene(ctx)
    sc.set_buffers(oracle.assemble_desc(d))
    tg = Target(ctx, 40, 24)
    render_forward(sc, d.view, tg, 0, **PARAMS)
    v = target_view(tg)
    torch.cuda.synchronize()
    assert v.shape == (24, 40, 4) and v.is_cuda
    assert np.array_equal(v.cpu().numpy().view(np.uint32), tg.download().view(np.uint32))
    tg.close()
    sc.close()


def test_target_view_waits_for_the_render(ctx):
    """The library renders on its own non-blocking stream; a torch kernel
    reading the view right after the render call (no download, no
    synchronize) must see the finished frame: target_view orders torch's
    current stream after the library's enqueued work."""
    import torch
    from pulse_b200.multigpu import target_view
    d = scenes.cornell(256, 256)
    sc = Scene(ctx)
    sc.set_buffers(oracle.assemble_desc(d))
    tg = Target(ctx, 256, 256)
    for spp in (64, 128):  # a frame of several milliseconds on a fresh target
        render_forward(sc, d.view, tg, 0, **dict(PARAMS, spp=spp))
        snap = target_view(tg).clone()
        torch.cuda.synchronize()
        assert np.array_equal(snap.cpu().numpy().view(np.uint32), tg.download().view(np.uint32))
    tg.close()
    sc.close()


CHILD = textwrap.dedent("""
    import sys
    sys.path.insert(0, {root!r})
    import numpy as np, torch, torch.distributed as dist
    import oracle
    from pulse_b200 import multigpu, scenes
    from pulse_b200.tracer import Context, Scene, Target, render_forward
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:{port}", rank=0, world_size=1)
    d = scenes.cornell(40, 24)
    sb = oracle.assemble_desc(d)
    got = multigpu.broadcast_scene(sb, src=0)
    assert all(np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))
               for a, b in zip(got.arrays(), sb.arrays()))
    ctx = Context(0)
    sc = Scene(ctx); sc.set_buffers(got)
    tg = Target(ctx, 40, 24)
    # the collective right after the render call: no download, no synchronize
    render_forward(sc, d.view, tg, 0, **{params!r})
    img = multigpu.combine_images(multigpu.target_view(tg))
    snap = img.clone()
    # the library's next render waits for the collective
    render_forward(sc, d.view, tg, 1, **{params!r})
    torch.cuda.synchronize()
    ref, _ = oracle.render(sb, d.view, 40, 24, 0, **{params!r})
    assert np.array_equal(snap.cpu().numpy().view(np.uint32), ref.view(np.uint32))
    oracle.render(sb, d.view, 40, 24, 1, image=ref, **{params!r})
    assert np.array_equal(tg.download().view(np.uint32), ref.view(np.uint32))
    tg.close(); sc.close(); ctx.close()
    dist.destroy_process_group()
    print("nccl helpers ok")
""")


def test_helpers_over_nccl_one_rank():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    r = subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT, port=port, params=PARAMS)],
                       capture_output=True, text=True, timeout=300, env=dict(os.environ, NCCL_NVLS_ENABLE="0"))
    assert r.returncode == 0 and "nccl helpers ok" in r.stdout, (r.stdout[-1500:], r.stderr[-3000:])
