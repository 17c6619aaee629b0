"""Batched rendering (pulse_render_batch): several scenes of uneven sizes,
resolutions, bounce limits and seeds in one wavefront frame.

Every item's image must be bit-identical to the oracle's render of that item
alone with the item's max_depth and seed, over several accumulated frames, with
and without the CUDA graph, and across batch compositions that change between
calls (the context's graph is then instantiated anew).
"""
import numpy as np
import pytest

import oracle
from pulse_b200 import _ffi, scenes
from pulse_b200.tracer import BatchItem, PulseError, Scene, Target, render_batch, render_forward

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trio():
    """(desc, buffers) of three scenes: Cornell box, sparse spheres, dense spheres."""
    out = []
    d = scenes.cornell(48, 40)
    out.append((d, oracle.assemble(d.meshes, d.materials, d.instances, 16, 4)))
    d = scenes.spheres_1080p(level=4, n_instances=16, width=96, height=54)
    out.append((d, oracle.assemble(d.meshes, d.materials, d.instances, 20, 8)))
    d = scenes.spheres_1080p(level=3, n_instances=24, width=40, height=30, box=3.0, seed=5)
    out.append((d, oracle.assemble(d.meshes, d.materials, d.instances, 20, 8)))
    return out


# (scene index, max_depth (0 = params'), seed) of the batch items
ITEMS = [(0, 0, 11), (1, 3, 12), (2, 8, 13), (0, 1, 14), (1, 0, 0)]


def _setup(ctx, trio, items):
    scs = []
    for d, sb in trio:
        sc = Scene(ctx)
        sc.set_buffers(sb)
        scs.append(sc)
    tgs = [Target(ctx, trio[i][0].width, trio[i][0].height) for i, _, _ in items]
    return scs, tgs


def _close(scs, tgs):
    for x in tgs + scs:
        x.close()


def _oracle_frames(trio, items, frames, params):
    refs = []
    for i, md, seed in items:
        d, sb = trio[i]
        img = np.zeros((d.height, d.width, 4), np.float32)
        p = dict(params, seed=seed, max_depth=md or params["max_depth"])
        for acc in range(frames):
            oracle.render(sb, d.view, d.width, d.height, acc, image=img, **p)
        refs.append(img)
    return refs


def _assert_same(got, ref, what):
    diff = got.view(np.uint32) != ref.view(np.uint32)
    assert not diff.any(), f"{what}: {diff.any(axis=2).sum()} of {ref.shape[0] * ref.shape[1]} texels differ"


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("graph", [True, False])
def test_batch_bit_exact(ctx, trio, mode, graph):
    params = dict(max_depth=5, nee_mode=mode, light_pick=1 if mode == 2 else 0, quirks=1)
    scs, tgs = _setup(ctx, trio, ITEMS)
    for acc in range(3):
        batch = [BatchItem(scs[i], trio[i][0].view, tgs[k], acc, md, seed) for k, (i, md, seed) in enumerate(ITEMS)]
        render_batch(ctx, batch, graph=graph, **params)
    refs = _oracle_frames(trio, ITEMS, 3, params)
    for k, ref in enumerate(refs):
        assert np.isfinite(ref).all()
        _assert_same(tgs[k].download(), ref, f"item {k}")
    _close(scs, tgs)


@pytest.mark.parametrize("trace_blocks,wf_segments,block_size,ray_sort", [(1, 0, 0, 0), (2, 1, 0, 0), (8, 3, 0, 0),
                                                                         (3, 20, 0, 0), (5, 3, 64, 0), (5, 4, 0, 1),
                                                                         (8, 20, 64, 1), (8, 0xFFFFFFFF, 0, 0),
                                                                         (4, 0xFFFFFFFF, 64, 0)])
def test_batch_launch_shapes(ctx, trio, trace_blocks, wf_segments, block_size, ray_sort):
    """Traversal grid size, block size, the wavefront/tail split (0xFFFFFFFF:
    one persistent kernel for every path) and the ray sort change nothing."""
    params = dict(max_depth=6, nee_mode=2, light_pick=1, quirks=0, trace_blocks=trace_blocks,
                  wf_segments=wf_segments, block_size=block_size, ray_sort=ray_sort)
    scs, tgs = _setup(ctx, trio, ITEMS)
    batch = [BatchItem(scs[i], trio[i][0].view, tgs[k], 0, md, seed) for k, (i, md, seed) in enumerate(ITEMS)]
    render_batch(ctx, batch, **params)
    refs = _oracle_frames(trio, ITEMS, 1, params)
    for k, ref in enumerate(refs):
        _assert_same(tgs[k].download(), ref, f"item {k}")
    _close(scs, tgs)


def test_batch_equals_forward_and_composition_changes(ctx, trio):
    """Batches of 1, 5, 2 and 5 items in a row (graph re-instantiated or
    updated in place) each equal the per-scene forward render."""
    params = dict(max_depth=5, nee_mode=2, light_pick=1, quirks=0, spp=2)
    scs, tgs = _setup(ctx, trio, ITEMS)
    solo = [Target(ctx, trio[i][0].width, trio[i][0].height) for i, _, _ in ITEMS]
    for sel in ([2], [0, 1, 2, 3, 4], [4, 1], [0, 1, 2, 3, 4]):
        batch = [BatchItem(scs[ITEMS[k][0]], trio[ITEMS[k][0]][0].view, tgs[k], 0, ITEMS[k][1], ITEMS[k][2])
                 for k in sel]
        render_batch(ctx, batch, **params)
        for k in sel:
            i, md, seed = ITEMS[k]
            render_forward(scs[i], trio[i][0].view, solo[k], 0, **dict(params, seed=seed,
                                                                         max_depth=md or params["max_depth"]))
            _assert_same(tgs[k].download(), solo[k].download(), f"selection {sel} item {k}")
    _close(scs, tgs + solo)


def test_batch_rejects_bad_input(ctx, trio):
    scs, tgs = _setup(ctx, trio, ITEMS[:2])
    d = trio[0][0]
    with pytest.raises(PulseError) as e:
        render_batch(ctx, [])
    assert e.value.code == _ffi.PULSE_ERR_INVALID_ARG
    with pytest.raises(PulseError) as e:
        render_batch(ctx, [BatchItem(scs[0], d.view, tgs[0]), BatchItem(scs[0], d.view, tgs[0])])
    assert e.value.code == _ffi.PULSE_ERR_INVALID_ARG and "repeated" in str(e.value)
    many = [BatchItem(scs[0], d.view, tgs[0])] * 65
    with pytest.raises(PulseError) as e:
        render_batch(ctx, many)
    assert e.value.code == _ffi.PULSE_ERR_INVALID_ARG
    empty = Scene(ctx)
    with pytest.raises(PulseError) as e:
        render_batch(ctx, [BatchItem(empty, d.view, tgs[0])])
    assert e.value.code == _ffi.PULSE_ERR_NOT_READY
    empty.close()
    # nothing above touched the targets' device work: a valid batch still renders
    render_batch(ctx, [BatchItem(scs[0], d.view, tgs[0], 0, 0, 3)], max_depth=2)
    _close(scs, tgs)
