"""Several GPUs, one process per GPU (torch.distributed).

Pixels and sample streams are independent, so the frame itself needs no
exchange: every rank traces its own sample stream of the same frame (seed =
rank) into its own target.  Two steps do exchange data, once each:

* ``broadcast_scene``: the scene is prepared once (meshes, BVHs, instances,
  light CDFs) on the source rank and its 13 bind-group buffers are sent to the
  others, which load them with ``Scene.set_buffers`` (validated on arrival);
* ``combine_images``: after k frames every rank holds the mean of its own k
  samples per texel; the all-ranks image is the mean of those means (equal
  counts), one all-reduce of the float4 image (33 MB at 1080p).

Batched frames shard without any exchange: ``assign_scenes`` splits a batch
of scenes over the ranks by estimated cost (the same answer on every rank,
computed locally), and each rank renders its share with one
``pulse_render_batch`` call (``render_batch_share``).

Both are collectives: every rank calls them in the same order.  On NCCL the
tensors live on the rank's GPU; ``target_view`` gives a zero-copy tensor over
a target's device image for that.

Stream order.  The library enqueues its work on its context's stream (its own
non-blocking stream unless the caller set one), torch and NCCL on torch's
current stream.  ``target_view`` and ``combine_images`` therefore make
torch's current stream wait for the work the library has enqueued so far
(an event, no host synchronisation), and ``combine_images`` makes the
library's stream wait for the collective before the library's next render
writes the image again.  A render enqueued after ``target_view`` was called
is ordered only by a later ``combine_images`` (or ``after_library``) call.
With frame pipelining on (``Context.set_pipeline(2)``) frames run on streams
of the context's own; the stream these helpers wait for
(``pulse_ctx_get_stream``) waits for the frames queued before the call.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist

from .layout import SceneBuffers

# The 12 arrays of SceneBuffers.arrays(), in that order, with their row widths.
_FIELDS = [("primitives", np.float32, 12), ("triangle_data", np.float32, 20), ("triangle_indices", np.uint32, 0),
           ("blas_nodes", np.uint32, 8), ("tlas_nodes", np.uint32, 8), ("instance_indices", np.uint32, 0),
           ("instances", np.uint32, 40), ("materials", np.float32, 12),
           ("light_emission_strength_cdf", np.float32, 0), ("light_triangle_area_cdfs", np.float32, 0),
           ("light_mesh_areas", np.float32, 0), ("light_indices", np.uint32, 2)]


def _device_for(group=None) -> torch.device:
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
        else torch.device("cpu")


def broadcast_scene(sb: SceneBuffers | None, src: int = 0, group=None) -> SceneBuffers:
    """The source rank's scene buffers on every rank (``sb`` is read on
    ``src`` only).  Row counts go first, then each array as raw 32-bit words."""
    dev = _device_for(group)
    rank = dist.get_rank(group)
    counts = torch.zeros(2 + len(_FIELDS), dtype=torch.int64, device=dev)
    if rank == src:
        arrs = sb.arrays()
        counts[0], counts[1] = sb.instance_count, sb.light_count
        for i, a in enumerate(arrs):
            counts[2 + i] = int(np.asarray(a).size)
    dist.broadcast(counts, src, group=group)
    c = counts.cpu().tolist()
    out = {}
    for i, (name, dtype, width) in enumerate(_FIELDS):
        n = c[2 + i]
        if rank == src:
            words = np.ascontiguousarray(getattr(sb, name), dtype=dtype).reshape(-1).view(np.int32)
            t = torch.from_numpy(words.copy()).to(dev)
        else:
            t = torch.empty(n, dtype=torch.int32, device=dev)
        if n:
            dist.broadcast(t, src, group=group)
        a = t.cpu().numpy().view(dtype)
        out[name] = a.reshape(-1, width) if width else a
    return SceneBuffers(instance_count=c[0], light_count=c[1], **out)


class _CudaArray:
    """__cuda_array_interface__ of a library-owned device buffer (no copy)."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


def _library_stream(ctx) -> torch.cuda.ExternalStream:
    return torch.cuda.ExternalStream(ctx.stream_ptr(), device=torch.device("cuda", torch.cuda.current_device()))


def after_library(ctx):
    """Make torch's current stream wait for the work ctx has enqueued so far."""
    torch.cuda.current_stream().wait_stream(_library_stream(ctx))


def library_after_torch(ctx):
    """Make ctx's stream wait for the work enqueued on torch's current stream
    so far (before the library writes memory torch is still using)."""
    _library_stream(ctx).wait_stream(torch.cuda.current_stream())


def target_view(target) -> torch.Tensor:
    """A (H, W, 4) float32 CUDA tensor over the target's device image (the
    library keeps owning it; valid until the target is destroyed).  Torch's
    current stream is ordered after the library's work enqueued so far, and
    the tensor remembers the context (``combine_images`` orders again)."""
    t = torch.as_tensor(_CudaArray(target.device_ptr(), (target.height, target.width, 4), "<f4"), device="cuda")
    after_library(target.ctx)
    t.pulse_ctx = target.ctx
    return t


def combine_images(image: torch.Tensor, group=None, ctx=None) -> torch.Tensor:
    """In place: every rank's image becomes the mean over ranks (each rank's
    image being the mean of the same number of its own samples).  For an
    image from ``target_view`` (or with ctx given) the collective waits for
    the library's enqueued renders, and the library's later work waits for
    the collective."""
    ctx = ctx if ctx is not None else getattr(image, "pulse_ctx", None)
    on_gpu = image.is_cuda and ctx is not None
    if on_gpu:
        after_library(ctx)
    world = dist.get_world_size(group)
    if world > 1:
        dist.all_reduce(image, op=dist.ReduceOp.SUM, group=group)
        image.div_(float(world))
    if on_gpu:
        library_after_torch(ctx)
    return image


def scene_cost(width: int, height: int, spp: int, max_depth: int, triangles: int) -> float:
    """Estimated cost of one scene's frame: paths x bounces x traversal steps
    per ray, the last growing with the logarithm of the triangle count (the
    depth of the trees).  Only ratios between scenes matter."""
    return float(width) * height * spp * max(max_depth, 1) * (8.0 + np.log2(max(triangles, 2)))


def assign_scenes(costs, world: int):
    """Longest-processing-time split of scenes over ranks: scenes in
    decreasing cost (ties by index) go to the rank with the least total so
    far (ties to the lower rank).  Deterministic, so every rank computes the
    same assignment without communicating.  Returns one sorted index list per
    rank; the largest rank load is at most 4/3 of the optimum (Graham)."""
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    loads = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        out[r].append(i)
        loads[r] += float(costs[i])
    return [sorted(x) for x in out]


def render_batch_share(ctx, items, costs, rank: int, world: int, **params):
    """This rank's share of a batched frame: the items assign_scenes gives
    it, rendered by one pulse_render_batch call (no exchange between ranks).
    Returns the indices rendered here."""
    from .tracer import render_batch
    mine = assign_scenes(costs, world)[rank]
    if mine:
        render_batch(ctx, [items[i] for i in mine], **params)
    return mine
