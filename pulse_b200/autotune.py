"""Launch-shape autotuner for the renderer, with a persisted JSON cache.

The knobs are the render parameters that change speed but never the image
(every setting renders the same bits, which the parity tests check): the
kernel family (1 megakernel, 2 wavefront), the megakernel's register budget
(``min_blocks``), the wavefront/tail split (``wf_segments``), the persistent
traversal grid (``trace_blocks`` per SM), the traversal block size
(``block_size``: threads per block of the persistent traversal kernels), the
warp step policy of the traversal (``step_policy``: which of the lanes'
pending actions -- node visit, triangle test, instance entry or exit -- a
warp's step performs) and the ray-sort policy (``ray_sort``: whether each
bounce's queue is reordered by direction octant and origin cell before it is
traced).

The traversal stack depth is not searched by default.  The library sizes the
stacks from the trees' levels (min(stack_depth, levels - 1) per level), so
every depth at or above levels - 1 runs the same code, and a depth below it
can drop a subtree on some ray the tuning frames did not trace, which changes
the image and switches the exact culling shortcuts off.  A caller who passes
``stack_depth`` in an explicit space still gets the old guard: a candidate is
kept only if its frames dropped no push and hit no iteration cap.

``tune`` times one library render call per candidate with the context's own
CUDA events (``last_render_ms``) and walks the knobs one at a time
(coordinate descent from the defaults), so a tuning run costs about
(candidates x (warmup + reps)) frames.  Results are keyed by device name and a
workload signature and stored as JSON at ``path`` (default
``$PULSE_AUTOTUNE_CACHE`` or ``~/.cache/pulse_b200/autotune.json``).
"""
from __future__ import annotations

import json
import os
import statistics
from pathlib import Path

TAIL_ONLY = 0xFFFFFFFF  # wf_segments value: no wavefront segments


def step_weights(node: int, tri: int, enter: int, leave: int) -> int:
    """step_policy value of the warp step weights (one byte each)."""
    return node | (tri << 8) | (enter << 16) | (leave << 24)


DEFAULT_SPACE = {
    # wavefront segments before the persistent kernel; TAIL_ONLY: the
    # persistent kernel runs every path (one traversal launch per frame)
    "wf_segments": [1, 2, 3, 4, TAIL_ONLY],
    "trace_blocks": [4, 5, 6, 8],
    # threads per traversal block: 0 = 128, or 64 (same threads per SM)
    "block_size": [0, 64],
    # 0 = library default weights, 1 = divergent steps, then weight variants
    "step_policy": [0, 1, step_weights(15, 30, 15, 20), step_weights(15, 25, 45, 45)],
    # reorder each bounce's queue by direction octant and origin cell
    "ray_sort": [0, 1],
}
MEGA_SPACE = {"min_blocks": [4, 6, 8]}
# the library's value of each knob when the parameter is left out
KNOB_DEFAULTS = {"wf_segments": 0, "trace_blocks": 0, "stack_depth": 32, "min_blocks": 0, "step_policy": 0,
                 "iter_cap": 100000, "block_size": 0, "ray_sort": 0}


def cache_path(path=None) -> Path:
    if path:
        return Path(path)
    env = os.environ.get("PULSE_AUTOTUNE_CACHE")
    if env:
        return Path(env)
    return Path.home() / ".cache" / "pulse_b200" / "autotune.json"


def _load(path: Path) -> dict:
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(path: Path, data: dict):
    path.parent.mkdir(parents=True, exist_ok=True)
    tmp = path.with_suffix(".tmp")
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def device_name(index: int = 0) -> str:
    try:
        import torch
        return torch.cuda.get_device_name(index)
    except Exception:
        return "cuda"


def signature(kind: str, paths: int, triangles: int, n_scenes: int, params: dict) -> str:
    """Workload key: sizes rounded to powers of two, estimator and depth exact."""
    def p2(x):
        return 1 << max(0, int(x) - 1).bit_length()
    return (f"{kind}|scenes={n_scenes}|paths~{p2(paths)}|tris~{p2(triangles)}|mode={params.get('nee_mode', 0)}"
            f"|depth={params.get('max_depth', 5)}|spp={params.get('spp', 1)}")


def _guards(ctx) -> tuple:
    st = ctx.stats()
    return st["stack_overflows"], st["iter_cap_hits"]


def _time(ctx, call, params: dict, warmup: int, reps: int):
    """Median frame time over reps calls and whether any traversal guard
    fired (a dropped stack push or an iteration cap hit).  The frame time is
    what call returns, else the context's last_render_ms."""
    g0 = _guards(ctx)
    for _ in range(warmup):
        call(params)
    ms = []
    for _ in range(reps):
        r = call(params)
        st = ctx.stats()  # synchronizes the context's stream
        ms.append(float(r) if r is not None else st["last_render_ms"])
    return statistics.median(ms), _guards(ctx) != g0


def tune(ctx, call, base: dict, key: str, space: dict | None = None, warmup: int = 1, reps: int = 2,
         path=None, force: bool = False, log=None) -> dict:
    """Best render parameters for `call(params)` (one frame: a library render
    call, or several returning their own time in ms).

    base: the render parameters the knobs are added to; key: the workload
    signature (see signature()).  A cached result for (device, key) is returned
    without timing unless force is set.  Returns base updated with the winning
    knobs; the timing table is stored beside them in the cache."""
    p = cache_path(path)
    data = _load(p)
    full = f"{device_name()}|{key}"
    if not force and full in data:
        return dict(base, **data[full]["best"])
    space = DEFAULT_SPACE if space is None else space
    best = dict(base)
    for k in space:
        best.setdefault(k, KNOB_DEFAULTS.get(k, 0))
    best_ms, overflow = _time(ctx, call, best, warmup, reps)
    table = [{"params": {k: best.get(k, 0) for k in space}, "ms": best_ms, "overflow": overflow}]
    for knob, values in space.items():
        for v in values:
            if best.get(knob) == v:
                continue
            cand = dict(best, **{knob: v})
            ms, overflow = _time(ctx, call, cand, warmup, reps)
            table.append({"params": {k: cand.get(k, 0) for k in space}, "ms": ms, "overflow": overflow})
            if log:
                log(f"{knob}={v}: {ms:.3f} ms{' (stack overflow)' if overflow else ''}")
            if not overflow and ms < best_ms:
                best, best_ms = cand, ms
    chosen = {k: best[k] for k in space}
    data[full] = {"best": chosen, "ms": best_ms, "table": table}
    _store(p, data)
    return dict(base, **chosen)
