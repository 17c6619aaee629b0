#!/usr/bin/env python
"""Throughput of the path-tracing hot path: Mpaths/s at 1920x1080.

Workload (the plain 1080p configuration): 64 rigid instances of one displaced
icosphere (subdivision 7, 327,680 triangles, noise amplitude 0.1) in a 20^3
box with per-instance GGX roughness U(0.05, 1), metallic Bernoulli(0.3),
albedo U(0, 1)^3, plus 8 emissive patches (256 emissive triangles, radiance
U(1, 20)); 1920x1080, 1 sample per pixel per frame, 8 bounces, next-event
estimation with the emission-strength (power) light CDF.  Synthetic, seeded.

A step is one frame: every pixel's path traced to termination and accumulated.
  value  Mpaths/s from CUDA events around each frame's render kernel on the
         launching stream, scene resident in HBM, L2 flushed between frames.
  e2e    the same metric through the C ABI per frame: instances uploaded from
         pinned host memory (prepare_mesh_instances + TLAS build on the
         device), the render, and the image read back to pinned host memory
         (pulse_target_download_async: frame k's copy overlaps frame k+1's
         tracing; the last frame's copy is waited for inside the timed region),
         with frame pipelining on (pulse_ctx_set_pipeline depth 2: frame k+1's
         first launches start while frame k's last ones drain); e2e.serial is
         the same loop at depth 1.
N GPUs: one process per GPU, each tracing its own sample stream of the same
frame (seed = rank); no collective in the timed region; max over ranks.

--impl reference times the CPU restatement of the reference path tracer (the
reference itself is Rust + WGSL through wgpu and cannot run on this machine)
on all host cores over a bounded sample of the same frame.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "Mpaths/s @1080p batched vs plain at equal RMSE; adjoint/forward time ratio"
WORKLOAD = ("spheres_1080p: 64 instances of a displaced icosphere (subdivision 7, 327,680 tris, amplitude 0.1) "
            "+ 8 emissive patches (256 tris, radiance U(1,20)); 1920x1080, 1 spp/frame, 8 bounces, "
            "NEE with power-proportional light CDF (corrected estimator, MIS), reference FP32 quirks off")
# The corrected estimator (nee_mode 2) runs with the reference's FP32 quirks off:
# the converged-image comparison against the FP64 oracle is only defined without
# them, and with them a BLAS miss records a hit ~1e30 away whose next segment
# traverses every node up to the iteration cap (parity with quirks on is tested).
PARAMS = dict(max_depth=8, nee_mode=2, light_pick=1, spp=1, quirks=0)
ORACLE_KEYS = ("max_depth", "nee_mode", "light_pick", "spp", "quirks", "seed")
TAIL_ONLY = 0xFFFFFFFF  # wf_segments: no wavefront segments, one persistent kernel per frame


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--level", type=int, default=7, help="icosphere subdivision (7 = the benchmark scene)")
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--min-blocks", type=int, default=0, help="megakernel register budget variant (0 = default)")
    ap.add_argument("--kernel", type=int, default=2, help="1 megakernel, 2 wavefront")
    ap.add_argument("--wf-segments", type=int, default=0,
                    help="wavefront segments before the tail kernel (0: the library default, 3)")
    ap.add_argument("--cpu-row-stride", type=int, default=1, help="row subsample of the CPU legs (1 = full frame)")
    ap.add_argument("--trace-blocks", type=int, default=0, help="wavefront traversal blocks per SM (0 = default)")
    ap.add_argument("--no-batch", action="store_true", help="skip the mixed-batch leg")
    ap.add_argument("--batch-steps", type=int, default=5, help="timed frames of the mixed-batch leg")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="skip autotuning both arms of the mixed-batch leg")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the differentiable (adjoint) leg")
    ap.add_argument("--no-gi", action="store_true", help="skip the realtime GI leg")
    ap.add_argument("--no-large", action="store_true", help="skip the large terrain leg (33.5M triangles, 4K)")
    ap.add_argument("--large-check", action="store_true", help="compare the full-size terrain BLAS with the "
                    "CPU builder (single-threaded, minutes; by default a 1024^2 terrain is compared)")
    ap.add_argument("--no-small", action="store_true", help="skip the small Cornell leg")
    ap.add_argument("--no-converged", action="store_true", help="skip the FP64 converged-image comparison")
    ap.add_argument("--gt-spp", type=int, default=1024, help="samples per texel of the FP64 ground truth")
    ap.add_argument("--large-n", type=int, default=4096, help="terrain vertices per side of the large leg")
    ap.add_argument("--adjoint-res", type=int, default=512, help="resolution of the adjoint leg")
    ap.add_argument("--autotune-cache", default=None, help="autotuner JSON cache path")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def measured_hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(name: str, key: str = "dram_bytes_per_frame"):
    """DRAM bytes per frame from a committed ncu summary (profiles/<name>.md), if any."""
    path = os.path.join(ROOT, "profiles", name + ".md")
    try:
        for line in open(path):
            if line.strip().startswith(key):
                return float(line.split("=")[1].split()[0])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1].split()[0]))
                mx = float(parts[2].split()[0])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def build_scene(ctx, desc):
    from pulse_b200.tracer import Scene
    p = desc.params
    sc = Scene(ctx)
    ids = []
    build_ms = []
    for m in desc.meshes:
        ids.append(sc.upload_mesh(m, p.get("bins", 20), p.get("max_leaf", 8)))
        build_ms.append(ctx.stats()["last_build_ms"])
    sc.set_materials(desc.materials)
    sc.set_instances(desc.instances, ids)
    return sc, ids, build_ms


def instance_descs(desc, ids):
    """The per-frame instance array (PulseInstanceDesc rows) in pinned host memory."""
    import ctypes as C

    import torch

    from pulse_b200 import _ffi
    n = len(desc.instances)
    pinned = torch.empty(n * C.sizeof(_ffi.InstanceDesc), dtype=torch.uint8, pin_memory=True)
    arr = (_ffi.InstanceDesc * n).from_address(pinned.data_ptr())
    for i, inst in enumerate(desc.instances):
        arr[i].object_world[:] = [float(x) for x in inst.columns()]
        arr[i].mesh_id = ids[inst.mesh]
        arr[i].material_index = inst.material
    return pinned, arr


def cpu_legs(desc, args, nthreads, steps=1, params=None):
    """The CPU restatement on a row subsample of the same frame (oracle port):
    frame 0 (accumulation count 0, seed 0) of PARAMS updated by params; the
    last step's image and texel list are returned with the rates."""
    import oracle
    W, H = desc.width, desc.height
    t0 = time.perf_counter()
    sb = oracle.assemble_desc(desc)
    prep_s = time.perf_counter() - t0
    from pulse_b200.layout import triangle_soup
    prims, _ = triangle_soup(desc.meshes[0])
    t0 = time.perf_counter()
    nodes, _ = oracle.build_blas(prims, desc.params.get("bins", 20), desc.params.get("max_leaf", 8))
    build_ms = (time.perf_counter() - t0) * 1e3
    rates, times = [], []
    stride = args.cpu_row_stride
    params = {k: v for k, v in dict(PARAMS, **(params or {})).items() if k in ORACLE_KEYS}
    for s in range(steps):
        rows = np.arange(s % stride, H, stride)
        pix = (rows[:, None] * W + np.arange(W)[None, :]).astype(np.uint32).ravel()
        img = np.zeros((H, W, 4), np.float32)
        t0 = time.perf_counter()
        oracle.render(sb, desc.view, W, H, 0, image=img, pixels=pix, nthreads=nthreads, **params)
        dt = time.perf_counter() - t0
        times.append(dt)
        rates.append(pix.size / dt / 1e6)
    return dict(rates=rates, times=times, paths=int(len(np.arange(0, H, stride)) * W), build_ms=build_ms,
                prep_s=prep_s, sb=sb, blas_nodes=nodes, n_tris=int(prims.shape[0]), image=img, pixels=pix)


def tree_depth(nodes) -> int:
    """Levels of a (N, 8) u32 BVH node array (root = level 1)."""
    depth, stack = 0, [(0, 1)]
    while stack:
        i, d = stack.pop()
        depth = max(depth, d)
        if nodes[i, 7] == 0:
            a = int(nodes[i, 3])
            stack += [(a, d + 1), (a + 1, d + 1)]
    return depth


def build_roofline(n_tris: int, nodes, gpu_ms: float, cpu_ms: float, peak: float) -> dict:
    """The BLAS build against HBM: per SAH level every triangle's 48 B primitive,
    12 B centroid and 4 B index are read once, plus 32 B per node written."""
    levels = tree_depth(nodes)
    algo = n_tris * (48 + 12 + 4) * levels + nodes.shape[0] * 32
    achieved = algo / (gpu_ms / 1e3) / 1e9
    return {"triangles": n_tris, "levels": levels, "algorithmic_bytes": algo, "gpu_ms": gpu_ms,
            "cpu_ms_1thread": cpu_ms, "speedup_vs_cpu": cpu_ms / gpu_ms, "achieved_gbs": achieved,
            "peak_gbs": peak, "frac": achieved / peak,
            "note": "latency-bound: nodes of at most 512 triangles are split in shared memory, one warp per node of a level"}


def subsample_pixels(W: int, H: int, stride: int = 4) -> np.ndarray:
    """Every stride-th row and column (stride 4: 1/16 of the texels)."""
    rows, cols = np.arange(0, H, stride), np.arange(0, W, stride)
    return (rows[:, None] * W + cols[None, :]).astype(np.uint32).ravel()


def _mse_stats(x: np.ndarray, gt: np.ndarray):
    """Mean over texels of the per-texel mean squared RGB error, and its
    standard error (texels are independent samples)."""
    e = np.mean((x - gt) ** 2, axis=1)
    return float(e.mean()), float(e.std(ddof=1) / math.sqrt(e.size)), e


def converged_vs_fp64(sb, desc, img, frames: int, params: dict, seed: int = 0, stride: int = 4,
                      gt_spp: int = 1024) -> dict:
    """The converged-image layer: the GPU's image (the running mean of
    `frames` samples per texel, seed `seed`) and the FP64 oracle's image of
    the same number of samples from an independent stream (seed + 1), both
    against an FP64 ground truth of gt_spp samples per texel (seed + 2), on
    every stride-th row and column.  Equal estimators give equal expected
    MSE; the difference of the two MSEs is reported in standard errors.

    Two same-stream checks sit beside it: the FP32 oracle accumulated over the
    same samples (seed `seed`) must equal the GPU's image bit for bit, and the
    FP64 oracle on that stream measures how many texels FP32 rounding sends
    down another path (a flipped roulette draw, lobe choice or triangle edge):
    those texels differ by a whole independent sample, so the fraction is a
    property of the scene and the precision, not of the GPU."""
    import oracle
    W, H = desc.width, desc.height
    pix = subsample_pixels(W, H, stride)
    op = {k: v for k, v in params.items() if k in ORACLE_KEYS and k != "seed"}
    t0 = time.perf_counter()
    gt = oracle.render_mean64(sb, desc.view, W, H, gt_spp, pixels=pix, seed=seed + 2, **op)
    t_gt = time.perf_counter() - t0
    ind = oracle.render_mean64(sb, desc.view, W, H, frames, pixels=pix, seed=seed + 1, **op)
    same64 = oracle.render_mean64(sb, desc.view, W, H, frames, pixels=pix, seed=seed, **op)
    acc = np.zeros((H, W, 4), np.float32)
    for a in range(frames):
        oracle.render(sb, desc.view, W, H, a, image=acc, pixels=pix, seed=seed, **op)
    gpu_rows = img.reshape(-1, 4)[pix]
    fp32_rows = acc.reshape(-1, 4)[pix]
    differ = int(np.any(gpu_rows.view(np.uint32) != fp32_rows.view(np.uint32), axis=1).sum())
    gpu = gpu_rows[:, :3].astype(np.float64)
    m_gpu, se_gpu, _ = _mse_stats(gpu, gt)
    m_ind, se_ind, _ = _mse_stats(ind, gt)
    z = (m_gpu - m_ind) / math.sqrt(se_gpu ** 2 + se_ind ** 2)
    d = np.abs(gpu - same64)
    worst = d.max(axis=1)
    return {"texels": int(pix.size), "subsample": f"every {stride}th row and column (1/{stride * stride})",
            "ground_truth": {"precision": "fp64", "samples_per_texel": gt_spp, "seed": seed + 2,
                             "seconds": t_gt, "mean": float(gt.mean())},
            "samples_per_texel": frames,
            "rmse_gpu": math.sqrt(m_gpu), "rmse_fp64_oracle_independent_stream": math.sqrt(m_ind),
            "rmse_ratio_gpu_over_fp64": math.sqrt(m_gpu / m_ind) if m_ind > 0 else None,
            "mse_difference_in_standard_errors": z,
            "equal_rmse": bool(abs(z) <= 3.0),
            "fp32_oracle_same_stream": {"texels_differing": differ, "bit_exact": differ == 0},
            "fp64_same_stream": {
                "close_fraction": float(np.mean(worst <= np.maximum(1e-3 * same64.max(axis=1), 1e-5))),
                "note": "texels whose paths all keep their decisions in FP64 agree to rounding; the rest "
                        "hold at least one path that FP32 rounding sent elsewhere (an independent sample)"}}


BATCH_WORKLOAD = ("mixed batch: 32 scenes, each a displaced icosphere + displaced ground grid + emissive disc, "
                  "triangles log-uniform in [10k, 2M], resolution drawn from {256^2, 512^2, 1280x720, 1920x1080}, "
                  "1-8 bounces per scene, NEE with power CDF, 1 spp/frame, per-scene seeds")


def batch_leg(ctx, stream, args):
    """Aggregate Mpaths/s of the mixed batch: every scene rendered by its own
    pulse_render_forward call (plain) against one pulse_render_batch frame
    (batched, CUDA graph); both arms accumulate the same frames, so their images
    are compared bit for bit afterwards."""
    import torch

    from pulse_b200 import scenes
    from pulse_b200.tracer import BatchItem, Target, render_batch, render_forward
    descs = scenes.batch_scenes()
    built = [build_scene(ctx, d)[0] for d in descs]
    plain_t = [Target(ctx, d.width, d.height) for d in descs]
    batch_t = [Target(ctx, d.width, d.height) for d in descs]
    paths = sum(d.width * d.height for d in descs)
    base = dict(PARAMS, kernel=2, wf_segments=args.wf_segments, trace_blocks=args.trace_blocks)

    def plain_frame(acc, params):
        for d, sc, tg in zip(descs, built, plain_t):
            render_forward(sc, d.view, tg, acc, **dict(params, max_depth=d.params["max_depth"], seed=d.params["seed"]))

    def batch_frame(acc, params):
        items = [BatchItem(sc, d.view, tg, acc, d.params["max_depth"], d.params["seed"])
                 for d, sc, tg in zip(descs, built, batch_t)]
        render_batch(ctx, items, **params)

    tuned = {}
    if args.autotune:
        from pulse_b200 import autotune
        tris = sum(d.triangle_count for d in descs)

        def timed(frame):
            def call(params):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                frame(0, params)
                e1.record(stream)
                e1.synchronize()
                return e0.elapsed_time(e1)
            return call
        with torch.cuda.stream(stream):
            for name, frame in (("plain", plain_frame), ("batched", batch_frame)):
                key = autotune.signature(name, paths, tris, len(descs), base)
                best = autotune.tune(ctx, timed(frame), base, key, path=args.autotune_cache, force=True)
                tuned[name] = {k: best[k] for k in autotune.DEFAULT_SPACE}
    steps = max(1, min(args.steps, args.batch_steps))
    out = {"workload": BATCH_WORKLOAD, "scenes": len(descs), "paths_per_frame": paths,
           "triangles": sum(d.triangle_count for d in descs), "steps": steps, "warmup": args.warmup,
           "l2": "inputs larger than L2 (path state of the frame alone is 156 B/path)"}
    with torch.cuda.stream(stream):
        for name, frame in (("plain", plain_frame), ("batched", batch_frame)):
            params = dict(base, **tuned.get(name, {}))
            for i in range(args.warmup):
                frame(i, params)
            stream.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            l0 = ctx.stats()["kernel_launches"]
            e0.record(stream)
            for i in range(steps):
                frame(args.warmup + i, params)
            e1.record(stream)
            stream.synchronize()
            ms = e0.elapsed_time(e1)
            out[name] = {"value": paths * steps / (ms / 1e3) / 1e6, "unit": "Mpaths/s", "ms_per_step": ms / steps,
                         "gpu_launches": ctx.stats()["kernel_launches"] - l0,
                         "params": {k: params.get(k, 0) for k in ("wf_segments", "trace_blocks", "stack_depth",
                                                                    "step_policy", "block_size", "ray_sort")},
                         "autotuned": name in tuned}
    out["ratio_batched_over_plain"] = out["batched"]["value"] / out["plain"]["value"]
    imgs = [b.download() for b in batch_t]
    same = all(np.array_equal(a.download().view(np.uint32), b.view(np.uint32)) for a, b in zip(plain_t, imgs))
    out["images_bit_identical"] = bool(same)
    out["equal_rmse"] = "yes: identical images" if same else "NO: images differ"
    out["traversal_guards"] = {k: ctx.stats()[k] for k in ("iter_cap_hits", "stack_overflows")}
    # The same batch with every path traced and shaded by one persistent
    # kernel from its primary ray (wf_segments = tail only): one traversal
    # launch per frame instead of three wavefront segments and the tail.
    one_t = [Target(ctx, d.width, d.height) for d in descs]
    one_params = dict(base, **tuned.get("batched", {}))
    one_params["wf_segments"] = TAIL_ONLY

    def one_frame(acc):
        items = [BatchItem(sc, d.view, tg, acc, d.params["max_depth"], d.params["seed"])
                 for d, sc, tg in zip(descs, built, one_t)]
        render_batch(ctx, items, **one_params)
    with torch.cuda.stream(stream):
        for i in range(args.warmup):
            one_frame(i)
        stream.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = ctx.stats()["kernel_launches"]
        e0.record(stream)
        for i in range(steps):
            one_frame(args.warmup + i)
        e1.record(stream)
        stream.synchronize()
        ms = e0.elapsed_time(e1)
    same1 = all(np.array_equal(a.download().view(np.uint32), b.download().view(np.uint32))
                for a, b in zip(plain_t, one_t))
    out["batched_one_persistent_launch"] = {
        "value": paths * steps / (ms / 1e3) / 1e6, "unit": "Mpaths/s", "ms_per_step": ms / steps,
        "gpu_launches_per_frame": (ctx.stats()["kernel_launches"] - l0) / steps,
        "images_bit_identical": bool(same1),
        "note": "one persistent kernel traces and shades every path from its primary ray (wf_segments tail only); "
                "the default frame runs three wavefront segments before that kernel"}
    for x in one_t:
        x.close()
    # One scene of the batch (the one with the fewest paths x triangles)
    # rendered by the oracle with its own CPU-built trees, the reference's
    # stack of 32, over the same samples: its batched image must match.
    frames = args.warmup + steps
    k = min(range(len(descs)), key=lambda i: descs[i].width * descs[i].height * descs[i].triangle_count)
    d = descs[k]
    import oracle
    sb = oracle.assemble_desc(d)
    ref = np.zeros((d.height, d.width, 4), np.float32)
    op = {kk: v for kk, v in dict(PARAMS, max_depth=d.params["max_depth"], seed=d.params["seed"]).items()
          if kk in ORACLE_KEYS}
    for a in range(frames):
        oracle.render(sb, d.view, d.width, d.height, a, image=ref, stack_depth=32, **op)
    differ = int(np.any(imgs[k].view(np.uint32) != ref.view(np.uint32), axis=2).sum())
    out["oracle_check"] = {"scene": k, "width": d.width, "height": d.height, "triangles": d.triangle_count,
                           "max_depth": d.params["max_depth"], "samples_per_texel": frames,
                           "oracle_stack_depth": 32, "texels_differing": differ, "bit_exact": differ == 0}
    for x in plain_t + batch_t + built:
        x.close()
    return out


ADJOINT_WORKLOAD = ("differentiable Cornell box: 36 triangles, 8 material groups (RGB albedo, GGX roughness, "
                    "emission scale), 512x512, 64 spp, 6 bounces, NEE+MIS (nee_mode 2), Russian roulette off; "
                    "MSE against a target rendered from hidden parameters U(0.1, 0.9) (seed 1)")


def adjoint_leg(ctx, stream, args):
    """Adjoint/forward time ratio of the differentiable workload, its gradient
    against central differences (eps 1e-3, all 40 parameters) and against the
    FP64 CPU adjoint on a subsample of texels."""
    import torch

    import oracle
    from pulse_b200 import diff, scenes
    from pulse_b200.tracer import Target, render_backward, render_forward
    W = H = args.adjoint_res
    spp = 64
    desc = scenes.cornell(W, H)
    sc, ids, _ = build_scene(ctx, desc)
    tg = Target(ctx, W, H)
    mats = desc.materials
    base_em = diff.base_emission(mats)
    theta = diff.GroupParams.of_materials(mats)
    rng = np.random.default_rng(1)
    hidden = diff.GroupParams(rng.uniform(0.1, 0.9, (8, 3)).astype(np.float32),
                              rng.uniform(0.1, 0.9, 8).astype(np.float32),
                              rng.uniform(0.1, 0.9, 8).astype(np.float32))
    render = dict(max_depth=6, nee_mode=2, light_pick=1, quirks=0, spp=spp, no_roulette=1)
    sc.set_materials(diff.apply(mats, base_em, hidden))
    ref = diff.render_image(sc, desc.view, tg, 1, **render)
    sc.set_materials(diff.apply(mats, base_em, theta))
    out = {"workload": ADJOINT_WORKLOAD, "paths": W * H * spp}
    with torch.cuda.stream(stream):
        def fwd():
            render_forward(sc, desc.view, tg, 0, **render)
        for _ in range(args.warmup):
            fwd()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(5)]
        for a, b in ev:
            a.record(stream)
            fwd()
            b.record(stream)
        stream.synchronize()
        f_ms = statistics.median(a.elapsed_time(b) for a, b in ev)
        img = tg.download()
        dl = diff.dmse(img, ref)
        for _ in range(2):
            render_backward(sc, desc.view, W, H, spp, dl, **render)
        b_ms = []
        e2e = []
        for _ in range(5):
            t0 = time.perf_counter()
            g = render_backward(sc, desc.view, W, H, spp, dl, **render)
            e2e.append((time.perf_counter() - t0) * 1e3)
            b_ms.append(ctx.stats()["last_render_ms"])
        b_ms = statistics.median(b_ms)
    out.update({"forward_ms": f_ms, "backward_ms": b_ms, "adjoint_over_forward": b_ms / f_ms,
                "backward_e2e_ms": statistics.median(e2e),
                "forward_mpaths_s": W * H * spp / f_ms / 1e3, "loss": diff.mse(img, ref)})
    grad = diff.group_grad(g, base_em).flat()
    # central differences of the same seeded estimator
    eps = 1e-3
    x0 = theta.flat()
    fd = np.zeros_like(x0)
    t0 = time.perf_counter()
    for k in range(x0.size):
        vals = []
        for sgn in (1, -1):
            x = x0.copy()
            x[k] += sgn * eps
            sc.set_materials(diff.apply(mats, base_em, diff.GroupParams.from_flat(x, 8)))
            vals.append(diff.mse(diff.render_image(sc, desc.view, tg, 1, **render), ref))
        fd[k] = (vals[0] - vals[1]) / (2 * eps)
    sc.set_materials(diff.apply(mats, base_em, theta))

    def rel(a, b, idx):
        return float(np.linalg.norm(a[idx] - b[idx]) / max(np.linalg.norm(b[idx]), 1e-30))

    def blocks(a, b):
        return {"rel_l2_all": rel(a, b, np.r_[0:40]), "rel_l2_albedo": rel(a, b, np.r_[0:24]),
                "rel_l2_roughness": rel(a, b, np.r_[24:32]), "rel_l2_emission": rel(a, b, np.r_[32:40])}
    out["fd_seeded"] = dict(blocks(grad, fd), eps=eps, seconds=time.perf_counter() - t0, note=(
        "central differences of the seeded MSE (one seed): sampling moves with the parameters; albedo and emission "
        "do not move it, roughness moves the GGX half vectors, so its differences hold visibility jumps and the "
        "variance of another estimator (see fd_seeded_over_seeds)"))
    # FP64 CPU adjoint and detached central differences on 2048 random texels
    # (dloss/dimage zero elsewhere)
    pick = np.random.default_rng(2).choice(W * H, 2048, replace=False).astype(np.uint32)
    dl_sub = np.zeros_like(dl)
    dl_sub.reshape(-1, 4)[pick] = dl.reshape(-1, 4)[pick]
    g_gpu = render_backward(sc, desc.view, W, H, spp, dl_sub, **render)
    t0 = time.perf_counter()
    sb = oracle.assemble(desc.meshes, diff.apply(mats, base_em, theta), desc.instances, desc.params["bins"],
                         desc.params["max_leaf"])
    g_cpu = oracle.backward(sb, desc.view, W, H, spp, dl_sub, **render)[:, :7]
    out["fp64_cpu_adjoint"] = {"texels": int(pick.size), "samples": spp,
                               "max_abs_err_over_max": float(np.abs(g_gpu - g_cpu).max() / np.abs(g_cpu).max()),
                               "seconds": time.perf_counter() - t0}
    t0 = time.perf_counter()

    def rows_at(x):
        return np.stack([m.to_words() for m in diff.apply(mats, base_em, diff.GroupParams.from_flat(x, 8))])
    fd_det = oracle.detached_fd(sb, desc.view, W, H, spp, dl_sub, rows_at, theta.flat(), eps=eps, pixels=pick,
                                **render)
    out["fd_detached"] = dict(blocks(diff.group_grad(g_gpu, base_em).flat(), fd_det), eps=eps, texels=int(pick.size),
                              samples=spp, seconds=time.perf_counter() - t0, note=(
        "the GPU adjoint against central differences of the estimator it differentiates: the same seeded paths "
        "with sampling detached, weighted by the BSDF values and emissions at theta +/- eps (the CPU oracle "
        "evaluates eval_g itself, not its derivatives), every parameter"))
    out["fd_seeded_over_seeds"] = seeded_fd_over_seeds(ctx, stream)
    out["traversal_guards"] = {k: ctx.stats()[k] for k in ("iter_cap_hits", "stack_overflows")}
    tg.close()
    sc.close()
    return out


def seeded_fd_over_seeds(ctx, stream, W=64, H=48, spp=32, seeds=32, eps=1e-3) -> dict:
    """Roughness: the detached adjoint and the seeded central differences
    (sampling moving with roughness) estimate the same derivative of the
    expected image; for a fixed linear functional sum(w . I) of the Cornell
    box (roughness 0.6, 32 spp) both are averaged over independent seeds and
    their mean difference per parameter is reported in standard errors."""
    import torch

    from pulse_b200 import diff, scenes
    from pulse_b200.tracer import Target, render_backward
    desc = scenes.cornell(W, H)
    sc, ids, _ = build_scene(ctx, desc)
    tg = Target(ctx, W, H)
    mats = desc.materials
    base_em = diff.base_emission(mats)
    theta = diff.GroupParams.of_materials(mats)
    theta.roughness[:] = 0.6
    w = np.random.default_rng(9).normal(size=(H, W, 4)).astype(np.float32) / (W * H)
    wv = w[..., :3].astype(np.float64)
    render = dict(max_depth=6, nee_mode=2, light_pick=1, quirks=0, spp=spp, no_roulette=1)
    x0 = theta.flat()
    g = np.zeros((seeds, 8))
    f = np.zeros((seeds, 8))
    t0 = time.perf_counter()
    with torch.cuda.stream(stream):
        for s in range(seeds):
            sc.set_materials(diff.apply(mats, base_em, theta))
            gm = render_backward(sc, desc.view, W, H, spp, w, **dict(render, seed=s))
            g[s] = diff.group_grad(gm, base_em).flat()[24:32]
            for j in range(8):
                vals = []
                for sgn in (1, -1):
                    x = x0.copy()
                    x[24 + j] += sgn * eps
                    sc.set_materials(diff.apply(mats, base_em, diff.GroupParams.from_flat(x, 8)))
                    img = diff.render_image(sc, desc.view, tg, 1, **dict(render, seed=s))
                    vals.append(float(np.sum(wv * img[..., :3])))
                step = float(np.float32(x0[24 + j] + eps)) - float(np.float32(x0[24 + j] - eps))
                f[s, j] = (vals[0] - vals[1]) / step
    tg.close()
    sc.close()
    d = g - f
    z = d.mean(axis=0) / (d.std(axis=0, ddof=1) / math.sqrt(seeds))
    gm_, fm_ = g.mean(axis=0), f.mean(axis=0)
    return {"workload": f"Cornell {W}x{H}, {spp} spp, roughness 0.6, random linear functional, {seeds} seeds",
            "eps": eps, "mean_difference_in_standard_errors": [round(float(v), 3) for v in z],
            "max_abs_z": float(np.abs(z).max()),
            "rel_l2_roughness_of_means": float(np.linalg.norm(gm_ - fm_) / np.linalg.norm(fm_)),
            "rel_l2_roughness_single_seed_median": float(np.median(
                np.linalg.norm(g - f, axis=1) / np.linalg.norm(f, axis=1))),
            "seconds": time.perf_counter() - t0}


GI_WORKLOAD = ("realtime GI pass (src/pulse/gi.wgsl constants: 2 chained samples, 5 diffuse bounces, NEE with "
               "uniform light pick) on the 1080p sphere scene, from the primary-hit G-buffer at 1920x1080")


def gi_leg(ctx, stream, sc, desc, args, sb=None):
    """The realtime GI mode on the benchmark scene: the primary-hit G-buffer
    and the GI frame (device-resident G-buffer, L2 flushed between frames),
    and, given the oracle's scene buffers sb, the CPU restatement on a row
    sample of the same frame."""
    import torch

    import oracle
    from pulse_b200.tracer import Target, gbuffer_primary, render_gi
    W, H = desc.width, desc.height
    tg = Target(ctx, W, H)
    gb = torch.empty(W * H * 16, dtype=torch.float32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    gp = dict(quirks=0)
    steps = 10
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            gbuffer_primary(sc, desc.view, W, H, out=gb, **gp)
            render_gi(sc, gb, tg, gw=W, gh=H, **gp)
        ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(steps)]
        launches0 = ctx.stats()["kernel_launches"]
        for i in range(steps):
            flush.zero_()
            ev[i][0].record(stream)
            gbuffer_primary(sc, desc.view, W, H, out=gb, **gp)
            ev[i][1].record(stream)
            render_gi(sc, gb, tg, gw=W, gh=H, **gp)
            ev[i][2].record(stream)
        stream.synchronize()
        launches = ctx.stats()["kernel_launches"] - launches0
    g_ms = statistics.median(a.elapsed_time(b) for a, b, _ in ev)
    gi_ms = statistics.median(b.elapsed_time(c) for _, b, c in ev)
    paths = W * H * 2
    out = {"workload": GI_WORKLOAD, "gbuffer_ms": g_ms, "gi_ms": gi_ms, "gi_mpaths_s": paths / gi_ms / 1e3,
           "frame_ms": g_ms + gi_ms, "gpu_launches_per_frame": launches / steps}
    if sb is not None:
        host_gb = gb.cpu().numpy().reshape(H, W, 16)
        rows = np.arange(0, H, 16)
        pix = (rows[:, None] * W + np.arange(W)[None, :]).reshape(-1).astype(np.uint32)
        img = tg.download()
        t0 = time.perf_counter()
        ref, _ = oracle.render_gi(sb, host_gb, W, H, pixels=pix, spp=2, max_depth=5, quirks=0)
        cpu_s = time.perf_counter() - t0
        same = bool(np.array_equal(img.reshape(-1, 4)[pix].view(np.uint32), ref.reshape(-1, 4)[pix].view(np.uint32)))
        out["cpu_baseline"] = {"value": pix.size * 2 / cpu_s / 1e6, "unit": "Mpaths/s",
                               "cores": os.cpu_count() or 1, "kind": "port",
                               "sample": f"{pix.size} texels (every 16th row), 2 samples each",
                               "image_bit_exact_on_sample": same}
    tg.close()
    return out


SMALL_WORKLOAD = ("small Cornell box: 36 triangles (5 wall quads, 2 boxes rotated +/-18 degrees, ceiling light of "
                  "radiance (17,12,4)), diffuse albedos white/red/green, GGX roughness 1; 256x256, 64 frames x 1 spp "
                  "accumulated, 4 bounces, NEE with power CDF (corrected estimator), seed 0; BVH 16 bins, leaf 4")


def small_leg(ctx, stream, args, cpu: bool = True):
    """The small configuration: one accumulation of 64 frames of the Cornell
    box at 256^2 (4 bounces), Mpaths/s over the 64 frames (CUDA events), the
    image against the FP32 oracle bit for bit and against an FP64 ground
    truth of 4096 samples per texel (1/16 of the texels)."""
    import torch

    from pulse_b200 import scenes
    from pulse_b200.tracer import Target, render_forward
    desc = scenes.cornell(256, 256)
    W, H, frames = desc.width, desc.height, 64
    params = dict(PARAMS, max_depth=4, kernel=2)
    sc, ids, build_ms = build_scene(ctx, desc)
    tg = Target(ctx, W, H)
    out = {"workload": SMALL_WORKLOAD, "frames": frames, "paths": W * H * frames,
           "gpu_blas_build_ms": build_ms}
    with torch.cuda.stream(stream):
        for _ in range(max(1, args.warmup)):
            for a in range(frames):
                render_forward(sc, desc.view, tg, a, **params)
        stream.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = ctx.stats()["kernel_launches"]
        e0.record(stream)
        for a in range(frames):
            render_forward(sc, desc.view, tg, a, **params)
        e1.record(stream)
        stream.synchronize()
    ms = e0.elapsed_time(e1)
    out.update({"ms_for_64_frames": ms, "value": W * H * frames / (ms / 1e3) / 1e6, "unit": "Mpaths/s",
                "gpu_launches": ctx.stats()["kernel_launches"] - l0,
                "traversal_guards": {k: ctx.stats()[k] for k in ("iter_cap_hits", "stack_overflows")},
                "l2": "not flushed (the 36-triangle scene is L2-resident by design)"})
    img = tg.download()
    # The same 64 frames with frame pipelining (pulse_ctx_set_pipeline depth
    # 2): frame k+1 starts while frame k drains.  ctx.stream_ptr()
    # (pulse_ctx_get_stream) orders the stream after the frames in flight.
    with torch.cuda.stream(stream):
        ctx.set_pipeline(2)
        for a in range(frames):
            render_forward(sc, desc.view, tg, a, **params)
        ctx.stream_ptr()
        stream.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for a in range(frames):
            render_forward(sc, desc.view, tg, a, **params)
        ctx.stream_ptr()
        p1.record(stream)
        stream.synchronize()
        ctx.set_pipeline(1)
    pms = p0.elapsed_time(p1)
    img_p = tg.download()
    out["pipelined"] = {"ms_for_64_frames": pms, "value": W * H * frames / (pms / 1e3) / 1e6, "unit": "Mpaths/s",
                        "image_bit_identical": bool(np.array_equal(img_p.view(np.uint32), img.view(np.uint32))),
                        "note": "the same 64 frames at pipeline depth 2 (pulse_ctx_set_pipeline)"}
    tg.close()
    sc.close()
    if cpu:
        import oracle
        sb = oracle.assemble_desc(desc)
        ref = np.zeros((H, W, 4), np.float32)
        op = {k: v for k, v in params.items() if k in ORACLE_KEYS}
        t0 = time.perf_counter()
        for a in range(frames):
            oracle.render(sb, desc.view, W, H, a, image=ref, **op)
        cpu_s = time.perf_counter() - t0
        differ = int(np.any(img.view(np.uint32) != ref.view(np.uint32), axis=2).sum())
        out["parity_vs_fp32_oracle"] = {"texels": W * H, "texels_differing": differ, "bit_exact": differ == 0,
                                        "frames": frames}
        out["cpu_baseline"] = {"value": W * H * frames / cpu_s / 1e6, "unit": "Mpaths/s",
                               "cores": os.cpu_count() or 1, "kind": "port", "sample": "the whole 64-frame image"}
        out["converged_vs_fp64"] = converged_vs_fp64(sb, desc, img, frames, params, seed=0, gt_spp=4096)
    return out


LARGE_WORKLOAD = ("large: fBm terrain of 4096^2 vertices (33,538,050 triangles) + 4096 instances of a 20,480-triangle "
                  "rock + 10,000 emissive triangles (radiance log-uniform 0.5-50), GGX roughness U(0.02, 1); "
                  "3840x2160, 1 spp, 16 bounces, NEE with power CDF; BLAS on the GPU with 32 bins / leaf 4")


def large_leg(ctx, stream, args):
    """The large configuration: GPU BLAS build of the 33.5M-triangle terrain
    (timed), Mpaths/s of the 4K frame with its traversal guards, frame 0
    against the FP32 oracle bit for bit on a row sample (the oracle traces the
    scene buffers the GPU prepared: its trees equal the CPU builder's, as the
    next check shows on a 1024^2 terrain of the same generator, or with
    --large-check on the full terrain)."""
    import torch

    from pulse_b200 import scenes
    from pulse_b200.layout import triangle_soup
    from pulse_b200.tracer import Target, render_forward
    t0 = time.perf_counter()
    desc = scenes.terrain_scene(n=args.large_n)
    gen_s = time.perf_counter() - t0
    sc, ids, build_ms = build_scene(ctx, desc)
    out = {"workload": LARGE_WORKLOAD, "terrain_vertices_per_side": args.large_n,
           "triangles_in_scene": desc.triangle_count, "terrain_triangles": desc.meshes[0].triangle_count,
           "generate_s": gen_s, "gpu_blas_build_ms": {"terrain": build_ms[0], "rock": build_ms[1]}}
    W, H = desc.width, desc.height
    tg = Target(ctx, W, H)
    params = dict(PARAMS, max_depth=16, kernel=2)
    g0 = {k: ctx.stats()[k] for k in ("iter_cap_hits", "stack_overflows")}
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    with torch.cuda.stream(stream):
        for i in range(2):
            render_forward(sc, desc.view, tg, i, **params)
        frames = 3
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(frames)]
        for i in range(frames):
            flush.zero_()
            ev[i][0].record(stream)
            render_forward(sc, desc.view, tg, 2 + i, **params)
            ev[i][1].record(stream)
        stream.synchronize()
        render_forward(sc, desc.view, tg, 0, **params)  # frame 0 alone, for the oracle comparison
    del flush
    ms = statistics.mean(a.elapsed_time(b) for a, b in ev)
    out.update({"ms_per_frame": ms, "value": W * H / (ms / 1e3) / 1e6, "unit": "Mpaths/s",
                "l2": "flushed between timed frames",
                "traversal_guards": {k: ctx.stats()[k] - g0[k] for k in ("iter_cap_hits", "stack_overflows")}})
    img0 = tg.download()
    tg.close()
    if not args.no_cpu_baseline:
        import oracle
        sb = sc.download()
        rows = np.arange(0, H, 72)
        pix = (rows[:, None] * W + np.arange(W)[None, :]).astype(np.uint32).ravel()
        ref = np.zeros((H, W, 4), np.float32)
        t0 = time.perf_counter()
        oracle.render(sb, desc.view, W, H, 0, image=ref, pixels=pix,
                      **{k: v for k, v in params.items() if k in ORACLE_KEYS})
        cpu_s = time.perf_counter() - t0
        del sb
        differ = int(np.any(img0.reshape(-1, 4)[pix].view(np.uint32) != ref.reshape(-1, 4)[pix].view(np.uint32),
                            axis=1).sum())
        out["parity_vs_fp32_oracle"] = {"texels": int(pix.size), "sample": "every 72nd row of frame 0",
                                        "texels_differing": differ, "bit_exact": differ == 0,
                                        "nonfinite_texels": int((~np.isfinite(img0)).any(axis=2).sum()),
                                        "oracle_scene": "the scene buffers the GPU prepared, downloaded"}
        out["cpu_baseline"] = {"value": pix.size / cpu_s / 1e6, "unit": "Mpaths/s", "cores": os.cpu_count() or 1,
                               "kind": "port", "sample": f"{pix.size} paths (every 72nd row of frame 0)"}
    sc.close()
    import oracle
    if args.large_check:
        prims, _ = triangle_soup(desc.meshes[0])
        which = f"the full terrain ({args.large_n}^2 vertices)"
    else:
        prims, _ = triangle_soup(scenes.fbm_grid(1024, 400.0, 12.0, 0))
        which = "a 1024^2-vertex terrain of the same generator (2,093,058 triangles)"
    t0 = time.perf_counter()
    rn, ri = oracle.build_blas(prims, 32, 4)
    cpu_ms = (time.perf_counter() - t0) * 1e3
    gn, gi = ctx.build_blas(prims, 32, 4)
    gpu_ms = ctx.stats()["last_build_ms"]
    out["blas_vs_cpu_builder"] = {"mesh": which, "triangles": int(prims.shape[0]), "bins": 32, "max_leaf": 4,
                                  "bit_exact": bool(np.array_equal(rn, gn) and np.array_equal(ri, gi)),
                                  "cpu_ms_1thread": cpu_ms, "gpu_ms": gpu_ms, "speedup": cpu_ms / gpu_ms}
    return out


def headline_config(args, desc, world: int) -> dict:
    """The config dict of the headline line, identical in both arms."""
    return {"workload": WORKLOAD, "width": desc.width, "height": desc.height, "spp": PARAMS["spp"],
            "max_depth": PARAMS["max_depth"], "nee_mode": PARAMS["nee_mode"], "light_pick": "power CDF",
            "quirks": PARAMS["quirks"], "stack_depth": 32,
            "parallelism": f"{world} GPU(s), disjoint sample streams",
            "l2": "flushed between timed frames (256 MiB write outside the events)",
            "triangles": desc.triangle_count,
            "kernel": {1: "megakernel", 2: "wavefront"}.get(args.kernel, "auto"),
            "launch": {"wf_segments": args.wf_segments or 3, "trace_blocks": args.trace_blocks or 8}}


# The reference's own path_trace (src/path_tracer/path_tracer.wgsl:58-124):
# no NEE, its FP32 quirks, 5 bounces.
REFERENCE_MODE = dict(nee_mode=0, light_pick=0, quirks=1, max_depth=5)


def run_reference(args, rank, world):
    from pulse_b200 import scenes
    if rank != 0:
        return
    desc = scenes.spheres_1080p(level=args.level, width=args.width, height=args.height)
    cores = os.cpu_count() or 1
    r = cpu_legs(desc, args, cores, steps=args.warmup + args.steps)
    rates = r["rates"][args.warmup:]
    times = r["times"][args.warmup:]
    v = statistics.mean(rates)
    rm = cpu_legs(desc, args, cores, steps=1, params=REFERENCE_MODE)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "Mpaths/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": headline_config(args, desc, world),
        "cpu_baseline": {"value": v, "unit": "Mpaths/s", "cores": cores, "kind": "port",
                         "sample": f"{r['paths']} paths per step (every {args.cpu_row_stride}th row of the frame)",
                         "bvh_build_ms_1thread": r["build_ms"]},
        "e2e": {"value": v, "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_estimator_cpu": {
            "value": rm["rates"][0], "unit": "Mpaths/s", "cores": cores,
            "params": REFERENCE_MODE,
            "note": "context only: the reference's own path_trace (no NEE, its FP32 quirks, 5 bounces) on the "
                    "same scene, same C++ port"},
        "note": "C++ CPU port of this library's estimator (nee_mode 2: NEE with the power CDF and MIS, quirks 0), "
                "OpenMP over all host cores; results bit-identical to the GPU's.  The reference's WGSL tracer "
                "needs a graphics API (wgpu on Vulkan/GL) and a Rust toolchain: unavailable on this box",
    }
    print(json.dumps(line), flush=True)


def max_over_ranks(ms: float, world: int, device: str) -> float:
    """The slowest rank's time (every rank calls it, in the same order)."""
    if world <= 1:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def main():
    args = parse()
    rank, local_rank, world = dist_env()
    if world > 1:
        import datetime

        import torch.distributed as dist
        if args.impl == "ours":
            import torch
            torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl" if args.impl == "ours" else "gloo",
                                timeout=datetime.timedelta(seconds=300))
    if args.impl == "reference":
        run_reference(args, rank, world)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    import torch

    from pulse_b200 import build as pbuild
    pbuild.build()
    from pulse_b200 import scenes
    from pulse_b200.tracer import Context, Target, render_count, render_forward

    torch.cuda.set_device(local_rank)
    desc = scenes.spheres_1080p(level=args.level, width=args.width, height=args.height)
    W, H = desc.width, desc.height
    params = dict(PARAMS, seed=rank, min_blocks=args.min_blocks, kernel=args.kernel, wf_segments=args.wf_segments,
                  trace_blocks=args.trace_blocks)
    ctx = Context(local_rank)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    sc, ids, build_ms = build_scene(ctx, desc)
    tg = Target(ctx, W, H)
    paths = W * H * params["spp"]

    # Algorithmic work of one frame, counted by the device replaying the reference algorithm.
    work = render_count(sc, desc.view, tg, 0, **params)
    b_path = work["bytes"] / work["paths"]

    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    with torch.cuda.stream(stream):
        for i in range(args.warmup):
            render_forward(sc, desc.view, tg, i, **params)
        stream.synchronize()
        if world > 1:
            torch.distributed.barrier()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        launches0 = ctx.stats()["kernel_launches"]
        torch.cuda.synchronize()
        with ClockSampler(local_rank) as clk:
            for i in range(args.steps):
                flush.zero_()
                ev[i][0].record(stream)
                render_forward(sc, desc.view, tg, args.warmup + i, **params)
                ev[i][1].record(stream)
            stream.synchronize()
        torch.cuda.synchronize()
        launches = ctx.stats()["kernel_launches"] - launches0
        step_ms = [a.elapsed_time(b) for a, b in ev]
    frame_img = tg.download()  # samples 0 .. warmup + steps - 1
    # frame 0 of this rank's stream alone (accumulation count 0), for the
    # bit-exact comparison with the oracle's frame
    tg0 = Target(ctx, W, H)
    render_forward(sc, desc.view, tg0, 0, **params)
    frame0 = tg0.download()
    tg0.close()
    total_ms = sum(step_ms)
    total_ms = max_over_ranks(total_ms, world, "cuda")
    ms_per_step = total_ms / args.steps
    value = world * paths * args.steps / (total_ms / 1e3) / 1e6

    # End to end through the C ABI: pinned instance upload, render, pinned image read-back.
    pinned_inst, inst_arr = instance_descs(desc, ids)
    host_img = torch.empty((H, W, 4), dtype=torch.float32, pin_memory=True)
    import ctypes as C

    from pulse_b200 import _ffi
    lib = ctx.lib
    bp = _ffi.BvhParams(2, 1)
    from pulse_b200.tracer import make_view, render_params
    view_c = make_view(desc.view)
    params_c = render_params(**params)

    def e2e_step(acc):
        # frame acc's instances from pinned memory, the frame, and its image
        # read back to pinned memory while the next frame traces
        ctx.check(lib.pulse_instances_set(sc.h, inst_arr, len(desc.instances), C.byref(bp)), "instances_set")
        ctx.check(lib.pulse_render_forward(sc.h, C.byref(view_c), tg.h, acc, C.byref(params_c)), "render")
        ctx.check(lib.pulse_target_download_async(tg.h, C.c_void_p(host_img.data_ptr())), "download")

    def e2e_run(depth):
        # depth 2: frame k+1 is queued while frame k still traces
        # (pulse_ctx_set_pipeline), the way a real-time host drives it
        ctx.set_pipeline(depth)
        for i in range(args.warmup):
            e2e_step(i)
        ctx.check(lib.pulse_target_download_wait(tg.h), "download wait")
        if world > 1:
            torch.distributed.barrier()
        launch0 = ctx.stats()["kernel_launches"]
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(args.steps):
            e2e_step(args.warmup + i)
        ctx.check(lib.pulse_target_download_wait(tg.h), "download wait")  # the last frame's image is on the host
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        n = ctx.stats()["kernel_launches"] - launch0
        ctx.set_pipeline(1)
        return ms, n

    serial_ms, _ = e2e_run(1)
    e2e_ms, e2e_launches = e2e_run(2)
    serial_ms = max_over_ranks(serial_ms, world, "cuda")
    ctx.check(lib.pulse_instances_set(sc.h, inst_arr, len(desc.instances), C.byref(bp)), "instances_set")
    scene_update_ms = ctx.stats()["last_upload_ms"]
    e2e_ms = max_over_ranks(e2e_ms, world, "cuda")
    e2e_value = world * paths * args.steps / (e2e_ms / 1e3) / 1e6
    h2d = len(desc.instances) * C.sizeof(_ffi.InstanceDesc) + C.sizeof(_ffi.ViewC) + C.sizeof(_ffi.RenderParams)
    d2h = W * H * 16

    peak, peak_kind = measured_hbm_peak()
    avg_launch_ms = statistics.mean(step_ms)
    bytes_per_launch = b_path * paths
    achieved = bytes_per_launch / (avg_launch_ms / 1e3) / 1e9
    traffic = profile_traffic("wf_frame_spheres_1080p") if (W, H) == (1920, 1080) else None
    line = {
        "metric": METRIC, "value": value, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": headline_config(args, desc, world),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_source": peak_kind,
                     "unit_of_work": "one frame: the wavefront's kernels share the path queues and the "
                                     "persistent tail kernel finishes what the segment kernels leave, so "
                                     "algorithmic bytes (counted by the device) are defined per frame",
                     "traffic_source": "profiles/wf_frame_spheres_1080p.md (ncu DRAM bytes of a 540p frame, "
                                       "scaled by paths)",
                     "bytes_per_path": b_path, "bytes_per_launch": bytes_per_launch,
                     "work_per_frame": work},
        "e2e": {"value": e2e_value, "unit": "Mpaths/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_ms / args.steps, "gpu_launches": e2e_launches,
                "pipeline": "depth 2 (pulse_ctx_set_pipeline): each frame queued while the previous one traces",
                "serial": {"value": world * paths * args.steps / (serial_ms / 1e3) / 1e6,
                           "ms_per_step": serial_ms / args.steps,
                           "note": "the same loop at pipeline depth 1 (each frame queued behind the previous)"},
                "scene_update_ms": scene_update_ms,
                "scene_update": "pulse_instances_set of the 72 instances: records, bounds, light CDFs, TLAS "
                                "(device events around the call, last step)"},
        "gpu_launches": launches,
        "traversal_guards": {k: ctx.stats()[k] for k in ("iter_cap_hits", "stack_overflows")},
        "bvh_build_ms": {"sphere_blas_327680_tris_gpu": build_ms[0]},
        "clocks": clk.summary(),
    }
    if not args.no_batch:
        line["batched"] = batch_leg(ctx, stream, args)
    if not args.no_adjoint:
        line["adjoint"] = adjoint_leg(ctx, stream, args)
    if not args.no_small:
        line["small"] = small_leg(ctx, stream, args, cpu=rank == 0 and world == 1 and not args.no_cpu_baseline)
    if not args.no_large:
        line["large"] = large_leg(ctx, stream, args)
    r = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        r = cpu_legs(desc, args, cores, steps=1)
        line["cpu_baseline"] = {"value": r["rates"][0], "unit": "Mpaths/s", "cores": cores, "kind": "port",
                                "sample": f"{r['paths']} paths (every {args.cpu_row_stride}th row of the frame)",
                                "bvh_build_ms_1thread": r["build_ms"]}
        # the scene's first build includes its scratch allocations; on a
        # scratch scene, uploads after the first time the builder warm
        from pulse_b200.tracer import Scene
        warm = []
        p0 = desc.params
        tmp_scene = Scene(ctx)
        for i in range(4):
            mid = tmp_scene.upload_mesh(desc.meshes[0], p0.get("bins", 20), p0.get("max_leaf", 8))
            if i:
                warm.append(ctx.stats()["last_build_ms"])
            tmp_scene.remove_mesh(mid)
        tmp_scene.close()
        line["bvh_build"] = build_roofline(r["n_tris"], r["blas_nodes"], statistics.median(warm), r["build_ms"], peak)
        line["bvh_build"]["gpu_ms_first_build"] = build_ms[0]
        line["bvh_build"]["gpu_ms_warm"] = warm
        pix = r["pixels"]
        differ = int(np.any(frame0.reshape(-1, 4)[pix].view(np.uint32) !=
                            r["image"].reshape(-1, 4)[pix].view(np.uint32), axis=1).sum())
        line["parity_vs_fp32_oracle"] = {
            "frame": "accumulation count 0, seed 0, the benchmark's params", "texels": int(pix.size),
            "texels_differing": differ, "bit_exact": differ == 0,
            "nonfinite_texels": int((~np.isfinite(frame0)).any(axis=2).sum()),
            "compared": "RGBA bit patterns of every texel the CPU baseline rendered"}
        if not args.no_converged:
            line["converged_vs_fp64"] = converged_vs_fp64(r["sb"], desc, frame_img, args.warmup + args.steps,
                                                          PARAMS, seed=rank, gt_spp=args.gt_spp)
    if not args.no_gi:
        line["gi"] = gi_leg(ctx, stream, sc, desc, args, sb=r["sb"] if r else None)
    if rank == 0:
        print(json.dumps(line), flush=True)
    tg.close()
    sc.close()
    ctx.close()
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
