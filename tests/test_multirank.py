"""The multi-rank logic of bench.py on CPU (gloo, world size 2).

One process per GPU: each rank times its own frames, the reported time is the
slowest rank's (all_reduce MAX), and the reference arm prints one line from
rank 0 only.  Rendezvous on 127.0.0.1.
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out[rank] = bench.max_over_ranks(10.0 + 5.0 * rank, world, "cpu")
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    world = 2
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        assert dict(out) == {0: 15.0, 1: 15.0}


def test_reference_arm_two_ranks_prints_once():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1", "--level", "2",
           "--width", "32", "--height", "16"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0


def _scene_rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import numpy as np
    import oracle
    from pulse_b200 import multigpu, scenes
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        d = scenes.cornell(16, 12)
        local = oracle.assemble(d.meshes, d.materials, d.instances, 16, 4)
        got = multigpu.broadcast_scene(local if rank == 0 else None, src=0)
        same = got.instance_count == local.instance_count and got.light_count == local.light_count and all(
            a.shape == b.shape and np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))
            for a, b in zip(got.arrays(), local.arrays()))
        # disjoint sample streams (seed = rank), one all-reduce for the all-ranks mean
        params = dict(max_depth=4, nee_mode=2, light_pick=1, quirks=0)
        img, _ = oracle.render(got, d.view, 16, 12, 0, seed=rank, nthreads=1, **params)
        import torch
        t = torch.from_numpy(img.copy())
        multigpu.combine_images(t)
        imgs = [oracle.render(local, d.view, 16, 12, 0, seed=r, nthreads=1, **params)[0] for r in range(world)]
        want = (imgs[0] + imgs[1]) / np.float32(world)
        out[rank] = (same, bool(np.array_equal(t.numpy().view(np.uint32), want.view(np.uint32))))
    finally:
        dist.destroy_process_group()


def test_scene_broadcast_and_image_mean_gloo():
    """broadcast_scene gives every rank the source rank's 13 buffers bit for
    bit; combine_images gives every rank the mean of the ranks' images."""
    world = 2
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_scene_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        assert dict(out) == {0: (True, True), 1: (True, True)}
