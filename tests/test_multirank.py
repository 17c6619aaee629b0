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

import numpy as np
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


def test_assign_scenes_balances_and_agrees():
    from pulse_b200 import multigpu
    rng = np.random.default_rng(3)
    costs = rng.lognormal(0.0, 1.5, 32)
    for world in (1, 2, 3, 8):
        parts = multigpu.assign_scenes(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(32))
        loads = [costs[p].sum() if p else 0.0 for p in parts]
        lower = max(costs.sum() / world, costs.max())  # no split beats this
        assert max(loads) <= 4.0 / 3.0 * lower + 1e-9
        assert parts == multigpu.assign_scenes(list(costs), world)  # deterministic
    assert multigpu.assign_scenes([5.0, 1.0], 4) == [[0], [1], [], []]


def _batch_rank(rank, world, port, out):
    """Each rank renders its share of a small mixed batch (oracle renders on
    the CPU stand in for pulse_render_batch) and the images travel to rank 0,
    which checks them against renders of every scene in one process."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch
    import oracle
    from pulse_b200 import multigpu, scenes
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        descs = [scenes.cornell(16, 12), scenes.spheres_1080p(level=2, n_instances=4, width=24, height=16),
                 scenes.cornell(40, 20), scenes.spheres_1080p(level=1, n_instances=3, width=20, height=20, seed=2),
                 scenes.cornell(12, 12)]
        costs = [multigpu.scene_cost(d.width, d.height, 1, d.params["max_depth"], d.triangle_count) for d in descs]
        mine = multigpu.assign_scenes(costs, world)[rank]
        params = dict(nee_mode=2, light_pick=1, quirks=0)
        imgs = {}
        for i in mine:
            d = descs[i]
            sb = oracle.assemble_desc(d)
            imgs[i] = oracle.render(sb, d.view, d.width, d.height, 0, max_depth=d.params["max_depth"], seed=i,
                                    nthreads=1, **params)[0]
        # gather to rank 0: sizes are known from the descriptions on every rank
        ok = True
        for i, d in enumerate(descs):
            owner = next(r for r, p in enumerate(multigpu.assign_scenes(costs, world)) if i in p)
            t = torch.from_numpy(imgs[i].copy()) if owner == rank else torch.zeros((d.height, d.width, 4))
            if owner != 0:
                if rank == owner:
                    dist.send(t, 0)
                elif rank == 0:
                    dist.recv(t, owner)
            if rank == 0:
                sb = oracle.assemble_desc(d)
                want = oracle.render(sb, d.view, d.width, d.height, 0, max_depth=d.params["max_depth"], seed=i,
                                     nthreads=1, **params)[0]
                ok &= bool(np.array_equal(t.numpy().view(np.uint32), want.view(np.uint32)))
        out[rank] = (sorted(mine), ok)
    finally:
        dist.destroy_process_group()


def test_batch_shares_render_every_scene_once_gloo():
    world = 2
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_batch_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        shares = [out[r][0] for r in range(world)]
        assert sorted(i for s in shares for i in s) == list(range(5)) and all(shares)
        assert out[0][1]
