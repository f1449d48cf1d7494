"""Multi-rank path of the batched workload, on CPU with gloo (world size 2).

Independent bodies shard over ranks with no data-path collective: rank r steps bodies
r, r + N, ...  Here two gloo ranks each take their shard, build its solver scene through
the drop-in C ABI (no GPU: PrepareScene without upload), and check with collectives on
the host that the shards are disjoint and complete and that their dynamic rows and blocks
add up to those of the whole world (bodies never couple).  The max-over-ranks reduction
the benchmark times with is exercised on the same group.
"""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from physik_b200 import meshes


def small_batch(count=6):
    scene = meshes.small_box(2, 2, 2)
    scene.bodies = [meshes.small_box(2 + b % 3, 2 + (b // 2) % 2, 2, seed=20 + b).bodies[0] for b in range(count)]
    return scene


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        from physik_b200.world import SimWorld

        scene = small_batch()
        shard = bench.shard_scene(scene, rank, world)
        w = SimWorld(shard)
        rows = w.prepare(upload=False)
        _, col, _, _ = w.pattern()
        ids = torch.zeros(len(scene.bodies), dtype=torch.int64)
        for b in range(rank, len(scene.bodies), world):
            ids[b] = 1
        dist.all_reduce(ids)
        sizes = torch.tensor([rows, len(col)], dtype=torch.int64)
        dist.all_reduce(sizes)
        slowest = bench.max_over_ranks(dist, float(rank + 1), 0)
        if rank == 0:
            full = SimWorld(scene)
            full_rows = full.prepare(upload=False)
            _, full_col, _, _ = full.pattern()
            out.put((ids.tolist(), sizes.tolist(), [full_rows, len(full_col)], slowest))
    finally:
        dist.destroy_process_group()


def test_two_rank_body_sharding_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    ids, sizes, full, slowest = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert ids == [1] * 6          # every body on exactly one rank
    assert sizes == full           # rows and blocks add up: no coupling across bodies
    assert slowest == 2.0          # max over ranks
