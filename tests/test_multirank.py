"""World-size-2 checks of the multi-GPU sharding logic (rumi_b200.shard) on CPU with the
gloo backend: the CPU oracle stands in for each rank's GPU render, the films and gradient
buffers go through the same collective the GPU path uses."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from rumi_b200 import shard


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        import oraclelib as O
        from rumi_b200 import scenes
        sc = scenes.cornell_pt(16, 16, 4, 3)
        spp = shard.spp_shard(8, rank, world)
        film, nan = O.OracleScene(sc).render_pt(3, spp, seed=shard.replica_seed(77, rank))
        t = torch.from_numpy(film.astype(np.float32).copy())
        shard.reduce_sum(t)
        g = torch.full((7,), float(rank + 1))
        shard.reduce_sum(g)
        mine = shard.scene_shard(10, rank, world)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        if rank == 0:
            np.save(os.path.join(out_dir, "film.npy"), t.numpy())
            np.save(os.path.join(out_dir, "grad.npy"), g.numpy())
            np.save(os.path.join(out_dir, "scenes.npy"), np.array(sorted(sum(gathered, []))))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_shard_helpers():
    assert [shard.spp_shard(10, r, 4) for r in range(4)] == [3, 3, 2, 2]
    assert sum(shard.spp_shard(64, r, 8) for r in range(8)) == 64
    seeds = {shard.replica_seed(5, r) for r in range(8)}
    assert len(seeds) == 8
    parts = [shard.scene_shard(256, r, 8) for r in range(8)]
    assert sorted(sum(parts, [])) == list(range(256))


def test_two_gloo_ranks_sum_their_spp_shards(tmp_path):
    import oraclelib as O
    from rumi_b200 import scenes
    world = 2
    mp.start_processes(_worker, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    film = np.load(tmp_path / "film.npy")
    sc = scenes.cornell_pt(16, 16, 4, 3)
    want = np.zeros_like(film)
    for r in range(world):
        f, _ = O.OracleScene(sc).render_pt(3, shard.spp_shard(8, r, world), seed=shard.replica_seed(77, r))
        want = want + f.astype(np.float32)
    np.testing.assert_array_equal(film, want)
    np.testing.assert_array_equal(np.load(tmp_path / "grad.npy"), np.full(7, 3.0, np.float32))
    assert list(np.load(tmp_path / "scenes.npy")) == list(range(10))
