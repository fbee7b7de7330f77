"""Multi-GPU sharding of the rendering path (one process per GPU, torch.distributed).

The path needs no exchange inside a frame: pixel samples are independent.  A frame's
samples are split across ranks as independent spp shards (each rank renders all pixels
with its own Philox seed), a batch of scenes is split by scene, and the only collective
is the final sum of the float films (or, for the adjoint, of the gradient buffers).
"""
from __future__ import annotations

# Seeds of different ranks must give disjoint Philox streams: the key is the seed, so
# distinct seeds suffice; the stride keeps consecutive frames of one rank distinct too.
RANK_SEED_STRIDE = 1 << 32


def replica_seed(base_seed: int, rank: int) -> int:
    """Philox seed of `rank`'s spp shard of the frame seeded `base_seed`."""
    return (int(base_seed) + int(rank) * RANK_SEED_STRIDE) & 0xFFFFFFFFFFFFFFFF


def spp_shard(spp: int, rank: int, world: int) -> int:
    """Samples per pixel rendered by `rank` when a frame of `spp` is split over `world`
    ranks (the first spp % world ranks take one more)."""
    return spp // world + (1 if rank < spp % world else 0)


def scene_shard(n_scenes: int, rank: int, world: int) -> list:
    """Scene indices rendered by `rank` (round robin: uneven scene sizes spread out)."""
    return list(range(rank, n_scenes, world))


def reduce_sum(tensor, group=None):
    """Sums a film or gradient buffer over all ranks in place (the one collective)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(tensor, op=dist.ReduceOp.SUM, group=group)
    return tensor
