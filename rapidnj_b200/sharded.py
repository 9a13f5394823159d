"""One alignment over several GPUs: one process per GPU, tiles split by rank.

Every pair is independent, so each rank computes a contiguous range of the
alignment's triangle tiles (``rnj_shard_*``) from its own copy of the packed
alignment.  The one exchange is the saturation cap of the post-process
(KimuraDistance.cpp:366-395, JCdistance.cpp:201-230): a saturated pair becomes
twice the maximum over the whole matrix, so the ranks all-reduce one float (MAX)
between computing their tiles and rewriting their saturated pairs.  Each rank
then holds its own tiles (and their mirrors) on its device and can copy them to
host memory; no distance crosses between GPUs.
"""
from __future__ import annotations

from .api import Alignment, Context, Shard, shard_tiles, tile_coords  # noqa: F401


def exchange_max(local: float, group=None, device: int | None = None) -> float:
    """MAX over the ranks of ``group`` of one float (identity without a group).

    NCCL groups reduce a one-element tensor on ``device``; others (gloo) on the CPU.
    """
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return float(local)
    on_gpu = dist.get_backend(group) == "nccl"
    dev = f"cuda:{device if device is not None else torch.cuda.current_device()}" if on_gpu else "cpu"
    t = torch.tensor([local], dtype=torch.float32, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def run_sharded(shard, group=None, device: int | None = None) -> float:
    """Runs one shard through the two steps around the exchange; returns the global
    maximum.  ``shard`` needs ``run() -> local max`` and ``finish(global_max)``."""
    local = shard.run()
    g = exchange_max(local, group, device)
    shard.finish(g)
    return g


def sharded_distance(ctx: Context, aln: Alignment, model="kim", group=None, out=None):
    """This rank's shard of ``aln`` on ``ctx``'s device, finished: (Shard, global max).

    ``out``: optional CUDA float32 tensor (n, >= n) for the shard's tiles."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        rank, world = dist.get_rank(group), dist.get_world_size(group)
    else:
        rank, world = 0, 1
    sh = Shard(ctx, aln, model, rank, world, out)
    return sh, run_sharded(sh, group, ctx.device)
