"""Multi-GPU rendering: one process per GPU renders a contiguous shard of the camera samples
and the float films are summed with one all-reduce.

A render's camera samples are numbered pixel-major (pixel * spp + s, which is also each
sample's Halton index), and every sample's contribution depends only on that number, so the
films of disjoint sample ranges sum to the whole render's film (path and direct-lighting
integrators; up to the order of float additions).  The exchange is one all-reduce of the
film sum and weight (4 floats per pixel) over the process group: NCCL over NVLink between
GPUs, gloo between CPU processes in tests.

The reference renders on one GPU (Integrators/PathTracingIntegrator.cu:318-425); this is the
exchange step its one-process design lacks.
"""
from __future__ import annotations

from typing import Callable


def shard_range(total: int, rank: int, world: int) -> tuple[int, int]:
    """The contiguous sample range [begin, end) of `rank` among `world`: sizes differ by at
    most one, ranks in order."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of world {world}")
    base, extra = divmod(total, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def reduce_films(film_sum, film_weight, group=None):
    """Sums the shards' films in place on every rank with one all-reduce of one buffer."""
    import torch
    import torch.distributed as dist

    flat = torch.cat([film_sum.reshape(-1), film_weight.reshape(-1)])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    n = film_sum.numel()
    film_sum.view(-1).copy_(flat[:n])
    film_weight.view(-1).copy_(flat[n:])
    return film_sum, film_weight


def render_sharded(total_samples: int, render_shard: Callable[[int, int], tuple], group=None):
    """Renders this rank's shard with ``render_shard(begin, end) -> (film_sum, film_weight)``
    (torch tensors on the process group's device) and returns the summed films."""
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    begin, end = shard_range(total_samples, rank, world)
    s, w = render_shard(begin, end)
    return reduce_films(s, w, group)


def render_scene_sharded(scene, group=None, **render_kw):
    """`render_sharded` for a loaded `cavalry_b200.Scene` on this rank's GPU: device films
    of the scene's resolution (or width/height in render_kw), the path or direct integrator."""
    import torch

    info = scene.info()
    W = render_kw.get("width") or info.width
    H = render_kw.get("height") or info.height
    spp = render_kw.get("spp") or info.spp
    total = W * H * spp

    def shard(begin, end):
        s = torch.zeros(H * W * 3, device="cuda")
        w = torch.zeros(H * W, device="cuda")
        scene.render_into(s, w, sample_range=(begin, end), **render_kw)
        return s, w

    return render_sharded(total, shard, group)
