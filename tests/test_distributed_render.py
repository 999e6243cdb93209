"""Multi-GPU render sharding (cavalry_b200.distributed): the sample split and the film
all-reduce, run as two gloo processes on the CPU with the path-tracing oracle rendering
each shard (the sum of the shards' films equals the whole render's)."""
import os
import socket

import numpy as np
import pytest


def test_shard_ranges_cover_the_samples_once():
    from cavalry_b200.distributed import shard_range

    for total in (0, 1, 7, 1000, 1 << 20):
        for world in (1, 2, 3, 8):
            rs = [shard_range(total, r, world) for r in range(world)]
            assert rs[0][0] == 0 and rs[-1][1] == total
            assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
            sizes = [e - b for b, e in rs]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, kw, out_dir):
    import torch
    import torch.distributed as dist

    from cavalry_b200 import scenes
    from cavalry_b200.distributed import render_sharded
    from oracle import pyoracle as po

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        room = scenes.mini_room()
        total = kw["width"] * kw["height"] * kw["spp"]

        def shard(begin, end):
            s, w = po.render_path(room, first=begin, count=end - begin, **kw)
            return torch.from_numpy(s), torch.from_numpy(w)

        s, w = render_sharded(total, shard)
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), s=s.numpy(), w=w.numpy())
    finally:
        dist.destroy_process_group()


def test_two_process_sharded_render_sums_to_the_whole(tmp_path):
    import torch.multiprocessing as mp

    from cavalry_b200 import scenes
    from oracle import pyoracle as po

    kw = dict(width=48, height=40, spp=3, max_depth=4)
    mp.start_processes(_worker, args=(2, _free_port(), kw, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    s_full, w_full = po.render_path(scenes.mini_room(), **kw)
    for r in range(2):
        got = np.load(tmp_path / f"r{r}.npz")
        assert np.array_equal(got["w"], w_full)  # every sample splats on exactly one rank
        assert np.allclose(got["s"], s_full, rtol=1e-5, atol=1e-6)
