"""GPU test of the batched build (cav_bvh_build_batch): every tree equals the tree built
for its scene alone, bit for bit, and traces the same."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("rounds", [0, 2])
def test_batch_build_equals_single_builds(rounds):
    import torch

    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    ctx = cav.Context(0)
    sizes = [2, 3, 1000, 600000, 4097, 33000, 250000, 17]  # 600k: a tree that runs its rounds alone
    data = [scenes.soup(n, seed=40 + k) for k, n in enumerate(sizes)]
    room = scenes.mini_room()
    data.append((room["positions"], room["indices"]))
    dev = [(torch.from_numpy(p).cuda(), torch.from_numpy(i).cuda()) for p, i in data]
    batch = ctx.build_batch(dev, rounds=rounds)
    rays = torch.from_numpy(scenes.closest_rays(20000, seed=5)).cuda()
    for k, (p, i) in enumerate(dev):
        single = ctx.build(p, i, rounds=rounds)
        a, b = batch[k].export_nodes(), single.export_nodes()
        assert a.tobytes() == b.tobytes(), k
        sa, sb = batch[k].export_stages(), single.export_stages()
        for x, y in zip(sa, sb):
            assert np.array_equal(x, y), k
        pa, ta, _ = batch[k].trace_closest(rays)
        pb, tb, _ = single.trace_closest(rays)
        assert np.array_equal(pa.cpu().numpy(), pb.cpu().numpy())
        single.free()
    ctx.sync_check()


def test_many_small_scenes_with_treelet_rounds():
    """96 scenes of 2-6000 triangles with 3 treelet rounds: the rounds run for all trees in
    one leaf-list and one treelet launch per round, and every tree is still the one its
    scene builds alone."""
    import torch

    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    ctx = cav.Context(0)
    rng = np.random.default_rng(12)
    sizes = [2, 3, 4, 5] + [int(x) for x in np.exp(rng.uniform(np.log(6), np.log(6000), 92))]
    dev = []
    for k, n in enumerate(sizes):
        p, i = scenes.soup(n, seed=300 + k)
        dev.append((torch.from_numpy(p).cuda(), torch.from_numpy(i).cuda()))
    batch = ctx.build_batch(dev, rounds=3)
    for k, (p, i) in enumerate(dev):
        single = ctx.build(p, i, rounds=3)
        assert batch[k].export_nodes().tobytes() == single.export_nodes().tobytes(), (k, sizes[k])
        single.free()
    ctx.sync_check()
