"""Ray shards (kerrsplat_b200.shard): the partition of the sorted ray order, the all-reduce of
[chi^2, dparams] and the gather of the image over gloo ranks on CPU, and on the GPU the shards of one
screen (run one after another on one GPU) adding up to the whole screen's chi^2, gradient and image.

Tolerances (GPU): FP64 chi^2 within 1e-12 and the gradient within 1e-11 (relative L2) of the whole
screen's, the images within 1e-13 of the largest intensity (only the order of the sums over rays
differs); mixed within 1e-5 (chi^2, image) and 1e-4 (gradient): each ray's FP32 transport may be cut
into different work-unit segments when the screen is smaller."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from kerrsplat_b200.shard import ray_shards


def test_contiguous_shards_cover_the_order_and_balance_the_samples():
    rng = np.random.Generator(np.random.PCG64(60))
    for n, world in ((1, 1), (7, 3), (1000, 8), (4096, 5), (5, 8)):
        ns = rng.integers(64, 2049, n) // 64 * 64
        parts = ray_shards(ns, world, layout="contiguous")
        assert len(parts) == world
        assert np.array_equal(np.concatenate(parts), np.arange(n))   # contiguous, in order, each slot once
        for s in parts:
            assert abs(int(ns[s].sum()) - ns.sum() / world) <= ns.max()
    # uniform counts: sizes within one ray
    sizes = [len(s) for s in ray_shards(np.full(1001, 512), 4, layout="contiguous")]
    assert max(sizes) - min(sizes) <= 1 and sum(sizes) == 1001
    # zero-sample rays and an empty screen
    assert [len(s) for s in ray_shards(np.zeros(0, dtype=np.int64), 3, layout="contiguous")] == [0, 0, 0]
    assert np.array_equal(np.concatenate(ray_shards(np.zeros(6, dtype=np.int64), 2, layout="contiguous")), np.arange(6))
    assert [len(s) for s in ray_shards(np.zeros(0, dtype=np.int64), 3)] == [0, 0, 0]   # strided, the default


def test_strided_shards_deal_every_world_th_slot():
    parts = ray_shards(np.full(10, 128), 3, layout="strided")
    assert [list(p) for p in parts] == [[0, 3, 6, 9], [1, 4, 7], [2, 5, 8]]
    with pytest.raises(ValueError):
        ray_shards(np.full(4, 1), 0)
    with pytest.raises(ValueError):
        ray_shards(np.full(4, 1), 2, layout="rows")


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import torch.distributed as dist
    from kerrsplat_b200.shard import allreduce_sum, gather_screen
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # each rank's partial [chi^2, dparams]: the sum comes back on every rank
        part = np.arange(5, dtype=np.float64) * (rank + 1) + 0.25
        red = allreduce_sum(part)
        # a screen of 7 pixels dealt unevenly (rank 0: 3 pixels, rank 1: 4), (2 frequencies, 1 frame)
        pixels = [np.array([0, 2, 5]), np.array([1, 3, 4, 6])]
        px = pixels[rank]
        mine = np.stack([np.stack([np.outer(px + 10 * f, np.ones(4)) for _ in range(1)]) for f in range(2)])
        screen = gather_screen(pixels, mine, 7)
        q.put((rank, red.tolist(), screen.tolist()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_allreduce_and_gather_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = (np.arange(5) * 3 + 0.5).tolist()
    expect = np.stack([np.stack([np.outer(np.arange(7) + 10 * f, np.ones(4))]) for f in range(2)])
    for _, red, screen in out:
        assert red == want
        assert np.array_equal(np.asarray(screen), expect)


@pytest.mark.gpu
def test_ray_shards_add_up_to_the_whole_screen():
    import kerrsplat_b200 as ks
    from kerrsplat_b200 import scenes
    from kerrsplat_b200.shard import RayShard, chi2_gradient_shard
    c = scenes.config2(res=32, N=128)
    rng = np.random.Generator(np.random.PCG64(61))
    p = scenes.thermal_params(rng, 8, c["a"])
    cam = c["camera"]
    times, nus = [0.0, 5.0], [86e9, 230e9]
    for uneven in (None, (768.0, 64)):
        cache = ks.GeodesicCache(cam, c["N"])
        ks.regenerate(cache, c["a"], c["theta_o"], uneven=uneven)
        target = np.asarray(ks.render(cache, ks.PolarizedSplats(p * 1.03), times, nus, c["L"], precision=ks.KS_FP64))
        scale = float(np.abs(target[..., 0]).max())
        assert scale > 0
        sigma = 0.01 * scale * (1.0 + rng.uniform(0, 1, target.shape))
        data = target + sigma * rng.standard_normal(target.shape)
        mask = rng.uniform(0, 1, target.shape[:3]) > 0.1
        m = ks.PolarizedSplats(p)
        counts = cache.nsamples_per_ray
        for precision, tc, tg in ((ks.KS_FP64, 1e-12, 1e-11), (ks.KS_MIXED, 1e-5, 1e-4)):
            chi_full, g_full = ks.chi2_gradient(cache, m, times, nus, c["L"], data, sigma, mask=mask, precision=precision)
            img_full = np.asarray(ks.render(cache, m, times, nus, c["L"], precision=precision))
            timg = 1e-13 if precision == ks.KS_FP64 else 1e-5
            for layout in ("contiguous", "strided"):
                shards = [RayShard(cam, c["N"], c["a"], c["theta_o"], rank=r, world=3, layout=layout, uneven=uneven) for r in range(3)]
                try:
                    assert np.array_equal(np.sort(np.concatenate([s.pixels for s in shards])), np.arange(cam.npix))
                    assert sum(s.samples_by_rank[s.rank] for s in shards) == int(counts.sum())
                    if layout == "contiguous":
                        for s in shards:
                            assert abs(s.samples_by_rank[s.rank] - counts.sum() / 3) <= counts.max()
                    vec = sum(chi2_gradient_shard(s, m, times, nus, c["L"], data, sigma, mask=mask, precision=precision) for s in shards)
                    assert abs(vec[0] - chi_full) <= tc * chi_full
                    g = vec[1:].reshape(p.shape[1], 21).T
                    assert np.linalg.norm(g - g_full) <= tg * np.linalg.norm(g_full)
                    for s in shards:
                        part = np.asarray(ks.render(s.cache, m, times, nus, c["L"], precision=precision))
                        assert np.abs(part - img_full[:, :, s.pixels]).max() <= timg * scale
                finally:
                    for s in shards:
                        s.close()
        cache.close()
