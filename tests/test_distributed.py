"""Multi-GPU batch sharding (hellblast_b200.distributed) on CPU: shard ranges, and world-size-2
gloo runs of run_sharded / gather with the oracle standing in for the per-rank GPU transform."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from hellblast_b200 import distributed as D


def test_shard_range_partitions_every_batch():
    for n in [0, 1, 2, 3, 7, 64, 65, 1000]:
        for world in [1, 2, 3, 4, 8]:
            rs = [D.shard_range(n, r, world) for r in range(world)]
            assert rs[0][0] == 0 and rs[-1][1] == n
            assert all(rs[i][1] == rs[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in rs]
            assert max(sizes) - min(sizes) <= 1 and sum(sizes) == n


def test_shard_range_rejects_bad_arguments():
    for args in [(3, 2, 2), (3, -1, 2), (3, 0, 0), (-1, 0, 1)]:
        with pytest.raises(ValueError):
            D.shard_range(*args)


def test_single_process_is_identity():
    x = torch.arange(12.0).reshape(4, 3)
    assert D.world_info() == (0, 1)
    assert torch.equal(D.local_shard(x), x)
    assert torch.equal(D.gather(x, 4), x)
    assert torch.equal(D.run_sharded(lambda t: 2 * t, x, gather_result=True), 2 * x)
    with pytest.raises(ValueError):
        D.gather(x[:3], 4)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from oracle import sht_oracle as O
        nside, lmax = 4, 7
        geom = O.ring_tables(nside)
        nalm = (lmax + 1) * (lmax + 2) // 2
        rng = np.random.default_rng(5)
        maps = torch.from_numpy(rng.standard_normal((3, 12 * nside * nside)))

        def fn(x):
            if x.shape[0] == 0:
                return torch.empty(0, nalm, dtype=torch.complex128)
            return torch.from_numpy(np.stack([O.map2alm(m.numpy(), geom, lmax) for m in x]))

        local = D.run_sharded(fn, maps)
        full = D.run_sharded(fn, maps, gather_result=True)
        ref = fn(maps)
        # complex64 shards of unequal length through the real-view path
        c = (torch.arange(10, dtype=torch.float32).reshape(5, 2) * (1 + 1j)).to(torch.complex64)
        cg = D.gather(D.local_shard(c), 5)
        q.put((rank, local.shape[0], float((full - ref).abs().max()), bool(torch.equal(cg, c))))
    finally:
        dist.destroy_process_group()


def test_gloo_world2_sharded_map2alm_matches_unsharded():
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    mp.start_processes(_worker, args=(2, _free_port(), q), nprocs=2, start_method="spawn")
    res = sorted(q.get() for _ in range(2))
    assert [r[1] for r in res] == [2, 1]          # 3 maps over 2 ranks
    assert all(r[2] < 1e-12 for r in res)         # gathered result == unsharded transform
    assert all(r[3] for r in res)


@pytest.mark.gpu
def test_gpu_rank_local_transforms_match_batched():
    import hellblast_b200 as hb
    nside, lmax = 32, 63
    cl = 1.0 / (np.arange(lmax + 1) + 10.0) ** 2
    alm = torch.stack([hb.synalm(cl, lmax=lmax, seed=i, device="cuda", dtype=torch.complex64) for i in range(3)])
    m = D.alm2map(D.local_shard(alm), nside, lmax)
    assert torch.equal(m, hb.batched.alm2map(alm, nside, lmax))
    a = D.map2alm(D.local_shard(m), nside, lmax)
    assert torch.equal(a, hb.batched.map2alm(m, nside, lmax))
    assert D.map2alm(m[:0], nside, lmax).shape == (0, alm.shape[1])
