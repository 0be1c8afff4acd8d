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


# ---------------------------------------------------------------------------- m-sharded transform
def test_order_sets_and_pair_blocks_partition():
    for mmax in [0, 1, 7, 100, 4095]:
        for world in [1, 2, 3, 8]:
            s = D.order_sets(mmax, world)
            allm = np.sort(np.concatenate(s))
            assert np.array_equal(allm, np.arange(mmax + 1))
            loads = [int(np.sum(mmax + 1 - x)) for x in s]
            assert max(loads) - min(loads) <= mmax + 1  # within one order's l-range
    pix = np.array([4, 8, 12, 16, 16, 16, 16, 8])
    for world in [1, 2, 3, 8, 9]:
        b = D.pair_blocks(pix, world)
        assert b[0][0] == 0 and b[-1][1] == pix.size and all(b[i][1] == b[i + 1][0] for i in range(world - 1))


def _ms_worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from oracle import sht_oracle as O
        nside, lmax, nmaps = 8, 20, 2
        g = O.ring_tables(nside)
        nphi, rs = g["nphi"].astype(np.int64), g["ring_start"].astype(np.int64)
        north, south = D.healpix_pair_rings(nside)
        pix = nphi[north] + np.where(south >= 0, nphi[np.maximum(south, 0)], 0)
        lay = D.MShardLayout(lmax, pix, world)
        p0, p1 = lay.blocks[rank]
        mine = lay.msets[rank]
        rng = np.random.default_rng(1)
        maps = rng.standard_normal((nmaps, g["npix"]))
        cl = 1.0 / (np.arange(lmax + 1) + 3.0) ** 2
        alms = np.stack([O.synalm(cl, seed=7 + b) for b in range(nmaps)])

        def ring_F(b, r):  # oracle ring FFT of ring r alone: [mmax + 1]
            sg = O.ring_subset(g, int(r), int(r) + 1)
            return O.ring_analysis(maps[b, rs[r]:rs[r] + nphi[r]], sg, lmax, weights=g["weights_dz"][r:r + 1])[:, 0]

        # map2alm: this rank's ring pairs, exchange, this rank's orders
        F_local = np.zeros((nmaps, lmax + 1, p1 - p0, 2), dtype=np.complex128)
        for b in range(nmaps):
            for j, p in enumerate(range(p0, p1)):
                F_local[b, :, j, 0] = ring_F(b, north[p])
                if south[p] >= 0:
                    F_local[b, :, j, 1] = ring_F(b, south[p])
        Fm = D.exchange_analysis(torch.from_numpy(F_local), lay).numpy()
        assert Fm.shape == (nmaps, mine.size, lay.npairs, 2)
        alm_part = np.zeros((nmaps, alms.shape[1]), dtype=np.complex128)
        for b in range(nmaps):
            Fr = np.zeros((mine.size, g["nr"]), dtype=np.complex128)
            Fr[:, north] = Fm[b, :, :, 0]
            has = south >= 0
            Fr[:, south[has]] = Fm[b, :, has, 1].T
            rows = O.legendre_analysis_ms(Fr, g, lmax, mine)
            for j, m in enumerate(mine):
                alm_part[b, O.alm_index(lmax, np.arange(m, lmax + 1), int(m))] = rows[j, m:]
        full = torch.view_as_real(torch.from_numpy(alm_part)).contiguous()
        dist.all_reduce(full)
        full = torch.view_as_complex(full).numpy()
        err_a = max(float(np.max(np.abs(full[b] - O.map2alm(maps[b], g, lmax)))) for b in range(nmaps))

        # alm2map: this rank's orders, exchange, this rank's ring pairs
        Gm = np.zeros((nmaps, mine.size, lay.npairs, 2), dtype=np.complex128)
        for b in range(nmaps):
            Gr = O.legendre_synthesis_ms(O.alm_rows(alms[b], lmax, mine), g, lmax, mine)  # [|M_r|, nr]
            Gm[b, :, :, 0] = Gr[:, north]
            has = south >= 0
            Gm[b, :, has, 1] = Gr[:, south[has]].T
        Gl = D.exchange_synthesis(torch.from_numpy(Gm), lay).numpy()
        assert Gl.shape == (nmaps, lmax + 1, p1 - p0, 2)
        out = np.zeros((nmaps, g["npix"]))
        for b in range(nmaps):
            for j, p in enumerate(range(p0, p1)):
                for side, r in ((0, north[p]), (1, south[p])):
                    if r < 0:
                        continue
                    sg = O.ring_subset(g, int(r), int(r) + 1)
                    out[b, rs[r]:rs[r] + nphi[r]] = O.ring_synthesis(Gl[b, :, j, side][:, None], sg)
        tout = torch.from_numpy(out)
        dist.all_reduce(tout)
        err_m = max(float(np.max(np.abs(tout[b].numpy() - O.alm2map(alms[b], g, lmax)))) for b in range(nmaps))
        q.put((rank, err_a, err_m, int(mine.size), p1 - p0))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_msharded_transform_matches_unsharded_oracle(world):
    """The m-sharded split (ring-pair blocks for the FFTs, zig-zag order sets for the Legendre
    work, one all-to-all per direction) reproduces the unsharded oracle map2alm and alm2map."""
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    mp.start_processes(_ms_worker, args=(world, _free_port(), q), nprocs=world, start_method="spawn")
    res = sorted(q.get() for _ in range(world))
    assert all(r[1] < 1e-12 and r[2] < 1e-12 for r in res), res
    assert sum(r[3] for r in res) == 21 and sum(r[4] for r in res) == 16  # orders 0..20, 2 nside pairs


@pytest.mark.gpu
@pytest.mark.parametrize("world,prec", [(1, 64), (3, 64), (4, 32)])
def test_gpu_msharded_ranks_in_one_process_match_unsharded(world, prec):
    """Every rank's share of the m-sharded transform (its local ring geometry, the ring FFTs of
    its pairs, the Legendre stages of its orders through hb_legendre_*_ms) run in one process,
    the all-to-all done in memory: the combined result equals the single-GPU transform
    (FP64: 1e-10; FP32: 1e-5 against FP64)."""
    import hellblast_b200 as hb
    nside, lmax = 64, 150
    ct = torch.complex128 if prec == 64 else torch.complex64
    cl = 1.0 / (np.arange(lmax + 1) + 10.0) ** 2
    alm = torch.stack([hb.synalm(cl, lmax=lmax, seed=40 + i, device="cuda") for i in range(2)])
    ref_map = hb.hp_compat.alm2map(alm, nside, lmax=lmax)
    ref_alm = hb.hp_compat.map2alm(ref_map, lmax=lmax)
    ranks = [D.MShardedSHT(nside, lmax, precision=prec, rank=r, world=world) for r in range(world)]
    lay = ranks[0].layout
    # map2alm: ring FFTs per rank, in-memory all-to-all, Legendre per rank
    F = [s.ring_analysis(s.local_pixels(ref_map)) for s in ranks]
    got = torch.zeros_like(ref_alm, dtype=ct)
    for r, s in enumerate(ranks):
        idx = torch.as_tensor(lay.msets[r], dtype=torch.long, device="cuda")
        Fm = torch.cat([F[q].index_select(1, idx) for q in range(world)], dim=2)
        got += s.legendre_analysis(Fm)
    tol = 1e-10 if prec == 64 else 1e-5
    assert float(torch.linalg.norm(got.to(torch.complex128) - ref_alm) / torch.linalg.norm(ref_alm)) < tol
    # alm2map: Legendre per rank, in-memory all-to-all, ring FFTs per rank
    Gm = [s.legendre_synthesis(alm) for s in ranks]
    out = torch.zeros_like(ref_map, dtype=torch.float64)
    for r, s in enumerate(ranks):
        p0, p1 = lay.blocks[r]
        Gl = torch.zeros(2, lmax + 1, p1 - p0, 2, dtype=ct, device="cuda")
        for q in range(world):
            Gl[:, torch.as_tensor(lay.msets[q], dtype=torch.long, device="cuda")] = Gm[q][:, :, p0:p1]
        s.map_from_local(out, s.ring_synthesis(Gl).double())
    assert float(torch.linalg.norm(out - ref_map) / torch.linalg.norm(ref_map)) < tol
