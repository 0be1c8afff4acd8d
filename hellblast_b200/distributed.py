"""Multi-GPU batches: one process per GPU, the maps of a batch sharded across ranks.

The maps of a batch are independent, so the data path shards them with no collective: rank r
transforms maps [start_r, stop_r) on its own GPU (``scaling: weak`` in bench.py, every rank a
replica of the single-GPU path).  A collective runs only where a caller asks for the results
on every rank (``gather``), over NCCL between GPUs or gloo on CPU.  The reference has no
multi-GPU path (its SHT runs on CuPy's current device, sht_raw.py:30-57).

    from hellblast_b200 import distributed as D
    alm_local = D.map2alm(D.local_shard(maps), nside, lmax)        # no communication
    alm_all = D.gather(alm_local, maps.shape[0])                    # optional all-gather
"""
from __future__ import annotations

from typing import Callable

import torch
import torch.distributed as dist


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous, balanced shard [start, stop) of n items for ``rank`` of ``world``; the first
    n % world ranks take one item more."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    if n < 0:
        raise ValueError("n must be >= 0")
    q, r = divmod(n, world)
    start = rank * q + min(rank, r)
    return start, start + q + (1 if rank < r else 0)


def world_info(group=None) -> tuple[int, int]:
    """(rank, world size) of the default or given process group; (0, 1) without one."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def local_shard(batch: torch.Tensor, group=None) -> torch.Tensor:
    """This rank's rows of a ``[nmaps, ...]`` batch (a view, no copy)."""
    rank, world = world_info(group)
    a, b = shard_range(batch.shape[0], rank, world)
    return batch[a:b]


def gather(local: torch.Tensor, n_total: int, group=None) -> torch.Tensor:
    """Concatenate every rank's shard, in rank order, into the ``[n_total, ...]`` batch on every
    rank.  Shards are padded to the largest for the collective and trimmed after; complex
    tensors travel as their real view."""
    rank, world = world_info(group)
    counts = [b - a for a, b in (shard_range(n_total, r, world) for r in range(world))]
    if local.shape[0] != counts[rank]:
        raise ValueError(f"rank {rank} holds {local.shape[0]} rows, its shard of {n_total} has {counts[rank]}")
    if world == 1:
        return local
    cplx = local.is_complex()
    x = torch.view_as_real(local) if cplx else local
    pad = torch.zeros((max(counts),) + tuple(x.shape[1:]), dtype=x.dtype, device=x.device)
    pad[: x.shape[0]] = x
    outs = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(outs, pad, group=group)
    y = torch.cat([o[:c] for o, c in zip(outs, counts)])
    return torch.view_as_complex(y) if cplx else y


def run_sharded(fn: Callable[[torch.Tensor], torch.Tensor], batch: torch.Tensor, group=None,
                gather_result: bool = False) -> torch.Tensor:
    """Apply a batched transform ``fn`` to this rank's shard of ``batch``; with
    ``gather_result`` every rank receives the full result batch."""
    out = fn(local_shard(batch, group))
    return gather(out, batch.shape[0], group) if gather_result else out


def map2alm(maps_local: torch.Tensor, nside: int, lmax: int, mmax: int | None = None, **kw) -> torch.Tensor:
    """Batched map2alm of this rank's maps ([n, npix] float32 on this rank's GPU) through the
    tensor-core path; an empty shard gives an empty result."""
    from . import batched
    from .ops import alm_size
    if maps_local.shape[0] == 0:
        mm = lmax if mmax is None else mmax
        return torch.empty(0, alm_size(lmax, mm), dtype=torch.complex64, device=maps_local.device)
    return batched.map2alm(maps_local, nside, lmax, mmax, **kw)


def alm2map(alm_local: torch.Tensor, nside: int, lmax: int, mmax: int | None = None, **kw) -> torch.Tensor:
    """Batched alm2map of this rank's alm ([n, nalm] complex64 on this rank's GPU)."""
    from . import batched
    if alm_local.shape[0] == 0:
        return torch.empty(0, 12 * nside * nside, dtype=torch.float32, device=alm_local.device)
    return batched.alm2map(alm_local, nside, lmax, mmax, **kw)


# ----------------------------------------------------------------------------- m-sharded transform
# One transform split over ranks (the reference's split point sht_raw.py:38-43 | 46-56: per-ring
# FFTs, then per-order contractions).  Map2alm: rank r runs the ring FFTs of its block of ring
# pairs for every order m, one all-to-all sends each rank the orders it owns (for every pair),
# and rank r runs the Legendre analysis of its orders over all pairs.  Alm2map is the mirror
# image.  Orders go to ranks in a zig-zag over 2 * world (m and mmax - m on the same rank), so
# every rank gets nearly the same sum of l-range lengths; ring pairs go in contiguous blocks
# balanced by pixel count.  The exchange is one torch.distributed.all_to_all_single per
# direction (NCCL between GPUs, gloo on CPU), on the real view of the complex blocks.

def order_sets(mmax: int, world: int) -> list:
    """Orders of each rank: m goes to rank k if m mod 2w = k < w, else to 2w - 1 - (m mod 2w)."""
    if world <= 0 or mmax < 0:
        raise ValueError("need world >= 1 and mmax >= 0")
    sets = [[] for _ in range(world)]
    for m in range(mmax + 1):
        k = m % (2 * world)
        sets[k if k < world else 2 * world - 1 - k].append(m)
    import numpy as np
    return [np.asarray(s, dtype=np.int32) for s in sets]


def pair_blocks(pair_pixels, world: int) -> list:
    """Contiguous blocks [p0, p1) of ring pairs, one per rank, balanced by pixel count
    (``pair_pixels[p]``: pixels of pair p, both rings)."""
    import numpy as np
    pix = np.asarray(pair_pixels, dtype=np.int64)
    if world <= 0:
        raise ValueError("world must be >= 1")
    cum = np.concatenate([[0], np.cumsum(pix)])
    cuts = [0] + [int(np.searchsorted(cum, cum[-1] * k / world)) for k in range(1, world)] + [pix.size]
    cuts = np.maximum.accumulate(np.minimum(cuts, pix.size))
    return [(int(cuts[k]), int(cuts[k + 1])) for k in range(world)]


class MShardLayout:
    """Who owns what in an m-sharded transform: ``msets[r]`` (orders of rank r) and
    ``blocks[r]`` (its ring pairs [p0, p1)); npairs and mmax of the transform."""

    def __init__(self, mmax: int, pair_pixels, world: int):
        self.mmax, self.world = int(mmax), int(world)
        self.npairs = len(pair_pixels)
        self.msets = order_sets(self.mmax, self.world)
        self.blocks = pair_blocks(pair_pixels, self.world)

    def npl(self, r: int) -> int:
        return self.blocks[r][1] - self.blocks[r][0]


def _a2a(send_blocks, recv_shapes, dtype, device, group):
    """all_to_all_single over the real views of complex blocks; returns the received blocks."""
    rank, world = world_info(group)
    flat = [torch.view_as_real(b.contiguous()).reshape(-1) for b in send_blocks]
    send = torch.cat(flat) if flat else torch.empty(0, device=device)
    sizes_in = [f.numel() for f in flat]
    sizes_out = [2 * int(torch.Size(s).numel()) for s in recv_shapes]
    recv = torch.empty(sum(sizes_out), dtype=send.dtype, device=device)
    if world == 1:
        recv.copy_(send)
    else:
        dist.all_to_all_single(recv, send, sizes_out, sizes_in, group=group)
    out, o = [], 0
    for s, n in zip(recv_shapes, sizes_out):
        out.append(torch.view_as_complex(recv[o:o + n].reshape(tuple(s) + (2,))))
        o += n
    return out


def exchange_analysis(F_local: torch.Tensor, layout: MShardLayout, group=None) -> torch.Tensor:
    """[nmaps, mmax+1, npl_r, 2] ring-FFT output of this rank's pairs -> [nmaps, |M_r|, npairs, 2],
    the Fourier coefficients of this rank's orders for every pair (pairs in global order)."""
    rank, world = world_info(group)
    nmaps = F_local.shape[0]
    idx = [torch.as_tensor(layout.msets[q], dtype=torch.long, device=F_local.device) for q in range(world)]
    send = [F_local.index_select(1, idx[q]) for q in range(world)]
    shapes = [(nmaps, len(layout.msets[rank]), layout.npl(q), 2) for q in range(world)]
    recv = _a2a(send, shapes, F_local.dtype, F_local.device, group)
    return torch.cat(recv, dim=2)


def exchange_synthesis(G_m: torch.Tensor, layout: MShardLayout, group=None) -> torch.Tensor:
    """[nmaps, |M_r|, npairs, 2] Legendre-synthesis output of this rank's orders ->
    [nmaps, mmax+1, npl_r, 2], every order's coefficients for this rank's ring pairs."""
    rank, world = world_info(group)
    nmaps = G_m.shape[0]
    send = [G_m[:, :, layout.blocks[q][0]:layout.blocks[q][1]] for q in range(world)]
    shapes = [(nmaps, len(layout.msets[q]), layout.npl(rank), 2) for q in range(world)]
    recv = _a2a(send, shapes, G_m.dtype, G_m.device, group)
    out = torch.zeros(nmaps, layout.mmax + 1, layout.npl(rank), 2, dtype=G_m.dtype, device=G_m.device)
    for q in range(world):
        out[:, torch.as_tensor(layout.msets[q], dtype=torch.long, device=G_m.device)] = recv[q]
    return out


def healpix_pair_rings(nside: int):
    """Global ring indices (north, south) of each ring pair of a HEALPix grid, in the pair order
    of its geometry: pair p = rings (p, nr - 1 - p), the equator last and unpaired (south -1)."""
    import numpy as np
    nr = 4 * nside - 1
    north = np.arange((nr + 1) // 2)
    south = nr - 1 - north
    south[south == north] = -1
    return north, south


class MShardedSHT:
    """The m-sharded FP32 (or FP64) scalar transform of a HEALPix map on this rank's GPU.

    ``local_rings`` lists the global ring indices of this rank's pair block in the order of its
    local geometry (north rings ascending, then the south rings in ascending theta);
    ``local_pixels(maps)`` / ``map_from_local`` move between full RING maps and that order.
    ``map2alm(x_local)``: [nmaps, npix_local] -> [nmaps, nalm] with this rank's orders filled;
    ``alm2map(alm)``: the alm of this rank's orders (other rows ignored) -> [nmaps, npix_local].
    Every rank must make the same calls in the same order (each direction is one collective).
    The stages (``ring_analysis``, ``legendre_analysis``, ``legendre_synthesis``,
    ``ring_synthesis``) are public so that one process can run every rank's share (``rank`` /
    ``world`` given explicitly) with the exchange done in memory."""

    def __init__(self, nside: int, lmax: int, mmax: int | None = None, precision: int = 32, group=None,
                 device=None, rank: int | None = None, world: int | None = None):
        import numpy as np
        from . import geometry as G
        self.group = group
        self.rank, self.world = world_info(group)
        if rank is not None or world is not None:
            self.rank, self.world = int(rank), int(world)
        self.nside, self.lmax = int(nside), int(lmax)
        self.mmax = self.lmax if mmax is None else int(mmax)
        self.prec = int(precision)
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.g = G.healpix(self.nside)
        self.plan = G.plan(self.g, self.lmax, self.mmax, precision=self.prec)
        t = G.host_ring_tables(self.nside)
        north, south = healpix_pair_rings(self.nside)
        nphi = t["nphi"].astype(np.int64)
        pix = nphi[north] + np.where(south >= 0, nphi[np.maximum(south, 0)], 0)
        self.layout = MShardLayout(self.mmax, pix, self.world)
        p0, p1 = self.layout.blocks[self.rank]
        sl = [int(r) for r in south[p0:p1][::-1] if r >= 0]
        self.local_rings = np.concatenate([north[p0:p1], np.asarray(sl, dtype=np.int64)]).astype(np.int64)
        rs = t["ring_start"].astype(np.int64)
        self.local_index = torch.as_tensor(np.concatenate([np.arange(rs[r], rs[r] + nphi[r]) for r in self.local_rings])
                                           if self.local_rings.size else np.zeros(0, np.int64), device=self.device)
        if self.local_rings.size:
            lr = self.local_rings
            self.lg = G.generic(t["theta"][lr], nphi[lr].astype(np.int32), t["weights_dz"][lr],
                                phi0=t["phi0"][lr])
            if self.lg.npairs != p1 - p0:
                raise RuntimeError("local ring block did not pair up like the global grid")
            self.lplan = G.plan(self.lg, self.lmax, self.mmax, precision=self.prec)
        else:
            self.lg = self.lplan = None
        self.mlist = torch.as_tensor(self.layout.msets[self.rank], dtype=torch.int32, device=self.device)
        self.rt = torch.float32 if self.prec == 32 else torch.float64
        self.ct = torch.complex64 if self.prec == 32 else torch.complex128

    @property
    def npix_local(self) -> int:
        return int(self.local_index.numel())

    def local_pixels(self, maps: torch.Tensor) -> torch.Tensor:
        """This rank's pixels of full RING maps [nmaps, npix], in local ring order."""
        return maps.index_select(-1, self.local_index)

    def map_from_local(self, out: torch.Tensor, local: torch.Tensor) -> torch.Tensor:
        """Write this rank's pixels back into full RING maps ``out`` [nmaps, npix]."""
        out[:, self.local_index] = local
        return out

    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def ring_analysis(self, x_local: torch.Tensor) -> torch.Tensor:
        """[nmaps, npix_local] -> [nmaps, mmax+1, npl, 2]: ring FFTs of this rank's pairs."""
        from . import _lib as L
        nmaps = x_local.shape[0]
        F = torch.zeros(nmaps, self.mmax + 1, self.layout.npl(self.rank), 2, dtype=self.ct, device=self.device)
        if self.npix_local:
            x = x_local.to(self.rt).contiguous()
            L.call("hb_ring_analysis", self.lplan.handle, self.prec, nmaps, x.data_ptr(), None, F.data_ptr(), 0,
                   self._stream())
        return F

    def legendre_analysis(self, Fm: torch.Tensor) -> torch.Tensor:
        """[nmaps, |M_r|, npairs, 2] -> [nmaps, nalm] with this rank's orders filled."""
        from . import _lib as L
        Fm = Fm.to(self.ct).contiguous()
        nmaps = Fm.shape[0]
        alm = torch.zeros(nmaps, L.lib().hb_alm_size(self.lmax, self.mmax), dtype=self.ct, device=self.device)
        if self.mlist.numel():
            L.call("hb_legendre_analysis_ms", self.plan.handle, self.prec, nmaps, int(self.mlist.numel()),
                   self.mlist.data_ptr(), Fm.data_ptr(), alm.data_ptr(), self._stream())
        return alm

    def legendre_synthesis(self, alm: torch.Tensor) -> torch.Tensor:
        """alm [nmaps, nalm] (this rank's orders read) -> [nmaps, |M_r|, npairs, 2]."""
        from . import _lib as L
        a = alm.to(self.ct).contiguous()
        nmaps = a.shape[0]
        Gm = torch.zeros(nmaps, int(self.mlist.numel()), self.g.npairs, 2, dtype=self.ct, device=self.device)
        if self.mlist.numel():
            L.call("hb_legendre_synthesis_ms", self.plan.handle, self.prec, nmaps, int(self.mlist.numel()),
                   self.mlist.data_ptr(), a.data_ptr(), Gm.data_ptr(), self._stream())
        return Gm

    def ring_synthesis(self, G_local: torch.Tensor) -> torch.Tensor:
        """[nmaps, mmax+1, npl, 2] -> [nmaps, npix_local]: ring FFTs of this rank's pairs."""
        from . import _lib as L
        Gl = G_local.to(self.ct).contiguous()
        nmaps = Gl.shape[0]
        out = torch.empty(nmaps, self.npix_local, dtype=self.rt, device=self.device)
        if self.npix_local:
            L.call("hb_ring_synthesis", self.lplan.handle, self.prec, nmaps, Gl.data_ptr(), out.data_ptr(), 0,
                   self._stream())
        return out

    def map2alm(self, x_local: torch.Tensor) -> torch.Tensor:
        return self.legendre_analysis(exchange_analysis(self.ring_analysis(x_local), self.layout, self.group))

    def alm2map(self, alm: torch.Tensor) -> torch.Tensor:
        return self.ring_synthesis(exchange_synthesis(self.legendre_synthesis(alm), self.layout, self.group))
