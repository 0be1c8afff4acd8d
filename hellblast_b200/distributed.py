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
