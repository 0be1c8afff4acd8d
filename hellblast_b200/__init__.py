"""hellblast_b200: B200-native (sm_100a) HEALPix spherical-harmonic transforms.

Drop-in for the SHT hot path of hellblast (map2alm_gpu, alm2map_gpu, anafast_ring, alm2cl and
the hp_compat scalar/spin-2 entry points), healpy m-major alm packing by default.  All compute
runs in the hand-written CUDA kernels of hellblast_b200/_lib/libhbsht.so (C ABI:
include/hbsht.h), exposed as torch.ops.hb.*; there is no CPU fallback.
"""
__version__ = "0.2.0"

from . import _lib  # noqa: F401
from . import ops  # noqa: F401  (registers torch.ops.hb.*)
from .alm_ops import alm2cl, alm_index, alm_size, almxfl, getlmax, healpy_to_ref, ref_to_healpy, synalm
from .anafast import anafast_ring
from .isht import alm2map_gpu
from .ring_tables import HealpixRingTables
from .sht import map2alm_gpu
from .spin import eb_from_qu_gpu, map2alm_spin_gpu, qu_from_eb_gpu
from . import hp_compat  # noqa: F401
from . import autograd  # noqa: F401
from . import batched  # noqa: F401
from . import smoothing  # noqa: F401
from . import synfast  # noqa: F401
from . import distributed  # noqa: F401
from . import pixelfunc  # noqa: F401
from . import io_fits  # noqa: F401
from . import rotate  # noqa: F401

map2alm = map2alm_gpu
alm2map = alm2map_gpu
anafast = anafast_ring


def clear_caches() -> None:
    """Drop the cached geometries, transform plans and batched plans.  Their device memory
    (recursion checkpoints, tile and ring buffers: tens of GB at nside >= 2048) is freed as soon
    as no caller still holds the objects; the torch allocator's unused blocks are released too."""
    import gc

    import torch

    from . import geometry as _geometry

    with batched._lock:
        batched._cache.clear()
    with _geometry._lock:
        _geometry._cache.clear()
    gc.collect()
    if torch.cuda.is_available():
        torch.cuda.empty_cache()


__all__ = [
    "map2alm_gpu", "alm2map_gpu", "anafast_ring", "map2alm", "alm2map", "anafast",
    "almxfl", "alm2cl", "synalm", "alm_index", "alm_size", "getlmax", "healpy_to_ref", "ref_to_healpy",
    "HealpixRingTables", "map2alm_spin_gpu", "eb_from_qu_gpu", "qu_from_eb_gpu", "hp_compat", "autograd",
    "batched", "smoothing", "synfast", "distributed", "pixelfunc", "io_fits", "rotate", "clear_caches",
]
