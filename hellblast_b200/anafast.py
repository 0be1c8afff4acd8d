"""Power spectrum of a ring map (anafast.py:5-7 = alm2cl(map2alm_gpu(...)))."""
from __future__ import annotations

from . import alm_ops
from .sht import map2alm_gpu


def anafast_ring(rings, thetas, nphi_per_ring, weights_dz, lmax, *, precision=None):
    alm = map2alm_gpu(rings, thetas, nphi_per_ring, weights_dz, lmax, precision=precision)
    return alm_ops.alm2cl(alm, lmax=lmax)
