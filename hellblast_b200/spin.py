"""Spin-2 transforms with the names of hellblast's spin.py (spin.py:32-115), in one consistent
HEALPix convention: a(+-2)_lm = -(E_lm +- i B_lm), E = -(a2 + a-2)/2, B = i (a2 - a-2)/2."""
from __future__ import annotations

from . import transforms
from .util import like_input


def eb_from_qu_gpu(Q_rings, U_rings, thetas, nphi_per_ring, weights_dz, lmax, mmax=None, *, precision=None):
    g = transforms.geometry_for(thetas, nphi_per_ring, weights_dz)
    E, B = transforms.map2alm_spin2(Q_rings, U_rings, g, lmax, mmax, weights=weights_dz, precision=precision)
    ref = Q_rings[0] if isinstance(Q_rings, (list, tuple)) else Q_rings
    return like_input(E, ref), like_input(B, ref)


def map2alm_spin_gpu(Q_rings, U_rings, thetas, nphi_per_ring, weights_dz, lmax, mmax=None, *, precision=None):
    """Returns (a2_lm, a-2_lm) (spin.py:32-71)."""
    E, B = eb_from_qu_gpu(Q_rings, U_rings, thetas, nphi_per_ring, weights_dz, lmax, mmax, precision=precision)
    return -(E + 1j * B), -(E - 1j * B)


def qu_from_eb_gpu(Ealm, Balm, thetas, nphi_per_ring, lmax, mmax=None, *, flat=False, precision=None):
    """(Q rings, U rings) from E, B (spin.py:80-115, with a2 = -(E + iB))."""
    g = transforms.geometry_for(thetas, nphi_per_ring)
    Q, U = transforms.alm2map_spin2(Ealm, Balm, g, lmax, mmax, precision=precision)
    if flat:
        return like_input(Q, Ealm), like_input(U, Ealm)
    return ([like_input(r, Ealm) for r in transforms.split_rings(Q, g)],
            [like_input(r, Ealm) for r in transforms.split_rings(U, g)])
