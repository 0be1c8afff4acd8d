"""healpy-style flat-map API (hp_compat.py:24-117 of the reference), healpy m-major alm.

Differences from the reference, on purpose: ``anafast`` exists (the reference imports
_anafast_ring at hp_compat.py:15 but never wraps it); spin-2 uses one consistent convention;
``nest`` is accepted and ignored, as in the reference (hp_compat.py:40,50,57,71).
"""
from __future__ import annotations

import math

import torch

from . import alm_ops, transforms
from . import geometry as G
from .ring_tables import HealpixRingTables  # noqa: F401
from .util import as_tensor, like_input


def _geom(npix_or_nside, weights="dz", by_npix=True):
    nside = transforms.nside_from_npix(npix_or_nside) if by_npix else int(npix_or_nside)
    return G.healpix(nside, weights=weights), nside


def map2alm(m, lmax=None, mmax=None, nest=False, *, weights="dz", precision=None):
    """alm of a RING map ([npix] or [nmaps, npix]); default lmax = 3*nside (hp_compat.py:45)."""
    t = as_tensor(m)
    g, nside = _geom(t.shape[-1], "uniform" if weights == "uniform" else "dz")
    lmax = 3 * nside if lmax is None else int(lmax)
    w = None if isinstance(weights, str) else weights
    return like_input(transforms.map2alm(t, g, lmax, mmax, weights=w, precision=precision), m)


def alm2map(alm, nside, lmax=None, mmax=None, nest=False, *, precision=None):
    t = as_tensor(alm)
    lmax = alm_ops.getlmax(t.shape[-1], mmax) if lmax is None else int(lmax)
    g, _ = _geom(nside, by_npix=False)
    return like_input(transforms.alm2map(t, g, lmax, mmax, precision=precision), alm)


def anafast(map1, map2=None, lmax=None, mmax=None, alm=False, *, weights="dz", precision=None):
    """C_l of a map (or the cross spectrum of two); with ``alm=True`` also returns the alm."""
    a1 = map2alm(map1, lmax=lmax, mmax=mmax, weights=weights, precision=precision)
    a2 = None if map2 is None else map2alm(map2, lmax=lmax, mmax=mmax, weights=weights, precision=precision)
    cl = alm_ops.alm2cl(a1, a2, mmax=mmax)
    return (cl, a1, a2) if alm else cl


def alm2cl(alms, alms2=None, lmax=None, mmax=None):
    return alm_ops.alm2cl(alms, alms2, lmax=lmax, mmax=mmax)


def almxfl(alm, fl, mmax=None, inplace=False):
    return alm_ops.almxfl(alm, fl, mmax=mmax, inplace=inplace)


def synalm(cls, lmax=None, mmax=None, seed=None):
    return alm_ops.synalm(cls, lmax=lmax, mmax=mmax, seed=seed)


def map2alm_spin(Q, U=None, spin=2, lmax=None, mmax=None, nest=False, *, weights="dz", precision=None):
    """(E, B) from Q, U (hp_compat.py:57-69).  ``Q`` may also be the pair [Q, U] (healpy form)."""
    if U is None:
        Q, U = Q
    if spin != 2:
        raise ValueError("spin must be 2 (spin-1 is outside this library)")
    q = as_tensor(Q)
    g, nside = _geom(q.shape[-1], "uniform" if weights == "uniform" else "dz")
    lmax = 3 * nside if lmax is None else int(lmax)
    w = None if isinstance(weights, str) else weights
    E, B = transforms.map2alm_spin2(q, as_tensor(U), g, lmax, mmax, weights=w, precision=precision)
    return like_input(E, Q), like_input(B, Q)


def alm2map_spin(Aplus, Aminus=None, spin=2, nside=None, lmax=None, mmax=None, nest=False, *, precision=None):
    """(Q, U) from E, B (hp_compat.py:71-84); without nside the reference picks ceil(lmax/3)."""
    if Aminus is None:
        Aplus, Aminus = Aplus
    if spin != 2:
        raise ValueError("spin must be 2 (spin-1 is outside this library)")
    e = as_tensor(Aplus)
    lmax = alm_ops.getlmax(e.shape[-1], mmax) if lmax is None else int(lmax)
    if nside is None:
        nside = max(1, int(math.ceil(lmax / 3)))
        nside = 1 << (nside - 1).bit_length()
    g, _ = _geom(nside, by_npix=False)
    Q, U = transforms.alm2map_spin2(e, as_tensor(Aminus), g, lmax, mmax, precision=precision)
    return like_input(Q, Aplus), like_input(U, Aplus)


def iqu2eb(Q, U, lmax=None, nest=False):
    return map2alm_spin(Q, U, 2, lmax=lmax)


def eb2iqu(E, B, nside=None, lmax=None, nest=False):
    return alm2map_spin(E, B, 2, nside=nside, lmax=lmax)
