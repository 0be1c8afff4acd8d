"""Spin-2 transforms with the names of hellblast's spin.py (spin.py:32-115), in one consistent
HEALPix convention: a(+-2)_lm = -(E_lm +- i B_lm), E = -(a2 + a-2)/2, B = i (a2 - a-2)/2.

``ref_compat=True`` reproduces the reference's own conventions (no phi0 phase, no alias fold,
its m cut and its d^l_{m,+-2} spin functions, i.e. U -> -U), see transforms.map2alm_spin2;
``alm_layout="ref_lsquare"`` returns / takes the reference's l(l+1)+m layout."""
from __future__ import annotations

from . import alm_ops, transforms
from .util import as_tensor, like_input


def _out_layout(a, lmax, mmax, alm_layout):
    if alm_layout == "ref_lsquare":
        return alm_ops.healpy_to_ref(a, lmax, lmax if mmax is None else mmax)
    if alm_layout != "healpy":
        raise ValueError("alm_layout must be 'healpy' or 'ref_lsquare'")
    return a


def eb_from_qu_gpu(Q_rings, U_rings, thetas, nphi_per_ring, weights_dz, lmax, mmax=None, *, precision=None,
                   ref_compat=False, alm_layout="healpy"):
    """(E_lm, B_lm) of Q/U rings (spin.py:73-78)."""
    g = transforms.geometry_for(thetas, nphi_per_ring, weights_dz)
    E, B = transforms.map2alm_spin2(Q_rings, U_rings, g, lmax, mmax, weights=weights_dz, precision=precision,
                                    ref_compat=ref_compat)
    ref = Q_rings[0] if isinstance(Q_rings, (list, tuple)) else Q_rings
    return (like_input(_out_layout(E, lmax, mmax, alm_layout), ref),
            like_input(_out_layout(B, lmax, mmax, alm_layout), ref))


def map2alm_spin_gpu(Q_rings, U_rings, thetas, nphi_per_ring, weights_dz, lmax, mmax=None, *, precision=None,
                     ref_compat=False, alm_layout="healpy"):
    """Returns (a2_lm, a-2_lm) (spin.py:32-71)."""
    E, B = eb_from_qu_gpu(Q_rings, U_rings, thetas, nphi_per_ring, weights_dz, lmax, mmax, precision=precision,
                          ref_compat=ref_compat, alm_layout=alm_layout)
    return -(E + 1j * B), -(E - 1j * B)


def qu_from_eb_gpu(Ealm, Balm, thetas, nphi_per_ring, lmax, mmax=None, *, flat=False, precision=None,
                   ref_compat=False, alm_layout="healpy"):
    """(Q rings, U rings) from E, B (spin.py:80-115, with a2 = -(E + iB))."""
    if alm_layout == "ref_lsquare":
        Ealm = alm_ops.ref_to_healpy(as_tensor(Ealm), lmax, lmax if mmax is None else mmax)
        Balm = alm_ops.ref_to_healpy(as_tensor(Balm), lmax, lmax if mmax is None else mmax)
    elif alm_layout != "healpy":
        raise ValueError("alm_layout must be 'healpy' or 'ref_lsquare'")
    g = transforms.geometry_for(thetas, nphi_per_ring)
    Q, U = transforms.alm2map_spin2(Ealm, Balm, g, lmax, mmax, precision=precision, ref_compat=ref_compat)
    if flat:
        return like_input(Q, Ealm), like_input(U, Ealm)
    return ([like_input(r, Ealm) for r in transforms.split_rings(Q, g)],
            [like_input(r, Ealm) for r in transforms.split_rings(U, g)])
