"""Forward scalar SHT with the signature of hellblast's ``map2alm_gpu`` (sht.py:1-4 ->
sht_raw.py:30 / sht_fallback.py:36)."""
from __future__ import annotations

from . import alm_ops, transforms
from .util import like_input


def map2alm_gpu(rings, thetas, nphi_per_ring, weights_dz, lmax, mmax=None, *, precision=None,
                alm_layout="healpy", ref_compat=None, phi0=None):
    """a_lm = sum_pix (2 pi w_r / nphi_r) f(pix) conj(Y_lm(pix)).

    rings: list of per-ring arrays (as in the reference) or one flat RING-ordered array
    ([npix] or [nmaps, npix]); torch tensors, CuPy arrays (DLPack) or numpy arrays.
    precision: None (follow the input dtype: float32 -> FP32 kernels, else FP64), "fp32", "fp64".
    alm_layout: "healpy" (m-major, default) or "ref_lsquare" (the reference's l(l+1)+m).
    ref_compat: None (correct transform: phi0 phase, alias fold, 2 pi), "fallback" or "raw"
    (reproduce sht_fallback / sht_raw conventions, for parity runs).
    phi0: per-ring phi0 (rings that are not a HEALPix grid); HEALPix grids use the HEALPix phi0.
    """
    mmax = lmax if mmax is None else mmax
    g = transforms.geometry_for(thetas, nphi_per_ring, weights_dz, phi0)
    alm = transforms.map2alm(rings, g, lmax, mmax, weights=weights_dz, precision=precision, ref_compat=ref_compat)
    if alm_layout == "ref_lsquare":
        alm = alm_ops.healpy_to_ref(alm, lmax, mmax)
    elif alm_layout != "healpy":
        raise ValueError("alm_layout must be 'healpy' or 'ref_lsquare'")
    ref = rings[0] if isinstance(rings, (list, tuple)) else rings
    return like_input(alm, ref)
