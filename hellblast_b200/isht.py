"""Inverse scalar SHT with the signature of hellblast's ``alm2map_gpu`` (isht.py:5)."""
from __future__ import annotations

import torch

from . import alm_ops, transforms
from .util import as_tensor, like_input


def alm2map_gpu(alm, thetas, nphi_per_ring, lmax, mmax=None, dtype=None, *, alm_layout="healpy", flat=False,
                precision=None, phi0=None, ref_compat=None):
    """f(pix) = sum_lm a_lm Y_lm(pix) for a real field.  Returns a list of per-ring tensors
    like the reference (isht.py:14-26), or the flat RING map with ``flat=True``.
    dtype: output dtype (the reference's default is float64)."""
    mmax = lmax if mmax is None else mmax
    a = as_tensor(alm)
    if alm_layout == "ref_lsquare":
        a = alm_ops.ref_to_healpy(a, lmax, mmax)
    elif alm_layout != "healpy":
        raise ValueError("alm_layout must be 'healpy' or 'ref_lsquare'")
    g = transforms.geometry_for(thetas, nphi_per_ring, None, phi0)
    out = transforms.alm2map(a, g, lmax, mmax, precision=precision, ref_compat=ref_compat)
    if dtype is not None:
        out = out.to(torch.empty(0, dtype=dtype).dtype if not isinstance(dtype, torch.dtype) else dtype)
    if flat:
        return like_input(out, alm)
    return [like_input(r, alm) for r in transforms.split_rings(out, g)]
