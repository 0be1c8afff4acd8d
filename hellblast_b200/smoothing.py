"""Beam smoothing: map2alm -> almxfl -> alm2map, the main consumer of the transforms in the
reference (smoothing.py:5-15, beams.py:5-47 of hellblast), with its names and conventions.

For batches of float32 maps the filter is applied inside the tensor-core analysis kernel's alm
store (``hb_batched_map2alm_fl``), so a smoothed batch costs one batched map2alm and one batched
alm2map and no separate pass over the alm.
"""
from __future__ import annotations

import math

import torch

from . import alm_ops, batched, hp_compat
from .util import as_tensor, like_input


def gaussian_beam_fl(lmax: int, fwhm_rad: float, device=None) -> torch.Tensor:
    """b_l = exp(-l(l+1) sigma^2 / 2), sigma = fwhm / sqrt(8 ln 2) (smoothing.py:5-10)."""
    sigma = fwhm_rad / math.sqrt(8.0 * math.log(2.0))
    dev = torch.device("cuda") if device is None else torch.device(device)
    ell = torch.arange(lmax + 1, dtype=torch.float64, device=dev)
    return torch.exp(-0.5 * ell * (ell + 1.0) * sigma * sigma)


def pixel_window_fl(nside: int, lmax: int, pol: bool = False, device=None):
    """HEALPix pixel window p_l.  Like the reference without healpy (beams.py:6-21), this
    returns ones: the tabulated windows are not part of this library."""
    dev = torch.device("cuda") if device is None else torch.device(device)
    one = torch.ones(lmax + 1, dtype=torch.float64, device=dev)
    return (one, one.clone()) if pol else (one, None)


def smooth_alm_gaussian(alm, fwhm_rad: float, lmax: int | None = None):
    """alm * b_l for a Gaussian beam (smoothing.py:12-15), healpy layout."""
    t = as_tensor(alm)
    lmax = alm_ops.getlmax(t.shape[-1]) if lmax is None else lmax
    return alm_ops.almxfl(alm, gaussian_beam_fl(lmax, fwhm_rad, t.device), lmax=lmax)


def beam_filter(lmax: int, fwhm=None, bl=None, pixwin=None, device=None) -> torch.Tensor:
    """F_l = b_l * pixwin_l (beams.py:23-37): ``bl`` if given, else the Gaussian of ``fwhm``."""
    dev = torch.device("cuda") if device is None else torch.device(device)
    fl = torch.ones(lmax + 1, dtype=torch.float64, device=dev)
    if bl is not None:
        fl = fl * torch.as_tensor(bl, dtype=torch.float64, device=dev)[: lmax + 1]
    elif fwhm is not None:
        fl = fl * gaussian_beam_fl(lmax, fwhm, dev)
    if pixwin is not None:
        fl = fl * torch.as_tensor(pixwin, dtype=torch.float64, device=dev)[: lmax + 1]
    return fl


def smooth_alm_with_beam(alm, lmax: int, fwhm=None, bl=None, pixwin=None):
    t = as_tensor(alm)
    return alm_ops.almxfl(alm, beam_filter(lmax, fwhm, bl, pixwin, t.device), lmax=lmax)


def smooth_map(m, nside: int, lmax: int | None = None, fwhm=None, bl=None, use_pixel_window: bool = True,
               nest: bool = False):
    """Smoothed RING map(s) (beams.py:38-47).  ``m``: [npix] or [nmaps, npix]; float32 batches of
    two or more maps run the tensor-core path with the filter fused into map2alm."""
    t = as_tensor(m)
    lmax = 3 * int(nside) if lmax is None else int(lmax)
    pw = pixel_window_fl(int(nside), lmax, device=t.device)[0] if use_pixel_window else None
    fl = beam_filter(lmax, fwhm, bl, pw, t.device)
    if t.dim() == 2 and t.shape[0] > 1 and t.dtype == torch.float32:
        bp = batched.plan(int(nside), lmax, t.shape[0])
        alm = bp.map2alm(t, fl=fl.float())
        return like_input(bp.alm2map(alm).reshape(t.shape), m)
    alm = hp_compat.map2alm(t, lmax=lmax, nest=nest)
    alm = alm_ops.almxfl(alm, fl.to(alm.real.dtype), lmax=lmax)
    return like_input(hp_compat.alm2map(alm, int(nside), lmax=lmax, nest=nest), m)
