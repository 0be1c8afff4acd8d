"""Rotations of alm and maps, with the names of hellblast's rotate_alm.py, rotate_alm_euler.py,
wigner_fast.py / wigner_router.py and rotate.py.

``rotate_alm_euler(alm, alpha, beta, gamma)``: a'_{lm} = sum_{m'} exp(-i m alpha) d^l_{mm'}(beta)
exp(-i m' gamma) a_{lm'} (Euler ZYZ, the reference's convention, wigner_full.py:79-96), through
hb_rotate_alm (FP64, d^l by the three-term recursion in l; the reference's closed-form sum raises
cos and sin of beta/2 to the wrong powers, wigner_full.py:28-37, and is not a rotation).  The
reference's two variants (rotate_alm_euler_fast, rotate_alm_euler_risbo) compute the same map.
``rotate_alm_z`` (rotate_alm.py:5-19): a_{lm} exp(-i m alpha).  ``wigner_d_full(beta, l)``
(wigner_fast.py:15-25): the [B, 2l+1, 2l+1] matrices d^l_{mm'}(beta_b), m, m' = -l..l.
``rotate_map_z`` (rotate.py:5-25): a ring map turned about the z axis by delta_phi, as the
transform pair with the z rotation in between (the reference multiplies every FFT bin m,
including the ones that stand for negative frequencies, by exp(-i m delta)).
Alm are healpy-layout with mmax = lmax unless ``alm_layout="ref_lsquare"`` (the reference's
l(l+1)+m).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib as L
from . import alm_ops
from .util import as_tensor, like_input


def _to_healpy(alm, lmax, alm_layout):
    t = as_tensor(alm).to(torch.complex128)
    if alm_layout == "ref_lsquare":
        lmax = int(math.isqrt(t.shape[-1])) - 1 if lmax is None else lmax
        return alm_ops.ref_to_healpy(t, lmax, lmax), lmax
    if alm_layout != "healpy":
        raise ValueError("alm_layout must be 'healpy' or 'ref_lsquare'")
    lmax = alm_ops.getlmax(t.shape[-1]) if lmax is None else int(lmax)
    return t, lmax


def _from_healpy(t, lmax, alm_layout):
    return alm_ops.healpy_to_ref(t, lmax, lmax) if alm_layout == "ref_lsquare" else t


def rotate_alm_euler(alm, alpha, beta, gamma, lmax=None, *, alm_layout="healpy"):
    """[nalm] or [nmaps, nalm] complex alm rotated by Euler angles (ZYZ)."""
    t, lmax = _to_healpy(alm, lmax, alm_layout)
    squeeze = t.dim() == 1
    x = t.reshape(-1, t.shape[-1]).contiguous()
    if not x.is_cuda:
        raise ValueError("rotate_alm_euler needs CUDA tensors (there is no CPU path)")
    out = torch.empty_like(x)
    L.call("hb_rotate_alm", int(lmax), x.shape[0], x.data_ptr(), out.data_ptr(), float(alpha), float(beta),
           float(gamma), torch.cuda.current_stream(x.device).cuda_stream)
    out = _from_healpy(out, lmax, alm_layout)
    return like_input(out[0] if squeeze else out, alm)


rotate_alm_euler_fast = rotate_alm_euler
rotate_alm_euler_risbo = rotate_alm_euler


def rotate_alm_z(alm, alpha, lmax=None, *, alm_layout="healpy"):
    """a_{lm} exp(-i m alpha) (rotate_alm.py:5-19)."""
    t, lmax = _to_healpy(alm, lmax, alm_layout)
    m = alm_ops._m_of_index(lmax, lmax, str(t.device)).to(torch.float64)
    out = t * torch.exp(-1j * m * float(alpha))
    return like_input(_from_healpy(out, lmax, alm_layout), alm)


def wigner_d_full(beta, l: int, batch: int = 1):
    """d^l_{mm'}(beta_b) for m, m' = -l..l: [B, 2l+1, 2l+1] float64 (wigner_fast.py:15-25)."""
    b = as_tensor(beta, torch.float64).to(torch.float64).reshape(-1).contiguous()
    if not b.is_cuda:
        b = b.cuda()
    out = torch.empty(b.numel(), 2 * l + 1, 2 * l + 1, dtype=torch.float64, device=b.device)
    L.call("hb_wigner_d", int(l), b.numel(), b.data_ptr(), out.data_ptr(), torch.cuda.current_stream(b.device).cuda_stream)
    return out


def D_slice(alpha, beta, gamma, l, method="auto"):
    """D^l_{mm'}(alpha, beta, gamma) = exp(-i m alpha) d^l_{mm'}(beta) exp(-i m' gamma)
    (wigner_router.py:5-11)."""
    d = wigner_d_full([beta], l)[0].to(torch.complex128)
    m = torch.arange(-l, l + 1, dtype=torch.float64, device=d.device)
    return torch.exp(-1j * m[:, None] * alpha) * d * torch.exp(-1j * m[None, :] * gamma)


def rotate_map_z(m, delta_phi, lmax=None):
    """A RING map ([npix] or [nmaps, npix]) turned about the z axis by delta_phi: its alm
    times exp(-i m delta_phi), synthesised again (band-limited to lmax, default 3 nside - 1)."""
    from . import hp_compat
    t = as_tensor(m)
    nside = int(round((t.shape[-1] / 12) ** 0.5))
    lmax = 3 * nside - 1 if lmax is None else int(lmax)
    a = hp_compat.map2alm(t, lmax=lmax)
    a = rotate_alm_z(a, delta_phi, lmax=lmax).to(a.dtype)
    return like_input(hp_compat.alm2map(a, nside, lmax=lmax), m)
