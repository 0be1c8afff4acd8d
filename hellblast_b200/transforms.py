"""Transform drivers shared by the hellblast-compatible entry points.

Every function here ends in one torch.ops.hb call (or two), i.e. in the CUDA kernels of
libhbsht.so; nothing computes on the host.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib as L
from . import geometry as G
from . import ops
from .util import as_tensor, flatten_rings, host_array

REF_COMPAT = {
    None: 0,
    # sht_fallback.py:36-65: no phi0 phase, no alias fold (bins m >= nphi read as 0)
    "fallback": L.HB_F_NOPHASE | L.HB_F_NOFOLD,
    # sht_raw.py:30-57: additionally no 2*pi (and m cut at max(nphi)/2, applied after the call)
    "raw": L.HB_F_NOPHASE | L.HB_F_NOFOLD | L.HB_F_NO2PI,
}


def resolve_precision(precision, dtype: torch.dtype) -> torch.dtype:
    """'fp32'/'fp64'/None (follow the input) -> the real dtype the kernels compute in."""
    if precision in ("fp32", "float32", 32, torch.float32):
        return torch.float32
    if precision in ("fp64", "float64", 64, torch.float64):
        return torch.float64
    if precision is None:
        return torch.float32 if dtype in (torch.float32, torch.complex64) else torch.float64
    raise ValueError(f"unknown precision {precision!r}")


def geometry_for(thetas, nphi, weights=None, phi0=None, phi0_mode="healpix"):
    """Geometry for the reference's (thetas, nphi_per_ring, weights) arguments: the HEALPix
    geometry when the rings form a HEALPix grid (phi0 per ``phi0_mode``), else a generic one."""
    th = host_array(thetas, np.float64)
    nphi_h = host_array(nphi, np.int64)
    nside = G.detect_healpix(th, nphi_h) if phi0 is None else 0
    if nside:
        return G.healpix(nside, phi0=phi0_mode)
    w = np.zeros_like(th) if weights is None else host_array(weights, np.float64)
    return G.generic(th, nphi_h.astype(np.int32), w, phi0=None if phi0 is None else host_array(phi0, np.float64))


def device_weights(weights, g: G.Geometry, device) -> torch.Tensor | None:
    if weights is None:
        return None
    return as_tensor(weights, torch.float64).reshape(-1).contiguous().to(device)


def map2alm(maps, g: G.Geometry, lmax: int, mmax: int | None = None, weights=None, precision=None,
            ref_compat=None) -> torch.Tensor:
    """maps: flat [npix] or [nmaps, npix] -> alm [nalm] / [nmaps, nalm] (healpy layout)."""
    mmax = lmax if mmax is None else mmax
    t = flatten_rings(maps) if isinstance(maps, (list, tuple)) else as_tensor(maps)
    rt = resolve_precision(precision, t.dtype)
    squeeze = t.dim() == 1
    t = t.reshape(-1, g.npix).to(rt).contiguous()
    if ref_compat not in REF_COMPAT:
        raise ValueError("ref_compat must be None, 'fallback' or 'raw'")
    p = G.plan(g, lmax, mmax, precision=32 if rt == torch.float32 else 64)
    alm = ops.map2alm(t, p.pid, device_weights(weights, g, t.device), REF_COMPAT[ref_compat])
    if ref_compat == "raw":
        mcut = min(mmax, int(np.max(g.nphi)) // 2)  # sht_raw.py:43 mmax_eff
        if mcut < mmax:
            alm[:, ops.alm_size(lmax, mcut):] = 0
    return alm[0] if squeeze else alm


def alm2map(alm, g: G.Geometry, lmax: int, mmax: int | None = None, precision=None, ref_compat=None):
    mmax = lmax if mmax is None else mmax
    t = as_tensor(alm)
    rt = resolve_precision(precision, t.dtype)
    ct = torch.complex64 if rt == torch.float32 else torch.complex128
    squeeze = t.dim() == 1
    t = t.reshape(-1, t.shape[-1]).to(ct).contiguous()
    if t.shape[-1] != ops.alm_size(lmax, mmax):
        raise ValueError(f"alm has {t.shape[-1]} entries, expected {ops.alm_size(lmax, mmax)} for "
                         f"lmax={lmax}, mmax={mmax}")
    flags = L.HB_F_NOPHASE if ref_compat else 0
    p = G.plan(g, lmax, mmax, precision=32 if rt == torch.float32 else 64)
    out = ops.alm2map(t, p.pid, flags)
    return out[0] if squeeze else out


def map2alm_spin2(Q, U, g: G.Geometry, lmax: int, mmax: int | None = None, weights=None, precision=None,
                  ref_compat=False):
    """(Q, U) -> (E, B), healpy layout.  ``ref_compat=True`` reproduces the conventions of the
    reference's map2alm_spin_gpu / eb_from_qu_gpu (spin.py:43-78) with the Wigner d it intends:
    no phi0 phase, bins m >= nphi_r dropped instead of folded, orders above
    max_r min(mmax, nphi_r // 2) zero (spin.py:53,57,65), and its spin functions
    sqrt((2l+1)/4pi) d^l_{m,+-2} for a(+-2) (spin.py:29,58-59), where healpy's are d^l_{m,-+2}.
    That last difference is the U -> -U (and B -> -B) change of polarisation convention:
    E_ref(Q, U) = E(Q, -U), B_ref(Q, U) = -B(Q, -U)."""
    mmax = lmax if mmax is None else mmax
    q = flatten_rings(Q) if isinstance(Q, (list, tuple)) else as_tensor(Q)
    u = flatten_rings(U) if isinstance(U, (list, tuple)) else as_tensor(U)
    rt = resolve_precision(precision, q.dtype)
    squeeze = q.dim() == 1
    q = q.reshape(-1, g.npix).to(rt).contiguous()
    u = u.reshape(-1, g.npix).to(rt).contiguous()
    p = G.plan(g, lmax, mmax, precision=32 if rt == torch.float32 else 64, spin=True)
    flags = (L.HB_F_NOPHASE | L.HB_F_NOFOLD) if ref_compat else 0
    E, B = ops.map2alm_spin2(q, -u if ref_compat else u, p.pid, device_weights(weights, g, q.device), flags)
    if ref_compat:
        B = -B
        mcut = min(mmax, int(np.max(g.nphi)) // 2)  # spin.py:53 mmax_eff
        if mcut < mmax:
            E[:, ops.alm_size(lmax, mcut):] = 0
            B[:, ops.alm_size(lmax, mcut):] = 0
    return (E[0], B[0]) if squeeze else (E, B)


def alm2map_spin2(E, B, g: G.Geometry, lmax: int, mmax: int | None = None, precision=None, ref_compat=False):
    """(E, B) -> (Q, U).  ``ref_compat=True`` follows the reference's qu_from_eb_gpu
    (spin.py:80-115): no phi0 phase and its a(+2) = -(E - iB), which with its d^l_{m,+-2} spin
    functions gives Q_ref = Q, U_ref = -U of the healpy convention.  (The reference's synthesis
    is right for m = 0 input only: for m > 0 it fills the complex spin field's spectrum as if it
    were real, spin.py:104,106.)"""
    mmax = lmax if mmax is None else mmax
    e = as_tensor(E)
    b = as_tensor(B)
    rt = resolve_precision(precision, e.dtype)
    ct = torch.complex64 if rt == torch.float32 else torch.complex128
    squeeze = e.dim() == 1
    e = e.reshape(-1, e.shape[-1]).to(ct).contiguous()
    b = b.reshape(-1, b.shape[-1]).to(ct).contiguous()
    p = G.plan(g, lmax, mmax, precision=32 if rt == torch.float32 else 64, spin=True)
    Q, U = ops.alm2map_spin2(e, b, p.pid, L.HB_F_NOPHASE if ref_compat else 0)
    if ref_compat:
        U = -U
    return (Q[0], U[0]) if squeeze else (Q, U)


def split_rings(flat: torch.Tensor, g: G.Geometry) -> list:
    """Flat RING map -> list of per-ring views (the reference's ring-list form)."""
    rs = g.ring_start
    return [flat[..., int(rs[r]):int(rs[r + 1])] for r in range(g.nr)]


def nside_from_npix(npix: int) -> int:
    nside = int(math.isqrt(npix // 12))
    if 12 * nside * nside != npix:
        raise ValueError("npix is not 12*nside^2")
    return nside
