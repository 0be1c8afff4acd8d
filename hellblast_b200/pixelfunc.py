"""HEALPix pixel indexing on the GPU (hb_ring2nest / hb_nest2ring / hb_pix2ang / hb_ang2pix /
hb_reorder in libhbsht.so), with healpy's names and the reference's.

healpy-style: ``ring2nest(nside, ipix)``, ``nest2ring``, ``pix2ang(nside, ipix, nest=False)``,
``ang2pix(nside, theta, phi, nest=False)``, ``pix2vec``, ``vec2pix``, ``reorder(map, r2n=True)``.
The reference's names: ``RingMapperGPU(nside).ang2pix / pix2ang`` (coords_ring.py:26-54, its
own RING conventions: the reference phi0 table and the z-edge ring lookup), ``vec2pix_ring_gpu``
(coords_ring.py:60-68), ``ang2pix_nest_gpu(theta, phi, nside)`` (nested_gpu.py:16-24),
``pix2ang_nest_gpu(nside, ipnest)`` and ``pix2vec_nest_analytic_gpu`` (nested_pix2ang.py:15-29),
``ring2nest_full`` / ``nest2ring_full`` (order_convert.py:8-34).  ``ang2pix_nest_gpu`` returns the
HEALPix NESTED pixel; the reference's kernel for it does not (its face numbering and polar
coordinate differ from HEALPix), so it has no bit-compatible counterpart here.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib as L
from .util import as_tensor, like_input


def _dev(x=None):
    if isinstance(x, torch.Tensor) and x.is_cuda:
        return x.device
    return torch.device("cuda", torch.cuda.current_device())


def _stream(dev):
    return torch.cuda.current_stream(dev).cuda_stream


def _check(bad: torch.Tensor, who: str):
    if int(bad.item()):
        raise ValueError(f"{who}: input outside the valid range (pixel index, or theta outside [0, pi])")


def _i64(x, dev):
    return as_tensor(x).to(device=dev, dtype=torch.int64).reshape(-1).contiguous()


def _f64(x, dev):
    return as_tensor(x, torch.float64).to(device=dev, dtype=torch.float64).reshape(-1).contiguous()


def ring2nest(nside: int, ipix):
    dev = _dev(ipix)
    p = _i64(ipix, dev)
    out = torch.empty_like(p)
    bad = torch.zeros(1, dtype=torch.int32, device=dev)
    L.call("hb_ring2nest", int(nside), p.numel(), p.data_ptr(), out.data_ptr(), bad.data_ptr(), _stream(dev))
    _check(bad, "ring2nest")
    return like_input(out.reshape(as_tensor(ipix).shape), ipix)


def nest2ring(nside: int, ipix):
    dev = _dev(ipix)
    p = _i64(ipix, dev)
    out = torch.empty_like(p)
    bad = torch.zeros(1, dtype=torch.int32, device=dev)
    L.call("hb_nest2ring", int(nside), p.numel(), p.data_ptr(), out.data_ptr(), bad.data_ptr(), _stream(dev))
    _check(bad, "nest2ring")
    return like_input(out.reshape(as_tensor(ipix).shape), ipix)


def _ref_tables(nside: int, dev):
    """The reference's phi0 and z_edges tables (ring_tables_healpix.cu) on the device."""
    from .ring_tables import HealpixRingTables
    t = HealpixRingTables(int(nside), phi0="reference", device=dev)
    return t.phi_center0.to(torch.float64).contiguous(), t.z_edges.to(torch.float64).contiguous()


def pix2ang(nside: int, ipix, nest: bool = False, *, ref_compat: bool = False):
    """(theta, phi) of pixel centres.  ``ref_compat`` (RING only): the reference's phi0 table and
    wrap (coords_ring.cu:47-53)."""
    dev = _dev(ipix)
    p = _i64(ipix, dev)
    th = torch.empty(p.numel(), dtype=torch.float64, device=dev)
    ph = torch.empty_like(th)
    bad = torch.zeros(1, dtype=torch.int32, device=dev)
    flags = (L.HB_PIX_NEST if nest else 0) | (L.HB_PIX_REFERENCE if ref_compat else 0)
    phi0 = _ref_tables(nside, dev)[0] if ref_compat else None
    L.call("hb_pix2ang", int(nside), flags, None if phi0 is None else phi0.data_ptr(), p.numel(), p.data_ptr(),
           th.data_ptr(), ph.data_ptr(), bad.data_ptr(), _stream(dev))
    _check(bad, "pix2ang")
    shape = as_tensor(ipix).shape
    return like_input(th.reshape(shape), ipix), like_input(ph.reshape(shape), ipix)


def ang2pix(nside: int, theta, phi, nest: bool = False, *, ref_compat: bool = False):
    """Pixel holding each direction.  ``ref_compat`` (RING only): the reference's z-edge ring
    lookup and nearest phi centre (coords_ring.py:18-24, coords_ring.cu:9-29)."""
    dev = _dev(theta)
    th = _f64(theta, dev)
    ph = _f64(phi, dev)
    if th.numel() != ph.numel():
        raise ValueError("theta and phi must have the same number of entries")
    out = torch.empty(th.numel(), dtype=torch.int64, device=dev)
    bad = torch.zeros(1, dtype=torch.int32, device=dev)
    flags = (L.HB_PIX_NEST if nest else 0) | (L.HB_PIX_REFERENCE if ref_compat else 0)
    phi0, zed = _ref_tables(nside, dev) if ref_compat else (None, None)
    L.call("hb_ang2pix", int(nside), flags, None if zed is None else zed.data_ptr(),
           None if phi0 is None else phi0.data_ptr(), th.numel(), th.data_ptr(), ph.data_ptr(), out.data_ptr(),
           bad.data_ptr(), _stream(dev))
    _check(bad, "ang2pix")
    return like_input(out.reshape(as_tensor(theta).shape), theta)


def pix2vec(nside: int, ipix, nest: bool = False):
    th, ph = pix2ang(nside, ipix, nest)
    th, ph = as_tensor(th), as_tensor(ph)
    st = torch.sin(th)
    return like_input(st * torch.cos(ph), ipix), like_input(st * torch.sin(ph), ipix), like_input(torch.cos(th), ipix)


def vec2pix(nside: int, x, y, z, nest: bool = False):
    x, y, z = (as_tensor(v, torch.float64).to(torch.float64) for v in (x, y, z))
    r = torch.sqrt(x * x + y * y + z * z)
    th = torch.acos(torch.clamp(z / r, -1.0, 1.0))
    ph = torch.atan2(y, x)
    return ang2pix(nside, th, ph, nest)


def reorder(map_in, r2n: bool = False, n2r: bool = False):
    """RING -> NESTED (r2n) or NESTED -> RING (n2r) reordering of [npix] or [nmaps, npix] maps."""
    if r2n == n2r:
        raise ValueError("give exactly one of r2n, n2r")
    t = as_tensor(map_in)
    dev = _dev(t)
    squeeze = t.dim() == 1
    x = t.reshape(-1, t.shape[-1]).to(dev)
    if x.dtype not in (torch.float32, torch.float64):
        x = x.to(torch.float64)
    x = x.contiguous()
    npix = x.shape[-1]
    nside = int(round((npix / 12) ** 0.5))
    if 12 * nside * nside != npix:
        raise ValueError("map length is not 12 nside^2")
    out = torch.empty_like(x)
    L.call("hb_reorder", nside, 1 if r2n else 0, 32 if x.dtype == torch.float32 else 64, x.shape[0], x.data_ptr(),
           out.data_ptr(), _stream(dev))
    return like_input(out[0] if squeeze else out, map_in)


# ----------------------------------------------------------------------------- reference names
class RingMapperGPU:
    """coords_ring.py:26-57: RING ang2pix / pix2ang in the reference's conventions."""

    def __init__(self, nside: int):
        from .ring_tables import HealpixRingTables
        self.nside = int(nside)
        self.tables = HealpixRingTables(self.nside, phi0="reference")

    def ang2pix(self, theta, phi):
        return ang2pix(self.nside, theta, phi, ref_compat=True)

    def pix2ang(self, ipix):
        return pix2ang(self.nside, ipix, ref_compat=True)

    def weights_dz(self):
        return self.tables.weights_dz()


def vec2pix_ring_gpu(x, y, z, mapper: RingMapperGPU):
    """coords_ring.py:60-68."""
    x, y, z = (as_tensor(v, torch.float64).to(torch.float64) for v in (x, y, z))
    th = torch.acos(torch.clamp(z, -1.0, 1.0))
    ph = torch.atan2(y, x)
    ph = torch.where(ph < 0, ph + 2 * np.pi, ph)
    return mapper.ang2pix(th, ph)


def ang2pix_nest_gpu(theta, phi, nside: int):
    """nested_gpu.py:16-24 (argument order theta, phi, nside), HEALPix NESTED index."""
    return ang2pix(nside, theta, phi, nest=True)


def pix2ang_nest_gpu(nside: int, ipnest):
    """nested_pix2ang.py:15-23."""
    return pix2ang(nside, ipnest, nest=True)


def pix2vec_nest_analytic_gpu(nside: int, ipnest):
    """nested_pix2ang.py:25-29."""
    return pix2vec(nside, ipnest, nest=True)


def ring2nest_full(m_ring, nside: int):
    """order_convert.py:8-23: a RING map reordered to NESTED."""
    return reorder(m_ring, r2n=True)


def nest2ring_full(m_nest, nside: int):
    """order_convert.py:25-34: a NESTED map reordered to RING."""
    return reorder(m_nest, n2r=True)
