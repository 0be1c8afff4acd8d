"""Differentiable transforms: torch.autograd.Function wrappers whose backward passes call the
hand-written adjoint kernels (exact transposes; lambda is recomputed, never stored).

Gradients of complex alm follow PyTorch's convention for a real loss L:
grad = dL/dRe(a) + i dL/dIm(a).  The m = 0 imaginary parts do not enter a real map, so their
gradient through alm2map is zero.
"""
from __future__ import annotations

import torch

from . import alm_ops, ops
from . import geometry as G
from .transforms import device_weights


class Map2Alm(torch.autograd.Function):
    @staticmethod
    def forward(ctx, maps, gid, lmax, mmax, weights):
        ctx.save_for_backward(weights)
        ctx.cfg = (gid, lmax, mmax)
        return ops.map2alm(maps, gid, lmax, mmax, weights, 0)

    @staticmethod
    def backward(ctx, galm):
        (weights,) = ctx.saved_tensors
        gid, lmax, mmax = ctx.cfg
        gm = ops.map2alm_adjoint(galm.contiguous(), gid, lmax, mmax, weights, 0)
        return gm, None, None, None, None


class Alm2Map(torch.autograd.Function):
    @staticmethod
    def forward(ctx, alm, gid, lmax, mmax):
        ctx.cfg = (gid, lmax, mmax)
        return ops.alm2map(alm, gid, lmax, mmax, 0)

    @staticmethod
    def backward(ctx, gmap):
        gid, lmax, mmax = ctx.cfg
        return ops.alm2map_adjoint(gmap.contiguous(), gid, lmax, mmax, 0), None, None, None


class Map2AlmSpin2(torch.autograd.Function):
    @staticmethod
    def forward(ctx, Q, U, gid, lmax, mmax, weights):
        ctx.save_for_backward(weights)
        ctx.cfg = (gid, lmax, mmax)
        return ops.map2alm_spin2(Q, U, gid, lmax, mmax, weights, 0)

    @staticmethod
    def backward(ctx, gE, gB):
        (weights,) = ctx.saved_tensors
        gid, lmax, mmax = ctx.cfg
        gE = torch.zeros_like(gE) if gE is None else gE.contiguous()
        gB = torch.zeros_like(gB) if gB is None else gB.contiguous()
        gQ, gU = ops.map2alm_spin2_adjoint(gE, gB, gid, lmax, mmax, weights, 0)
        return gQ, gU, None, None, None, None


class Alm2MapSpin2(torch.autograd.Function):
    @staticmethod
    def forward(ctx, E, B, gid, lmax, mmax):
        ctx.cfg = (gid, lmax, mmax)
        return ops.alm2map_spin2(E, B, gid, lmax, mmax, 0)

    @staticmethod
    def backward(ctx, gQ, gU):
        gid, lmax, mmax = ctx.cfg
        gQ = torch.zeros_like(gQ) if gQ is None else gQ.contiguous()
        gU = torch.zeros_like(gU) if gU is None else gU.contiguous()
        gE, gB = ops.alm2map_spin2_adjoint(gQ, gU, gid, lmax, mmax, 0)
        return gE, gB, None, None, None


class Alm2Cl(torch.autograd.Function):
    """C_l = (|a_l0|^2 + 2 sum_{m>0} |a_lm|^2)/(2l+1); dC_l/da = 2 c_m a/(2l+1) (c_0 = 1, c_m = 2)."""

    @staticmethod
    def forward(ctx, alm, lmax, mmax):
        ctx.save_for_backward(alm)
        ctx.cfg = (lmax, mmax)
        return ops.alm2cl(alm, None, lmax, mmax)

    @staticmethod
    def backward(ctx, gcl):
        (alm,) = ctx.saved_tensors
        lmax, mmax = ctx.cfg
        dev = str(alm.device)
        l_of = alm_ops._l_of_index(lmax, mmax, dev)
        m_of = alm_ops._m_of_index(lmax, mmax, dev)
        rt = torch.float32 if alm.dtype == torch.complex64 else torch.float64
        cm = torch.where(m_of > 0, 2.0, 1.0).to(rt)
        fac = (2.0 * cm / (2.0 * l_of.to(rt) + 1.0))
        w = gcl.to(rt)[:, l_of] * fac
        return alm * w, None, None


def map2alm(maps: torch.Tensor, nside: int, lmax: int, mmax: int | None = None, weights="dz") -> torch.Tensor:
    """Differentiable map2alm on a HEALPix grid; maps [nmaps, npix] (float32 or float64)."""
    mmax = lmax if mmax is None else mmax
    g = G.healpix(nside, weights="uniform" if weights == "uniform" else "dz")
    w = None if isinstance(weights, str) else device_weights(weights, g, maps.device)
    return Map2Alm.apply(maps.contiguous(), g.gid, lmax, mmax, w)


def alm2map(alm: torch.Tensor, nside: int, lmax: int, mmax: int | None = None) -> torch.Tensor:
    mmax = lmax if mmax is None else mmax
    return Alm2Map.apply(alm.contiguous(), G.healpix(nside).gid, lmax, mmax)


def map2alm_spin(Q: torch.Tensor, U: torch.Tensor, nside: int, lmax: int, mmax: int | None = None, weights="dz"):
    mmax = lmax if mmax is None else mmax
    g = G.healpix(nside, weights="uniform" if weights == "uniform" else "dz")
    w = None if isinstance(weights, str) else device_weights(weights, g, Q.device)
    return Map2AlmSpin2.apply(Q.contiguous(), U.contiguous(), g.gid, lmax, mmax, w)


def alm2map_spin(E: torch.Tensor, B: torch.Tensor, nside: int, lmax: int, mmax: int | None = None):
    mmax = lmax if mmax is None else mmax
    return Alm2MapSpin2.apply(E.contiguous(), B.contiguous(), G.healpix(nside).gid, lmax, mmax)


def alm2cl(alm: torch.Tensor, lmax: int, mmax: int | None = None) -> torch.Tensor:
    mmax = lmax if mmax is None else mmax
    return Alm2Cl.apply(alm.contiguous(), lmax, mmax)
