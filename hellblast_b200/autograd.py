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
    def forward(ctx, maps, pid, weights):
        ctx.save_for_backward(weights)
        ctx.pid = pid
        return ops.map2alm(maps, pid, weights, 0)

    @staticmethod
    def backward(ctx, galm):
        (weights,) = ctx.saved_tensors
        return ops.map2alm_adjoint(galm.contiguous(), ctx.pid, weights, 0), None, None


class Alm2Map(torch.autograd.Function):
    @staticmethod
    def forward(ctx, alm, pid):
        ctx.pid = pid
        return ops.alm2map(alm, pid, 0)

    @staticmethod
    def backward(ctx, gmap):
        return ops.alm2map_adjoint(gmap.contiguous(), ctx.pid, 0), None


class Map2AlmSpin2(torch.autograd.Function):
    @staticmethod
    def forward(ctx, Q, U, pid, weights):
        ctx.save_for_backward(weights)
        ctx.pid = pid
        return ops.map2alm_spin2(Q, U, pid, weights, 0)

    @staticmethod
    def backward(ctx, gE, gB):
        (weights,) = ctx.saved_tensors
        gE = gE.contiguous()
        gB = gB.contiguous()
        gQ, gU = ops.map2alm_spin2_adjoint(gE, gB, ctx.pid, weights, 0)
        return gQ, gU, None, None


class Alm2MapSpin2(torch.autograd.Function):
    @staticmethod
    def forward(ctx, E, B, pid):
        ctx.pid = pid
        return ops.alm2map_spin2(E, B, pid, 0)

    @staticmethod
    def backward(ctx, gQ, gU):
        gE, gB = ops.alm2map_spin2_adjoint(gQ.contiguous(), gU.contiguous(), ctx.pid, 0)
        return gE, gB, None


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


def _prec(t: torch.Tensor) -> int:
    return 32 if t.dtype in (torch.float32, torch.complex64) else 64


def map2alm(maps: torch.Tensor, nside: int, lmax: int, mmax: int | None = None, weights="dz") -> torch.Tensor:
    """Differentiable map2alm on a HEALPix grid; maps [nmaps, npix] (float32 or float64)."""
    g = G.healpix(nside, weights="uniform" if weights == "uniform" else "dz")
    w = None if isinstance(weights, str) else device_weights(weights, g, maps.device)
    p = G.plan(g, lmax, mmax, precision=_prec(maps))
    return Map2Alm.apply(maps.contiguous(), p.pid, w)


def alm2map(alm: torch.Tensor, nside: int, lmax: int, mmax: int | None = None) -> torch.Tensor:
    p = G.plan(G.healpix(nside), lmax, mmax, precision=_prec(alm))
    return Alm2Map.apply(alm.contiguous(), p.pid)


def map2alm_spin(Q: torch.Tensor, U: torch.Tensor, nside: int, lmax: int, mmax: int | None = None, weights="dz"):
    g = G.healpix(nside, weights="uniform" if weights == "uniform" else "dz")
    w = None if isinstance(weights, str) else device_weights(weights, g, Q.device)
    p = G.plan(g, lmax, mmax, precision=_prec(Q), spin=True)
    return Map2AlmSpin2.apply(Q.contiguous(), U.contiguous(), p.pid, w)


def alm2map_spin(E: torch.Tensor, B: torch.Tensor, nside: int, lmax: int, mmax: int | None = None):
    p = G.plan(G.healpix(nside), lmax, mmax, precision=_prec(E), spin=True)
    return Alm2MapSpin2.apply(E.contiguous(), B.contiguous(), p.pid)


def alm2cl(alm: torch.Tensor, lmax: int, mmax: int | None = None) -> torch.Tensor:
    mmax = lmax if mmax is None else mmax
    return Alm2Cl.apply(alm.contiguous(), lmax, mmax)
