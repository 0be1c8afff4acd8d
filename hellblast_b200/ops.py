"""The C ABI exposed as PyTorch custom ops (``torch.ops.hb.*``): CUDA tensors in and out, the
caller's current stream, workspace from torch's caching allocator.  Plans (geometry + lmax +
mmax + FP32 recursion checkpoints) are passed as integer ids (see geometry.py)."""
from __future__ import annotations

from typing import Optional

import torch

from . import _lib as L
from . import geometry as G


def alm_size(lmax: int, mmax: int) -> int:
    return mmax * (2 * lmax + 1 - mmax) // 2 + lmax + 1


def _prec(dtype: torch.dtype) -> int:
    if dtype in (torch.float32, torch.complex64):
        return 32
    if dtype in (torch.float64, torch.complex128):
        return 64
    raise TypeError(f"unsupported dtype {dtype}")


def _stream(dev: torch.device) -> int:
    return torch.cuda.current_stream(dev).cuda_stream


def _check_cuda(*ts):
    for t in ts:
        if t is not None and not t.is_cuda:
            raise ValueError("hellblast_b200 ops take CUDA tensors (no CPU path exists)")


def _ws(p: G.Plan, prec, nmaps, dev, spin=False):
    n = p.workspace_bytes(prec, nmaps, spin)
    return torch.empty(max(n, 1), dtype=torch.uint8, device=dev)


def _wptr(w: Optional[torch.Tensor]) -> Optional[int]:
    if w is None:
        return None
    if w.dtype != torch.float64 or not w.is_contiguous():
        raise ValueError("weights must be a contiguous float64 CUDA tensor")
    return w.data_ptr()


def _ctype(prec):
    return torch.complex64 if prec == 32 else torch.complex128


def _rtype(prec):
    return torch.float32 if prec == 32 else torch.float64


@torch.library.custom_op("hb::map2alm", mutates_args=())
def map2alm(maps: torch.Tensor, pid: int, weights: Optional[torch.Tensor], flags: int) -> torch.Tensor:
    _check_cuda(maps, weights)
    p = G.get_plan(pid)
    maps = maps.contiguous()
    nmaps, prec = maps.shape[0], _prec(maps.dtype)
    out = torch.empty(nmaps, alm_size(p.lmax, p.mmax), dtype=_ctype(prec), device=maps.device)
    ws = _ws(p, prec, nmaps, maps.device)
    L.call(f"hb_map2alm_f{prec}", p.handle, nmaps, maps.data_ptr(), _wptr(weights), out.data_ptr(), ws.data_ptr(),
           ws.numel(), flags, _stream(maps.device))
    return out


@map2alm.register_fake
def _(maps, pid, weights, flags):
    p = G.get_plan(pid)
    return maps.new_empty((maps.shape[0], alm_size(p.lmax, p.mmax)), dtype=_ctype(_prec(maps.dtype)))


@torch.library.custom_op("hb::alm2map", mutates_args=())
def alm2map(alm: torch.Tensor, pid: int, flags: int) -> torch.Tensor:
    _check_cuda(alm)
    p = G.get_plan(pid)
    alm = alm.contiguous()
    nmaps, prec = alm.shape[0], _prec(alm.dtype)
    out = torch.empty(nmaps, p.npix, dtype=_rtype(prec), device=alm.device)
    ws = _ws(p, prec, nmaps, alm.device)
    L.call(f"hb_alm2map_f{prec}", p.handle, nmaps, alm.data_ptr(), out.data_ptr(), ws.data_ptr(), ws.numel(), flags,
           _stream(alm.device))
    return out


@alm2map.register_fake
def _(alm, pid, flags):
    return alm.new_empty((alm.shape[0], G.get_plan(pid).npix), dtype=_rtype(_prec(alm.dtype)))


@torch.library.custom_op("hb::alm2map_adjoint", mutates_args=())
def alm2map_adjoint(maps: torch.Tensor, pid: int, flags: int) -> torch.Tensor:
    _check_cuda(maps)
    p = G.get_plan(pid)
    maps = maps.contiguous()
    nmaps, prec = maps.shape[0], _prec(maps.dtype)
    out = torch.empty(nmaps, alm_size(p.lmax, p.mmax), dtype=_ctype(prec), device=maps.device)
    ws = _ws(p, prec, nmaps, maps.device)
    L.call(f"hb_alm2map_adjoint_f{prec}", p.handle, nmaps, maps.data_ptr(), out.data_ptr(), ws.data_ptr(),
           ws.numel(), flags, _stream(maps.device))
    return out


@alm2map_adjoint.register_fake
def _(maps, pid, flags):
    p = G.get_plan(pid)
    return maps.new_empty((maps.shape[0], alm_size(p.lmax, p.mmax)), dtype=_ctype(_prec(maps.dtype)))


@torch.library.custom_op("hb::map2alm_adjoint", mutates_args=())
def map2alm_adjoint(alm: torch.Tensor, pid: int, weights: Optional[torch.Tensor], flags: int) -> torch.Tensor:
    _check_cuda(alm, weights)
    p = G.get_plan(pid)
    alm = alm.contiguous()
    nmaps, prec = alm.shape[0], _prec(alm.dtype)
    out = torch.empty(nmaps, p.npix, dtype=_rtype(prec), device=alm.device)
    ws = _ws(p, prec, nmaps, alm.device)
    L.call(f"hb_map2alm_adjoint_f{prec}", p.handle, nmaps, alm.data_ptr(), _wptr(weights), out.data_ptr(),
           ws.data_ptr(), ws.numel(), flags, _stream(alm.device))
    return out


@map2alm_adjoint.register_fake
def _(alm, pid, weights, flags):
    return alm.new_empty((alm.shape[0], G.get_plan(pid).npix), dtype=_rtype(_prec(alm.dtype)))


@torch.library.custom_op("hb::map2alm_spin2", mutates_args=())
def map2alm_spin2(Q: torch.Tensor, U: torch.Tensor, pid: int, weights: Optional[torch.Tensor],
                  flags: int) -> tuple[torch.Tensor, torch.Tensor]:
    _check_cuda(Q, U, weights)
    p = G.get_plan(pid)
    Q, U = Q.contiguous(), U.contiguous()
    nmaps, prec = Q.shape[0], _prec(Q.dtype)
    E = torch.empty(nmaps, alm_size(p.lmax, p.mmax), dtype=_ctype(prec), device=Q.device)
    B = torch.empty_like(E)
    ws = _ws(p, prec, nmaps, Q.device, spin=True)
    L.call(f"hb_map2alm_spin2_f{prec}", p.handle, nmaps, Q.data_ptr(), U.data_ptr(), _wptr(weights), E.data_ptr(),
           B.data_ptr(), ws.data_ptr(), ws.numel(), flags, _stream(Q.device))
    return E, B


@map2alm_spin2.register_fake
def _(Q, U, pid, weights, flags):
    p = G.get_plan(pid)
    e = Q.new_empty((Q.shape[0], alm_size(p.lmax, p.mmax)), dtype=_ctype(_prec(Q.dtype)))
    return e, torch.empty_like(e)


@torch.library.custom_op("hb::alm2map_spin2", mutates_args=())
def alm2map_spin2(E: torch.Tensor, B: torch.Tensor, pid: int, flags: int) -> tuple[torch.Tensor, torch.Tensor]:
    _check_cuda(E, B)
    p = G.get_plan(pid)
    E, B = E.contiguous(), B.contiguous()
    nmaps, prec = E.shape[0], _prec(E.dtype)
    Q = torch.empty(nmaps, p.npix, dtype=_rtype(prec), device=E.device)
    U = torch.empty_like(Q)
    ws = _ws(p, prec, nmaps, E.device, spin=True)
    L.call(f"hb_alm2map_spin2_f{prec}", p.handle, nmaps, E.data_ptr(), B.data_ptr(), Q.data_ptr(), U.data_ptr(),
           ws.data_ptr(), ws.numel(), flags, _stream(E.device))
    return Q, U


@alm2map_spin2.register_fake
def _(E, B, pid, flags):
    q = E.new_empty((E.shape[0], G.get_plan(pid).npix), dtype=_rtype(_prec(E.dtype)))
    return q, torch.empty_like(q)


@torch.library.custom_op("hb::alm2map_spin2_adjoint", mutates_args=())
def alm2map_spin2_adjoint(gQ: torch.Tensor, gU: torch.Tensor, pid: int,
                          flags: int) -> tuple[torch.Tensor, torch.Tensor]:
    _check_cuda(gQ, gU)
    p = G.get_plan(pid)
    gQ, gU = gQ.contiguous(), gU.contiguous()
    nmaps, prec = gQ.shape[0], _prec(gQ.dtype)
    gE = torch.empty(nmaps, alm_size(p.lmax, p.mmax), dtype=_ctype(prec), device=gQ.device)
    gB = torch.empty_like(gE)
    ws = _ws(p, prec, nmaps, gQ.device, spin=True)
    L.call(f"hb_alm2map_spin2_adjoint_f{prec}", p.handle, nmaps, gQ.data_ptr(), gU.data_ptr(), gE.data_ptr(),
           gB.data_ptr(), ws.data_ptr(), ws.numel(), flags, _stream(gQ.device))
    return gE, gB


@alm2map_spin2_adjoint.register_fake
def _(gQ, gU, pid, flags):
    p = G.get_plan(pid)
    e = gQ.new_empty((gQ.shape[0], alm_size(p.lmax, p.mmax)), dtype=_ctype(_prec(gQ.dtype)))
    return e, torch.empty_like(e)


@torch.library.custom_op("hb::map2alm_spin2_adjoint", mutates_args=())
def map2alm_spin2_adjoint(gE: torch.Tensor, gB: torch.Tensor, pid: int, weights: Optional[torch.Tensor],
                          flags: int) -> tuple[torch.Tensor, torch.Tensor]:
    _check_cuda(gE, gB, weights)
    p = G.get_plan(pid)
    gE, gB = gE.contiguous(), gB.contiguous()
    nmaps, prec = gE.shape[0], _prec(gE.dtype)
    gQ = torch.empty(nmaps, p.npix, dtype=_rtype(prec), device=gE.device)
    gU = torch.empty_like(gQ)
    ws = _ws(p, prec, nmaps, gE.device, spin=True)
    L.call(f"hb_map2alm_spin2_adjoint_f{prec}", p.handle, nmaps, gE.data_ptr(), gB.data_ptr(), _wptr(weights),
           gQ.data_ptr(), gU.data_ptr(), ws.data_ptr(), ws.numel(), flags, _stream(gE.device))
    return gQ, gU


@map2alm_spin2_adjoint.register_fake
def _(gE, gB, pid, weights, flags):
    q = gE.new_empty((gE.shape[0], G.get_plan(pid).npix), dtype=_rtype(_prec(gE.dtype)))
    return q, torch.empty_like(q)


@torch.library.custom_op("hb::alm2cl", mutates_args=())
def alm2cl(alm1: torch.Tensor, alm2: Optional[torch.Tensor], lmax: int, mmax: int) -> torch.Tensor:
    _check_cuda(alm1, alm2)
    alm1 = alm1.contiguous()
    if alm2 is not None:
        alm2 = alm2.contiguous().to(alm1.dtype)
    nmaps, prec = alm1.shape[0], _prec(alm1.dtype)
    cl = torch.empty(nmaps, lmax + 1, dtype=torch.float64, device=alm1.device)
    L.call(f"hb_alm2cl_f{prec}", lmax, mmax, nmaps, alm1.data_ptr(), None if alm2 is None else alm2.data_ptr(),
           cl.data_ptr(), _stream(alm1.device))
    return cl


@alm2cl.register_fake
def _(alm1, alm2, lmax, mmax):
    return alm1.new_empty((alm1.shape[0], lmax + 1), dtype=torch.float64)


def ring_tables(nside: int, phi0_mode: int, device) -> dict:
    """Device ring tables from the hb_ring_tables kernel."""
    nr = 4 * nside - 1
    dev = torch.device(device)
    f64 = dict(dtype=torch.float64, device=dev)
    out = dict(z=torch.empty(nr, **f64), theta=torch.empty(nr, **f64),
               nphi=torch.empty(nr, dtype=torch.int32, device=dev), phi0=torch.empty(nr, **f64),
               ring_start=torch.empty(nr + 1, dtype=torch.int64, device=dev), z_edges=torch.empty(nr + 1, **f64),
               weights_dz=torch.empty(nr, **f64))
    L.call("hb_ring_tables", nside, phi0_mode, out["z"].data_ptr(), out["theta"].data_ptr(), out["nphi"].data_ptr(),
           out["phi0"].data_ptr(), out["ring_start"].data_ptr(), out["z_edges"].data_ptr(),
           out["weights_dz"].data_ptr(), _stream(dev))
    return out
