"""alm utilities (alm_ops.py of the reference, in healpy m-major layout).

Reference layout (alm_ops.py:4-5): idx = l*(l+1)+m, length (lmax+1)**2.
healpy layout (default here): idx = m*(2*lmax+1-m)/2 + l, length alm_size(lmax, mmax).
"""
from __future__ import annotations

import functools
import math

import numpy as np
import torch

from . import ops
from .util import as_tensor, like_input


def alm_size(lmax: int, mmax: int | None = None) -> int:
    mmax = lmax if mmax is None else mmax
    return ops.alm_size(lmax, mmax)


def alm_index(lmax: int, l, m):
    """healpy index of (l, m)."""
    return m * (2 * lmax + 1 - m) // 2 + l


def ref_index(l, m):
    """The reference's index l*(l+1)+m (alm_ops.py:4-5)."""
    return l * (l + 1) + m


def getlmax(size: int, mmax: int | None = None) -> int:
    """lmax of a healpy-layout vector of ``size`` entries (mmax = lmax unless given)."""
    if mmax is None:
        lmax = int((math.sqrt(1 + 8 * size) - 3) / 2)
        if alm_size(lmax) != size:
            raise ValueError(f"{size} is not a healpy alm size")
        return lmax
    lmax = (size + mmax * (mmax + 1) // 2) // (mmax + 1) - 1
    if alm_size(lmax, mmax) != size:
        raise ValueError(f"{size} is not a healpy alm size for mmax={mmax}")
    return lmax


@functools.lru_cache(maxsize=64)
def _l_of_index(lmax: int, mmax: int, device: str) -> torch.Tensor:
    ls = np.concatenate([np.arange(m, lmax + 1) for m in range(mmax + 1)])
    return torch.from_numpy(ls).to(device)


@functools.lru_cache(maxsize=64)
def _m_of_index(lmax: int, mmax: int, device: str) -> torch.Tensor:
    ms = np.concatenate([np.full(lmax + 1 - m, m) for m in range(mmax + 1)])
    return torch.from_numpy(ms).to(device)


@functools.lru_cache(maxsize=64)
def _ref_perm(lmax: int, mmax: int, device: str) -> torch.Tensor:
    ls = _l_of_index(lmax, mmax, "cpu").numpy()
    ms = _m_of_index(lmax, mmax, "cpu").numpy()
    return torch.from_numpy(ls * (ls + 1) + ms).to(device)


def healpy_to_ref(alm, lmax: int, mmax: int | None = None):
    """healpy layout -> reference layout (zeros in the unused l*(l+1)-l..l*(l+1)-1 slots)."""
    mmax = lmax if mmax is None else mmax
    t = as_tensor(alm)
    out = torch.zeros(*t.shape[:-1], (lmax + 1) ** 2, dtype=t.dtype, device=t.device)
    out[..., _ref_perm(lmax, mmax, str(t.device))] = t
    return like_input(out, alm)


def ref_to_healpy(alm, lmax: int | None = None, mmax: int | None = None):
    t = as_tensor(alm)
    lmax = int(math.isqrt(t.shape[-1])) - 1 if lmax is None else lmax
    mmax = lmax if mmax is None else mmax
    return like_input(t[..., _ref_perm(lmax, mmax, str(t.device))].contiguous(), alm)


def almxfl(alm, fl, mmax: int | None = None, inplace: bool = False, lmax: int | None = None):
    """a_lm * f_l (alm_ops.py:7-17), healpy layout."""
    t = as_tensor(alm)
    lmax = getlmax(t.shape[-1], mmax) if lmax is None else lmax
    mmax = lmax if mmax is None else mmax
    f = torch.as_tensor(np.asarray(fl) if not isinstance(fl, torch.Tensor) else fl, device=t.device)
    f = f.to(torch.float64 if t.dtype == torch.complex128 else torch.float32)
    fx = torch.zeros(lmax + 1, dtype=f.dtype, device=t.device)
    n = min(lmax + 1, f.numel())
    fx[:n] = f[:n]
    scale = fx[_l_of_index(lmax, mmax, str(t.device))]
    if inplace:
        t.mul_(scale)
        return alm
    return like_input(t * scale, alm)


def alm2cl(alms, alms2=None, lmax: int | None = None, mmax: int | None = None):
    """C_l = (|a_l0|^2 + 2 sum_{m>0} |a_lm|^2)/(2l+1) (alm_ops.py:19-32) on the GPU (hb_alm2cl).
    ``alms2`` gives the cross spectrum Re(a b*).  Accepts [nalm] or [nmaps, nalm]."""
    t = as_tensor(alms)
    lmax_in = getlmax(t.shape[-1], mmax)
    lmax = lmax_in if lmax is None else lmax
    mm = lmax_in if mmax is None else mmax
    squeeze = t.dim() == 1
    t2 = t.reshape(-1, t.shape[-1])
    b = None if alms2 is None else as_tensor(alms2).reshape(-1, t.shape[-1])
    cl = ops.alm2cl(t2, b, lmax_in, mm)
    cl = cl[:, :lmax + 1]
    return like_input(cl[0] if squeeze else cl, alms)


def synalm(cls, lmax: int | None = None, mmax: int | None = None, seed: int | None = None, device=None,
           dtype=torch.complex128):
    """Gaussian alm in healpy layout, drawn like alm_ops.py:34-54 (l ascending: m=0 real
    N(0,C_l), m>0 Re and Im N(0,C_l/2); nothing drawn for C_l <= 0) with numpy's default_rng."""
    cl = np.asarray(cls.detach().cpu().numpy() if isinstance(cls, torch.Tensor) else cls, dtype=np.float64)
    lmax = cl.size - 1 if lmax is None else lmax
    mmax = lmax if mmax is None else mmax
    rng = np.random.default_rng(seed)
    alm = np.zeros(alm_size(lmax, mmax), dtype=np.complex128)
    for l in range(lmax + 1):
        C = float(cl[l]) if l < cl.size else 0.0
        if C <= 0.0:
            continue
        alm[alm_index(lmax, l, 0)] = rng.normal(0.0, math.sqrt(C))
        if l > 0:
            sd = math.sqrt(C / 2.0)
            re = rng.normal(0.0, sd, size=l)
            im = rng.normal(0.0, sd, size=l)
            ms = np.arange(1, min(l, mmax) + 1)
            alm[alm_index(lmax, l, ms)] = (re + 1j * im)[:ms.size]
    dev = torch.device("cuda") if device is None else torch.device(device)
    return torch.from_numpy(alm).to(device=dev, dtype=dtype)
