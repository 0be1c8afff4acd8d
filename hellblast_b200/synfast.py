"""T, Q, U map simulation from power spectra (synfast), with the names and conventions of
hellblast's synfast_tqu.py.

* ``synalm_te`` draws Gaussian T/E/B alm: T and E correlated through the per-l Cholesky factor
  of [[C_TT, C_TE], [C_TE, C_EE]] (L11 = sqrt C_TT, L21 = C_TE / L11,
  L22 = sqrt(C_EE - L21^2); a non-positive-definite block falls back to L21 = 0), B
  independent; m = 0 real with variance C_l, m > 0 with Re and Im of variance C_l / 2
  (synfast_tqu.py:28-67).  The reference loops over l in Python with CuPy's legacy generator;
  here every (l, m) entry is drawn at once on the GPU (torch's Philox generator, seeded), in
  healpy's m-major layout.  ``te_from_normals`` is the algebra alone, for given unit normals.
* ``synfast_tqu`` applies the beam b_l (Gaussian of ``fwhm``) and the pixel window
  (ones, as the reference without healpy, beams.py:6-22) as one filter, synthesises T with the
  scalar transform and Q/U with the spin-2 transform (healpy convention: the reference's
  qu_from_eb_gpu fills the complex spin field's spectrum as if it were real, spin.py:104,106),
  and adds white noise per pixel (synfast_tqu.py:69-128).
"""
from __future__ import annotations

import math

import torch

from . import alm_ops, hp_compat
from .smoothing import beam_filter, pixel_window_fl


def _lm_of_index(lmax: int, device) -> tuple[torch.Tensor, torch.Tensor]:
    return alm_ops._l_of_index(lmax, lmax, str(device)), alm_ops._m_of_index(lmax, lmax, str(device))


def te_from_normals(cltt, clee, clbb, clte, z1, z2, zb, lmax: int):
    """aT, aE, aB (healpy layout) from unit complex normals z1, z2, zb (per alm entry; the m = 0
    entries' imaginary parts are ignored): aT = L11 z1, aE = L21 z1 + L22 z2, aB = sqrt(C_BB) zb,
    with the m > 0 normals' components scaled by 1/sqrt 2 (synfast_tqu.py:36-66)."""
    dev = z1.device
    l, m = _lm_of_index(lmax, dev)
    c = [torch.as_tensor(x, dtype=torch.float64, device=dev)[: lmax + 1] for x in (cltt, clee, clbb, clte)]
    Ctt, Cee, Cbb, Cte = (x[l] for x in c)
    ok = (Ctt > 0) & (Cee > 0) & (Ctt * Cee - Cte * Cte > 0)
    L11 = torch.sqrt(torch.clamp(Ctt, min=0.0))
    L21 = torch.where(ok, Cte / torch.where(ok, L11, torch.ones_like(L11)), torch.zeros_like(L11))
    L22 = torch.where(ok, torch.sqrt(torch.clamp(Cee - L21 * L21, min=0.0)), torch.sqrt(torch.clamp(Cee, min=0.0)))
    sb = torch.sqrt(torch.clamp(Cbb, min=0.0))
    half = torch.where(m > 0, torch.full_like(L11, math.sqrt(0.5)), torch.ones_like(L11))
    real0 = m == 0

    def fix(z):  # m = 0: real, unit variance; m > 0: components of variance 1/2
        z = z.to(torch.complex128) * half
        return torch.where(real0, z.real.to(torch.complex128), z)
    z1, z2, zb = fix(z1), fix(z2), fix(zb)
    return L11 * z1, L21 * z1 + L22 * z2, sb * zb


def synalm_te(cltt, clee, clbb, clte, lmax: int | None = None, seed: int | None = None, device=None,
              nsims: int = 1):
    """Correlated Gaussian (aT, aE, aB), each [nsims, nalm] complex128 in healpy layout."""
    dev = torch.device("cuda") if device is None else torch.device(device)
    lmax = len(cltt) - 1 if lmax is None else int(lmax)
    n = alm_ops.alm_size(lmax)
    gen = torch.Generator(device=dev)
    gen.manual_seed(0 if seed is None else int(seed))

    def normals():
        return torch.complex(torch.randn(nsims, n, generator=gen, device=dev, dtype=torch.float64),
                             torch.randn(nsims, n, generator=gen, device=dev, dtype=torch.float64))
    z1, z2, zb = normals(), normals(), normals()
    return te_from_normals(cltt, clee, clbb, clte, z1, z2, zb, lmax)


def synfast_tqu(cls: dict, nside: int, lmax: int | None = None, fwhm=None, use_pixel_window: bool = True,
                seed: int | None = None, sigmaT=None, sigmaQ=None, sigmaU=None, return_alm: bool = False,
                precision: str = "fp32", nsims: int = 1, alms=None):
    """T, Q, U RING maps ([nsims, npix]; [npix] when nsims = 1) from the spectra in ``cls``
    ('tt' alone, or 'tt', 'ee', 'bb', 'te').  ``alms`` = (aT, aE, aB) skips the draw (the
    filters, synthesis and noise still apply).  precision: "fp32" or "fp64" transforms."""
    dev = torch.device("cuda")
    if lmax is None:
        lmax = len(next(iter(cls.values()))) - 1
    lmax = int(lmax)
    n = alm_ops.alm_size(lmax)
    if alms is not None:
        aT, aE, aB = (torch.as_tensor(a, device=dev).to(torch.complex128).reshape(-1, n) for a in alms)
    else:
        pol = any(cls.get(k) is not None for k in ("ee", "bb", "te"))
        if pol and any(cls.get(k) is None for k in ("tt", "ee", "bb", "te")):
            raise ValueError("For polarized synfast provide tt, ee, bb, te spectra.")
        zero = [0.0] * (lmax + 1)
        aT, aE, aB = synalm_te(cls["tt"], cls.get("ee", zero), cls.get("bb", zero), cls.get("te", zero), lmax,
                               seed=seed, device=dev, nsims=nsims)
        if not pol:
            aE = torch.zeros_like(aT)
            aB = torch.zeros_like(aT)
    pT, pP = pixel_window_fl(int(nside), lmax, pol=True, device=dev) if use_pixel_window else (None, None)
    fT = beam_filter(lmax, fwhm=fwhm, pixwin=pT, device=dev)
    fP = beam_filter(lmax, fwhm=fwhm, pixwin=pP, device=dev)
    aT = alm_ops.almxfl(aT, fT, lmax=lmax)
    aE = alm_ops.almxfl(aE, fP, lmax=lmax)
    aB = alm_ops.almxfl(aB, fP, lmax=lmax)
    ct = torch.complex64 if precision == "fp32" else torch.complex128
    T = hp_compat.alm2map(aT.to(ct), int(nside), lmax=lmax)
    Q, U = hp_compat.alm2map_spin(aE.to(ct), aB.to(ct), 2, nside=int(nside), lmax=lmax)
    gen = torch.Generator(device=dev)
    gen.manual_seed(1 + (0 if seed is None else int(seed)))
    for x, s in ((T, sigmaT), (Q, sigmaQ), (U, sigmaU)):
        if s is not None and s > 0:
            x += float(s) * torch.randn(x.shape, generator=gen, device=dev, dtype=x.dtype)
    sq = aT.shape[0] == 1
    out = (T[0], Q[0], U[0]) if sq else (T, Q, U)
    if return_alm:
        return out + ((aT[0], aE[0], aB[0]) if sq else (aT, aE, aB))
    return out
