"""FP64 CPU oracle for the HEALPix SHT hot path (Python half).

TEST INFRASTRUCTURE ONLY: the arbiter the CUDA path is checked against.  Only tests/,
__graft_entry__.smoke() and bench.py's cpu_baseline leg may import this module; the
product package (hellblast_b200) never does.

The Legendre work is done by the C half (oracle/sht_oracle.c -> oracle/liborc.so, OpenMP).
This file restates the per-ring FFT step of the reference with numpy's pocketfft:

* ``sht_raw.py:38-43`` / ``sht_fallback.py:51-55``: ``F_r = fft(f_r) / nphi_r``, then the
  contraction weights ``weights_dz`` (``sht_raw.py:50-53``) and the 2*pi factor
  (``sht_fallback.py:63``).  Here the per-pixel quadrature weight is ``2*pi*w_r/nphi_r``.
* corrected relative to the reference (each correction can be switched off by ``ref_compat``):
  the per-ring phase ``exp(-i m phi0_r)`` and the m-aliasing fold ``m -> m mod nphi_r``
  (the reference reads bin m for m < nphi and uses 0 for m >= nphi, ``sht_raw.py:51``).
* ``isht.py:15-25`` (synthesis) corrected the same way: ``f(phi_j) = Re sum_m c_m G(m)
  exp(i m phi_j)`` with ``c_0 = 1, c_m = 2``, folded onto the ring's nphi bins.

alm layout: healpy m-major, ``idx(l, m) = m*(2*lmax+1-m)//2 + l``.
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liborc.so")
        if not os.path.exists(path):
            build()
        lib = ctypes.CDLL(path)
        D = ctypes.POINTER(ctypes.c_double)
        I32 = ctypes.POINTER(ctypes.c_int32)
        I64 = ctypes.POINTER(ctypes.c_int64)
        lib.orc_ring_tables.argtypes = [ctypes.c_int64, ctypes.c_int, D, D, I32, D, I64, D]
        lib.orc_lambda_lm.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int64, D, D, D]
        lib.orc_legendre_analysis.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int64, D, D, D, D]
        lib.orc_legendre_synthesis.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int64, D, D, D, D]
        lib.orc_spin2_lambda.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int64, D, D, D, D]
        lib.orc_spin2_analysis.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int64, D, D, D, D, D, D]
        lib.orc_spin2_synthesis.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int64, D, D, D, D, D, D]
        lib.orc_alm2cl.argtypes = [ctypes.c_int, ctypes.c_int, D, D, D]
        lib.orc_spin2_analysis_ms.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int64,
                                              D, D, D, D, D, D]
        lib.orc_legendre_analysis_ms.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                                 ctypes.c_int64, D, D, D, D]
        lib.orc_legendre_synthesis_ms.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                                  ctypes.c_int64, D, D, D, D]
        for f in (lib.orc_legendre_analysis_ms, lib.orc_legendre_synthesis_ms):
            f.restype = None
        lib.orc_ring2nest.argtypes = [ctypes.c_int64, ctypes.c_int64, I64, I64]
        lib.orc_nest2ring.argtypes = [ctypes.c_int64, ctypes.c_int64, I64, I64]
        lib.orc_pix2ang.argtypes = [ctypes.c_int64, ctypes.c_int, ctypes.c_int64, I64, D, D]
        lib.orc_ang2pix.argtypes = [ctypes.c_int64, ctypes.c_int, ctypes.c_int64, D, D, I64]
        for f in (lib.orc_ring2nest, lib.orc_nest2ring, lib.orc_pix2ang, lib.orc_ang2pix):
            f.restype = None
        lib.orc_wigner_d.argtypes = [ctypes.c_int, ctypes.c_double, D]
        lib.orc_wigner_d.restype = None
        for f in (lib.orc_ring_tables, lib.orc_lambda_lm, lib.orc_legendre_analysis,
                  lib.orc_legendre_synthesis, lib.orc_spin2_lambda, lib.orc_spin2_analysis,
                  lib.orc_spin2_synthesis, lib.orc_alm2cl, lib.orc_spin2_analysis_ms):
            f.restype = None
        _LIB = lib
    return _LIB


def build() -> None:
    """Compile oracle/liborc.so (gcc, OpenMP)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", _HERE, "liborc.so"], check=True)


def _p(a, ct=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(ct))


# ----------------------------------------------------------------------------- layout
def alm_size(lmax: int, mmax: int | None = None) -> int:
    mmax = lmax if mmax is None else mmax
    return mmax * (2 * lmax + 1 - mmax) // 2 + lmax + 1


def alm_index(lmax: int, l, m):
    return m * (2 * lmax + 1 - m) // 2 + l


def healpy_to_ref(alm: np.ndarray, lmax: int, mmax: int | None = None) -> np.ndarray:
    """healpy m-major -> the reference's l(l+1)+m layout (alm_ops.py:4-5), length (lmax+1)^2."""
    mmax = lmax if mmax is None else mmax
    out = np.zeros((lmax + 1) ** 2, dtype=np.complex128)
    for m in range(mmax + 1):
        l = np.arange(m, lmax + 1)
        out[l * (l + 1) + m] = alm[alm_index(lmax, l, m)]
    return out


def ref_to_healpy(alm_ref: np.ndarray, lmax: int, mmax: int | None = None) -> np.ndarray:
    mmax = lmax if mmax is None else mmax
    out = np.zeros(alm_size(lmax, mmax), dtype=np.complex128)
    for m in range(mmax + 1):
        l = np.arange(m, lmax + 1)
        out[alm_index(lmax, l, m)] = alm_ref[l * (l + 1) + m]
    return out


# ----------------------------------------------------------------------------- geometry
def ring_tables(nside: int, phi0: str = "healpix") -> dict:
    """HEALPix RING geometry (ring_tables_healpix.cu:14-51, ring_tables.py:39-40)."""
    nr = 4 * nside - 1
    z = np.empty(nr); th = np.empty(nr); ph = np.empty(nr); ze = np.empty(nr + 1)
    nphi = np.empty(nr, dtype=np.int32); rs = np.empty(nr + 1, dtype=np.int64)
    _lib().orc_ring_tables(nside, 1 if phi0 == "healpix" else 0, _p(z), _p(th), _p(nphi, ctypes.c_int32),
                           _p(ph), _p(rs, ctypes.c_int64), _p(ze))
    i = np.arange(1, nr + 1, dtype=np.float64)
    ip = np.minimum(i, 4 * nside - i)
    polar = ip < nside
    t = ip * ip / (3.0 * nside * nside)           # 1-|z| exactly on the polar caps
    sin_theta = np.where(polar, np.sqrt(t * (2.0 - t)), np.sqrt((1.0 - z) * (1.0 + z)))
    return dict(nside=nside, nr=nr, npix=int(rs[-1]), z=z, theta=th, nphi=nphi, phi0=ph,
                ring_start=rs, z_edges=ze, weights_dz=ze[:-1] - ze[1:], x=z.copy(),
                sin_theta=sin_theta)


def generic_geometry(theta, nphi, phi0=None, weights=None) -> dict:
    theta = np.asarray(theta, dtype=np.float64)
    nphi = np.asarray(nphi, dtype=np.int32)
    nr = theta.size
    rs = np.zeros(nr + 1, dtype=np.int64)
    rs[1:] = np.cumsum(nphi)
    return dict(nr=nr, npix=int(rs[-1]), theta=theta, nphi=nphi,
                phi0=np.zeros(nr) if phi0 is None else np.asarray(phi0, dtype=np.float64),
                ring_start=rs, weights_dz=None if weights is None else np.asarray(weights, dtype=np.float64),
                x=np.cos(theta), sin_theta=np.sin(theta))


def uniform_weights(geom: dict) -> np.ndarray:
    """Per-ring w such that 2*pi*w_r/nphi_r = 4*pi/npix (healpy's default quadrature)."""
    return 2.0 * geom["nphi"].astype(np.float64) / geom["npix"]


# ----------------------------------------------------------------------------- ring FFTs
def ring_analysis(maps: np.ndarray, geom: dict, mmax: int, weights=None, phase=True, fold=True,
                  scale: float = 2.0 * math.pi, mdouble: bool = False) -> np.ndarray:
    """F[m, r] = scale * w_r / nphi_r * exp(-i m phi0_r) * DFT_r[m mod nphi_r].

    With ``fold=False`` bins m >= nphi_r are zero (reference behaviour, sht_raw.py:51).
    ``weights=None`` means unit per-pixel weights (scale/nphi factor dropped); used by adjoints.
    ``mdouble`` multiplies m>0 by 2 (adjoint of the real-field synthesis).
    """
    nr = geom["nr"]
    F = np.zeros((mmax + 1, nr), dtype=np.complex128)
    m = np.arange(mmax + 1)
    for r in range(nr):
        n = int(geom["nphi"][r]); s = int(geom["ring_start"][r])
        R = np.fft.rfft(np.asarray(maps[s:s + n], dtype=np.float64))
        k = m % n
        D = np.where(k <= n // 2, R[np.minimum(k, n // 2)], np.conj(R[np.minimum(n - k, n // 2)]))
        if not fold:
            D = np.where(m < n, D, 0.0)
        if phase:
            D = D * np.exp(-1j * m * geom["phi0"][r])
        if weights is not None:
            D = D * (scale * weights[r] / n)
        if mdouble:
            D = D * np.where(m > 0, 2.0, 1.0)
        F[:, r] = D
    return F


def ring_synthesis(G: np.ndarray, geom: dict, weights=None, phase=True, mdouble=True,
                   scale: float = 2.0 * math.pi) -> np.ndarray:
    """f_r(phi_j) = Re sum_m c_m G[m, r] exp(i m phi_j), folded onto nphi_r bins.

    ``mdouble=True`` uses c_0 = 1, c_m = 2 (real field); False uses c_m = 1 (adjoint of the
    weighted analysis).  ``weights`` multiplies the result by scale*w_r/nphi_r (adjoint only).
    """
    mmax = G.shape[0] - 1
    out = np.zeros(int(geom["npix"]))
    m = np.arange(mmax + 1)
    c = np.where(m > 0, 2.0, 1.0) if mdouble else np.ones(mmax + 1)
    for r in range(geom["nr"]):
        n = int(geom["nphi"][r]); s = int(geom["ring_start"][r])
        T = c * G[:, r]
        if phase:
            T = T * np.exp(1j * m * geom["phi0"][r])
        k = m % n
        X = np.zeros(n // 2 + 1, dtype=np.complex128)
        edge = (k == 0) | (k * 2 == n)
        np.add.at(X, k[edge], T[edge].real)
        lo = (~edge) & (2 * k < n)
        np.add.at(X, k[lo], 0.5 * T[lo])
        hi = (~edge) & (2 * k > n)
        np.add.at(X, n - k[hi], 0.5 * np.conj(T[hi]))
        f = np.fft.irfft(X, n) * n
        if weights is not None:
            f = f * (scale * weights[r] / n)
        out[s:s + n] = f
    return out


# ----------------------------------------------------------------------------- transforms
def _c(a):
    return np.ascontiguousarray(a)


def legendre_analysis(F: np.ndarray, geom: dict, lmax: int) -> np.ndarray:
    mmax = F.shape[0] - 1
    Fi = _c(F.astype(np.complex128)).view(np.float64)
    alm = np.zeros(alm_size(lmax, mmax), dtype=np.complex128)
    _lib().orc_legendre_analysis(lmax, mmax, geom["nr"], _p(_c(geom["x"])), _p(_c(geom["sin_theta"])),
                                 _p(Fi), _p(alm.view(np.float64)))
    return alm


def legendre_synthesis(alm: np.ndarray, geom: dict, lmax: int, mmax: int) -> np.ndarray:
    G = np.zeros((mmax + 1, geom["nr"]), dtype=np.complex128)
    a = _c(np.asarray(alm, dtype=np.complex128))
    _lib().orc_legendre_synthesis(lmax, mmax, geom["nr"], _p(_c(geom["x"])), _p(_c(geom["sin_theta"])),
                                  _p(a.view(np.float64)), _p(G.view(np.float64)))
    return G


def map2alm(maps, geom: dict, lmax: int, mmax: int | None = None, weights=None, phase=True,
            fold=True, scale=2.0 * math.pi) -> np.ndarray:
    """a_lm = sum_pixels (scale*w_r/nphi_r) f lambda_lm e^{-i m phi} (healpy layout)."""
    mmax = lmax if mmax is None else mmax
    w = geom["weights_dz"] if weights is None else weights
    F = ring_analysis(maps, geom, mmax, weights=w, phase=phase, fold=fold, scale=scale)
    return legendre_analysis(F, geom, lmax)


def alm2map(alm, geom: dict, lmax: int, mmax: int | None = None, phase=True) -> np.ndarray:
    mmax = lmax if mmax is None else mmax
    G = legendre_synthesis(alm, geom, lmax, mmax)
    return ring_synthesis(G, geom, phase=phase)


def map2alm_ref_compat(maps, geom: dict, lmax: int, mmax: int | None = None, flavour: str = "fallback"):
    """The reference's own conventions (sht_raw.py:30-57 / sht_fallback.py:36-65): no phi0 phase,
    no alias fold, 2*pi only in the fallback flavour, and sht_raw's m <= 2*nside cut (its
    ``mmax_eff``, sht_raw.py:43).  Returned in healpy layout."""
    mmax = lmax if mmax is None else mmax
    scale = 2.0 * math.pi if flavour == "fallback" else 1.0
    alm = map2alm(maps, geom, lmax, mmax, phase=False, fold=False, scale=scale)
    if flavour == "raw":
        mcut = min(mmax, int(np.max(geom["nphi"])) // 2)
        for m in range(mcut + 1, mmax + 1):
            alm[alm_index(lmax, np.arange(m, lmax + 1), m)] = 0.0
    return alm


def map2alm_adjoint(galm, geom: dict, lmax: int, mmax: int | None = None, weights=None, phase=True):
    """Exact transpose of map2alm (real map -> complex alm, Re/Im as independent outputs)."""
    mmax = lmax if mmax is None else mmax
    w = geom["weights_dz"] if weights is None else weights
    G = legendre_synthesis(galm, geom, lmax, mmax)
    return ring_synthesis(G, geom, weights=w, phase=phase, mdouble=False)


def alm2map_adjoint(gmap, geom: dict, lmax: int, mmax: int | None = None, phase=True):
    """Exact transpose of alm2map (includes the m>0 real-field doubling)."""
    mmax = lmax if mmax is None else mmax
    F = ring_analysis(gmap, geom, mmax, weights=None, phase=phase, mdouble=True)
    return legendre_analysis(F, geom, lmax)


def map2alm_spin2(Q, U, geom: dict, lmax: int, mmax: int | None = None, weights=None, phase=True, fold=True):
    mmax = lmax if mmax is None else mmax
    w = geom["weights_dz"] if weights is None else weights
    Qf = _c(ring_analysis(Q, geom, mmax, weights=w, phase=phase, fold=fold))
    Uf = _c(ring_analysis(U, geom, mmax, weights=w, phase=phase, fold=fold))
    n = alm_size(lmax, mmax)
    E = np.zeros(n, dtype=np.complex128); B = np.zeros(n, dtype=np.complex128)
    _lib().orc_spin2_analysis(lmax, mmax, geom["nr"], _p(_c(geom["x"])), _p(_c(geom["theta"])),
                              _p(Qf.view(np.float64)), _p(Uf.view(np.float64)),
                              _p(E.view(np.float64)), _p(B.view(np.float64)))
    return E, B


def spin2_d_tables(geom: dict, lmax: int):
    """Wigner d^l_{m,+2}(theta_r) and d^l_{m,-2}(theta_r), [m][ring][l] (zero for l < max(m, 2)), from
    the oracle's own recursion (orc_spin2_lambda: _{-2}lambda = N_l d^l_{m,+2},
    _{+2}lambda = N_l d^l_{m,-2}, N_l = sqrt((2l+1)/4pi))."""
    th = _c(np.asarray(geom["theta"], dtype=np.float64))
    nl = np.sqrt((2.0 * np.arange(lmax + 1) + 1.0) / (4.0 * math.pi))
    dp2 = np.zeros((lmax + 1, th.size, lmax + 1)); dm2 = np.zeros_like(dp2)
    for m in range(lmax + 1):
        lp2, lm2 = spin2_lambda(lmax, m, th)
        dp2[m] = lm2 / nl
        dm2[m] = lp2 / nl
    return dp2, dm2


def map2alm_spin2_ref_compat(Q, U, geom: dict, lmax: int, mmax: int | None = None, weights=None, d_tables=None):
    """The reference's spin-2 analysis, spin.py:43-78, restated with numpy.

    Per ring: P = Q + iU and M = Q - iU (spin.py:43-44), PF = fft(P)/nphi and MF = fft(M)/nphi
    (:50-51); the orders run to mmax_eff = max_r min(mmax, nphi_r // 2) (:53, :57) and ring r
    contributes bin m only for m < nphi_r, with no phi0 phase and no alias fold (:65-66);
    a_{+-2,lm} = 2 pi sqrt((2l+1)/4pi) sum_r w_r d^l_{m,+-2}(theta_r) PF/MF_r[m], l >= max(m, 2)
    (:61, :67-68); E = -(a2 + a-2)/2, B = i (a2 - a-2)/2 (:76-77).  Outputs in the reference's
    l(l+1)+m layout (:69-70): (a2, a-2, E, B).

    ``d_tables`` = (d_p2, d_m2), each [m][ring][l], are the Wigner-d values to contract with:
    the reference's own wigner_d_ms_sum tables reproduce its output exactly; the default is the
    oracle's recursion (spin2_d_tables), i.e. the textbook d^l_{m,+-2} the reference's kernel
    sets out to compute.
    """
    mmax = lmax if mmax is None else mmax
    w = geom["weights_dz"] if weights is None else weights
    dp2, dm2 = spin2_d_tables(geom, lmax) if d_tables is None else d_tables
    nr = geom["nr"]
    PF, MF = [], []
    mmax_eff = 0
    for r in range(nr):
        n = int(geom["nphi"][r]); s = int(geom["ring_start"][r])
        q = np.asarray(Q[s:s + n], dtype=np.float64); u = np.asarray(U[s:s + n], dtype=np.float64)
        PF.append(np.fft.fft(q + 1j * u) / n)
        MF.append(np.fft.fft(q - 1j * u) / n)
        mmax_eff = max(mmax_eff, min(mmax, n // 2))
    nl = np.sqrt((2.0 * np.arange(lmax + 1) + 1.0) / (4.0 * math.pi))
    a2 = np.zeros((lmax + 1) ** 2, dtype=np.complex128); am2 = np.zeros_like(a2)
    for m in range(mmax_eff + 1):
        pf = np.array([PF[r][m] if m < int(geom["nphi"][r]) else 0.0 for r in range(nr)])
        mf = np.array([MF[r][m] if m < int(geom["nphi"][r]) else 0.0 for r in range(nr)])
        for l in range(max(m, 2), lmax + 1):
            a2[l * (l + 1) + m] = np.sum(w * dp2[m][:, l] * pf) * nl[l] * (2.0 * math.pi)
            am2[l * (l + 1) + m] = np.sum(w * dm2[m][:, l] * mf) * nl[l] * (2.0 * math.pi)
    return a2, am2, -(a2 + am2) * 0.5, 1j * (a2 - am2) * 0.5


def ring_analysis_ms(maps: np.ndarray, geom: dict, ms, weights) -> np.ndarray:
    """ring_analysis for the harmonic orders ``ms`` only: F[j, r] for m = ms[j] (with the
    quadrature weights, phase and alias fold of ring_analysis)."""
    ms = np.asarray(ms, dtype=np.int64)
    nr = geom["nr"]
    F = np.zeros((ms.size, nr), dtype=np.complex128)
    for r in range(nr):
        n = int(geom["nphi"][r]); s = int(geom["ring_start"][r])
        R = np.fft.rfft(np.asarray(maps[s:s + n], dtype=np.float64))
        k = ms % n
        D = np.where(k <= n // 2, R[np.minimum(k, n // 2)], np.conj(R[np.minimum(n - k, n // 2)]))
        F[:, r] = D * np.exp(-1j * ms * geom["phi0"][r]) * (2.0 * math.pi * weights[r] / n)
    return F


def legendre_analysis_ms(F, geom: dict, lmax: int, ms) -> np.ndarray:
    """Legendre analysis of the orders ``ms`` only: F [len(ms), nr] -> [len(ms), lmax + 1]."""
    ms = np.ascontiguousarray(ms, dtype=np.int32)
    F = _c(np.asarray(F, dtype=np.complex128))
    out = np.zeros((ms.size, lmax + 1), dtype=np.complex128)
    _lib().orc_legendre_analysis_ms(lmax, int(ms.size), ms.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), geom["nr"],
                                    _p(_c(geom["x"])), _p(_c(geom["sin_theta"])), _p(F.view(np.float64)),
                                    _p(out.view(np.float64)))
    return out


def legendre_synthesis_ms(a, geom: dict, lmax: int, ms) -> np.ndarray:
    """Legendre synthesis of the orders ``ms`` only: a [len(ms), lmax + 1] -> G [len(ms), nr]."""
    ms = np.ascontiguousarray(ms, dtype=np.int32)
    a = _c(np.asarray(a, dtype=np.complex128))
    G = np.zeros((ms.size, geom["nr"]), dtype=np.complex128)
    _lib().orc_legendre_synthesis_ms(lmax, int(ms.size), ms.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), geom["nr"],
                                     _p(_c(geom["x"])), _p(_c(geom["sin_theta"])), _p(a.view(np.float64)),
                                     _p(G.view(np.float64)))
    return G


def alm_rows(alm, lmax: int, ms, mmax: int | None = None) -> np.ndarray:
    """healpy-layout alm -> [len(ms), lmax + 1] rows of the orders ``ms`` (l < m zero)."""
    mmax = lmax if mmax is None else mmax
    alm = np.asarray(alm, dtype=np.complex128)
    out = np.zeros((len(ms), lmax + 1), dtype=np.complex128)
    for j, m in enumerate(ms):
        m = int(m)
        out[j, m:] = alm[m * (2 * lmax + 1 - m) // 2 + np.arange(m, lmax + 1)]
    return out


def map2alm_ms(maps, geom: dict, lmax: int, ms, weights=None) -> np.ndarray:
    """a_lm of map2alm at the harmonic orders ``ms`` only: [len(ms), lmax + 1] (l < m zero).
    For spot checks of transforms too large for the full oracle."""
    w = geom["weights_dz"] if weights is None else weights
    return legendre_analysis_ms(ring_analysis_ms(maps, geom, ms, w), geom, lmax, ms)


def alm2map_ms(alm, geom: dict, lmax: int, ms, mmax: int | None = None) -> np.ndarray:
    """The map of alm2map when only the orders ``ms`` of ``alm`` (healpy layout) are kept."""
    ms = np.unique(np.asarray(ms, dtype=np.int64))
    Gj = legendre_synthesis_ms(alm_rows(alm, lmax, ms, mmax), geom, lmax, ms)
    G = np.zeros((int(ms.max()) + 1, geom["nr"]), dtype=np.complex128)
    G[ms] = Gj
    return ring_synthesis(G, geom)


def ring_subset(geom: dict, r0: int, r1: int) -> dict:
    """The rings [r0, r1) of a geometry as a geometry of their own (ring offsets rebased), for
    running the ring FFT steps of a transform over a block of rings."""
    rs = geom["ring_start"]
    sub = dict(geom)
    sub["nr"] = r1 - r0
    for k in ("nphi", "phi0", "theta", "x", "z", "sin_theta", "weights_dz"):
        if k in geom:
            sub[k] = geom[k][r0:r1]
    sub["ring_start"] = rs[r0:r1 + 1] - rs[r0]
    sub["npix"] = int(rs[r1] - rs[r0])
    return sub


def map2alm_spin2_ms(Q, U, geom: dict, lmax: int, ms):
    """(E, B) [len(ms), lmax + 1] of map2alm_spin2 at the harmonic orders ``ms`` only."""
    ms = np.ascontiguousarray(ms, dtype=np.int32)
    w = geom["weights_dz"]
    Qf = _c(ring_analysis_ms(Q, geom, ms, w))
    Uf = _c(ring_analysis_ms(U, geom, ms, w))
    E = np.zeros((ms.size, lmax + 1), dtype=np.complex128)
    B = np.zeros((ms.size, lmax + 1), dtype=np.complex128)
    _lib().orc_spin2_analysis_ms(lmax, int(ms.size), ms.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), geom["nr"],
                                 _p(_c(geom["x"])), _p(_c(geom["theta"])), _p(Qf.view(np.float64)),
                                 _p(Uf.view(np.float64)), _p(E.view(np.float64)), _p(B.view(np.float64)))
    return E, B


def alm2map_spin2(E, B, geom: dict, lmax: int, mmax: int | None = None, phase=True):
    mmax = lmax if mmax is None else mmax
    Qg = np.zeros((mmax + 1, geom["nr"]), dtype=np.complex128)
    Ug = np.zeros_like(Qg)
    E = _c(np.asarray(E, dtype=np.complex128)); B = _c(np.asarray(B, dtype=np.complex128))
    _lib().orc_spin2_synthesis(lmax, mmax, geom["nr"], _p(_c(geom["x"])), _p(_c(geom["theta"])),
                               _p(E.view(np.float64)), _p(B.view(np.float64)),
                               _p(Qg.view(np.float64)), _p(Ug.view(np.float64)))
    return ring_synthesis(Qg, geom, phase=phase), ring_synthesis(Ug, geom, phase=phase)


def lambda_lm(lmax: int, m: int, x, sin_theta) -> np.ndarray:
    x = _c(np.asarray(x, dtype=np.float64)); s = _c(np.asarray(sin_theta, dtype=np.float64))
    out = np.zeros((x.size, lmax + 1))
    _lib().orc_lambda_lm(lmax, m, x.size, _p(x), _p(s), _p(out))
    return out


def spin2_lambda(lmax: int, m: int, theta):
    th = _c(np.asarray(theta, dtype=np.float64)); x = np.cos(th)
    p2 = np.zeros((th.size, lmax + 1)); m2 = np.zeros_like(p2)
    _lib().orc_spin2_lambda(lmax, m, th.size, _p(x), _p(th), _p(p2), _p(m2))
    return p2, m2


def alm2cl(alm1, lmax: int, mmax: int | None = None, alm2=None) -> np.ndarray:
    mmax = lmax if mmax is None else mmax
    a1 = _c(np.asarray(alm1, dtype=np.complex128))
    a2 = None if alm2 is None else _c(np.asarray(alm2, dtype=np.complex128))
    cl = np.zeros(lmax + 1)
    _lib().orc_alm2cl(lmax, mmax, _p(a1.view(np.float64)),
                      None if a2 is None else _p(a2.view(np.float64)), _p(cl))
    return cl


def synalm(cl, lmax: int | None = None, seed: int = 0) -> np.ndarray:
    """Gaussian alm in healpy layout drawn like alm_ops.py:34-54 (l ascending; m=0 real
    N(0,C_l); m>0 Re, Im ~ N(0, C_l/2); nothing drawn when C_l <= 0), numpy default_rng."""
    cl = np.asarray(cl, dtype=np.float64)
    lmax = cl.size - 1 if lmax is None else lmax
    rng = np.random.default_rng(seed)
    alm = np.zeros(alm_size(lmax), dtype=np.complex128)
    for l in range(lmax + 1):
        C = float(cl[l])
        if C <= 0.0:
            continue
        alm[alm_index(lmax, l, 0)] = rng.normal(0.0, math.sqrt(C))
        if l > 0:
            sd = math.sqrt(C / 2.0)
            re = rng.normal(0.0, sd, size=l); im = rng.normal(0.0, sd, size=l)
            ms = np.arange(1, l + 1)
            alm[alm_index(lmax, l, ms)] = re + 1j * im
    return alm


def synalm_te_from_normals(cltt, clee, clbb, clte, z1, z2, zb, lmax: int):
    """The reference's correlated T/E/B draw (synfast_tqu.py:28-67) restated per l, with the unit
    normals supplied (complex, healpy layout; Re of the m = 0 entries used): per l the Cholesky
    factor of [[C_TT, C_TE], [C_TE, C_EE]] (:37-43; L21 = 0 when not positive definite),
    aT = L11 z1, aE = L21 z1 + L22 z2, aB = sqrt(C_BB) zb, the m > 0 components scaled to
    variance C/2 (:55, :60-64).  Returns (aT, aE, aB) in healpy layout."""
    n = alm_size(lmax)
    aT = np.zeros(n, dtype=np.complex128); aE = np.zeros_like(aT); aB = np.zeros_like(aT)
    for l in range(lmax + 1):
        Ctt, Cee, Cbb, Cte = float(cltt[l]), float(clee[l]), float(clbb[l]), float(clte[l])
        if Ctt <= 0 or Cee <= 0 or (Ctt * Cee - Cte * Cte) <= 0:
            L11, L21, L22 = math.sqrt(max(Ctt, 0.0)), 0.0, math.sqrt(max(Cee, 0.0))
        else:
            L11 = math.sqrt(Ctt)
            L21 = Cte / L11
            L22 = math.sqrt(Cee - L21 * L21)
        sb = math.sqrt(max(Cbb, 0.0))
        for m in range(l + 1):
            k = alm_index(lmax, l, m)
            if m == 0:
                a, b, c = z1[k].real, z2[k].real, zb[k].real
            else:
                h = math.sqrt(0.5)
                a, b, c = h * z1[k], h * z2[k], h * zb[k]
            aT[k] = L11 * a
            aE[k] = L21 * a + L22 * b
            aB[k] = sb * c
    return aT, aE, aB


# ----------------------------------------------------------------------------- pixel indexing
def _i64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int64))


def ring2nest(nside: int, ipix) -> np.ndarray:
    """HEALPix RING -> NESTED index (Gorski et al. 2005), the C oracle."""
    p = _i64(ipix); out = np.empty_like(p)
    _lib().orc_ring2nest(nside, p.size, p.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                         out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    return out


def nest2ring(nside: int, ipix) -> np.ndarray:
    p = _i64(ipix); out = np.empty_like(p)
    _lib().orc_nest2ring(nside, p.size, p.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                         out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    return out


def pix2ang(nside: int, ipix, nest: bool = False):
    p = _i64(ipix); th = np.empty(p.size); ph = np.empty(p.size)
    _lib().orc_pix2ang(nside, int(nest), p.size, p.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), _p(th), _p(ph))
    return th, ph


def ang2pix(nside: int, theta, phi, nest: bool = False) -> np.ndarray:
    th = _c(np.asarray(theta, dtype=np.float64)).reshape(-1); ph = _c(np.asarray(phi, dtype=np.float64)).reshape(-1)
    out = np.empty(th.size, dtype=np.int64)
    _lib().orc_ang2pix(nside, int(nest), th.size, _p(th), _p(ph), out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    return out


# ----------------------------------------------------------------------------- rotations
def wigner_d(l: int, beta: float) -> np.ndarray:
    """d^l_{mm'}(beta), [2l+1, 2l+1] with m, m' = -l..l (the C oracle's long double recursion)."""
    out = np.zeros((2 * l + 1) * (2 * l + 1))
    _lib().orc_wigner_d(int(l), float(beta), _p(out))
    return out.reshape(2 * l + 1, 2 * l + 1)


def rotate_alm_euler(alm, lmax: int, alpha: float, beta: float, gamma: float) -> np.ndarray:
    """a'_{lm} = sum_m' exp(-i m alpha) d^l_{mm'}(beta) exp(-i m' gamma) a_{lm'} (wigner_full.py:79-96,
    with the textbook d), healpy layout, a_{l,-m} = (-1)^m conj a_{lm}."""
    a = np.asarray(alm, dtype=np.complex128)
    out = np.zeros_like(a)
    for l in range(lmax + 1):
        m = np.arange(0, l + 1)
        pos = a[alm_index(lmax, l, m)]
        full = np.concatenate([((-1.0) ** m[:0:-1]) * np.conj(pos[:0:-1]), pos])  # m' = -l..l
        mm = np.arange(-l, l + 1)
        D = np.exp(-1j * mm[:, None] * alpha) * wigner_d(l, beta) * np.exp(-1j * mm[None, :] * gamma)
        out[alm_index(lmax, l, m)] = (D @ full)[l:]
    return out


def eval_alm(alm, lmax: int, theta, phi) -> np.ndarray:
    """f(theta, phi) = sum_lm a_lm Y_lm of a real field, at arbitrary points (direct sum)."""
    th = np.asarray(theta, dtype=np.float64); ph = np.asarray(phi, dtype=np.float64)
    a = np.asarray(alm, dtype=np.complex128)
    f = np.zeros(th.size)
    for m in range(lmax + 1):
        lam = lambda_lm(lmax, m, np.cos(th), np.sin(th))  # [npts, lmax+1]
        g = lam[:, m:] @ a[alm_index(lmax, np.arange(m, lmax + 1), m)]
        f += (1.0 if m == 0 else 2.0) * np.real(g * np.exp(1j * m * ph))
    return f
