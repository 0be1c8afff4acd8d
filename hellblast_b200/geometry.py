"""Ring geometries (device-resident, created once, immutable): HEALPix grids and arbitrary
iso-latitude ring sets, the latter being what hellblast's ``map2alm_gpu(rings, thetas,
nphi_per_ring, weights_dz, lmax)`` receives (sht_raw.py:30)."""
from __future__ import annotations

import ctypes
import hashlib
import math
import threading

import numpy as np

from . import _lib as L

_registry: dict[int, "Geometry"] = {}
_cache: dict[tuple, "Geometry"] = {}
_lock = threading.Lock()
_next_id = [1]


class Geometry:
    """Owns an ``hb_geom`` handle.  ``gid`` is the integer the torch ops take."""

    def __init__(self, handle: int, nside: int, theta: np.ndarray, nphi: np.ndarray, phi0: np.ndarray,
                 weights: np.ndarray, device_index: int):
        self.handle = ctypes.c_void_p(handle)
        self.nside = nside
        self.theta = theta
        self.nphi = nphi
        self.phi0 = phi0
        self.weights = weights
        self.device_index = device_index
        nr, npix, npairs, ns = (ctypes.c_int64() for _ in range(4))
        L.call("hb_geom_info", self.handle, ctypes.byref(nr), ctypes.byref(npix), ctypes.byref(npairs),
               ctypes.byref(ns))
        self.nr, self.npix, self.npairs = nr.value, npix.value, npairs.value
        self.ring_start = np.zeros(self.nr + 1, dtype=np.int64)
        self.ring_start[1:] = np.cumsum(self.nphi)
        with _lock:
            self.gid = _next_id[0]
            _next_id[0] += 1
            _registry[self.gid] = self

    def fft_launches(self, precision: int = 32) -> int:
        """Ring-FFT kernel launches per direction (one per transform-length class)."""
        n = ctypes.c_int(0)
        L.call("hb_geom_fft_launches", self.handle, int(precision), ctypes.byref(n))
        return n.value

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            if self.handle:
                L.lib().hb_geom_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


def get(gid: int) -> Geometry:
    return _registry[gid]


class Plan:
    """Owns an ``hb_plan``: a geometry, (lmax, mmax) and, for FP32, the FP64-computed recursion
    checkpoints.  ``pid`` is the integer the torch ops take."""

    def __init__(self, geom: Geometry, lmax: int, mmax: int, flags: int):
        self.geom = geom
        self.lmax, self.mmax, self.flags = int(lmax), int(mmax), int(flags)
        out = ctypes.c_void_p()
        L.call("hb_plan_create", geom.handle, self.lmax, self.mmax, self.flags, ctypes.byref(out))
        self.handle = out
        self.nbytes = int(L.lib().hb_plan_bytes(out))
        with _lock:
            self.pid = _next_id[0]
            _next_id[0] += 1
            _plans[self.pid] = self

    @property
    def npix(self):
        return self.geom.npix

    def workspace_bytes(self, precision: int, nmaps: int, spin: bool = False) -> int:
        fn = "hb_spin2_workspace_size" if spin else "hb_sht_workspace_size"
        return int(getattr(L.lib(), fn)(self.handle, precision, nmaps))

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            if self.handle:
                L.lib().hb_plan_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


_plans: dict[int, Plan] = {}


def get_plan(pid: int) -> Plan:
    return _plans[pid]


def plan(geom: Geometry, lmax: int, mmax: int | None = None, precision: int = 64, spin: bool = False) -> Plan:
    """Cached plan for (geometry, lmax, mmax); FP32 plans carry the checkpoint tables (scalar, or
    spin-2 with ``spin=True``)."""
    mmax = lmax if mmax is None else mmax
    flags = 0
    if precision == 32:
        flags = L.HB_PLAN_SPIN2_FP32 if spin else L.HB_PLAN_FP32
    key = ("plan", geom.gid, int(lmax), int(mmax), flags)
    with _lock:
        p = _cache.get(key)
    if p is None:
        p = Plan(geom, lmax, mmax, flags)
        with _lock:
            _cache[key] = p
    return p


def _current_device() -> int:
    import torch
    return torch.cuda.current_device()


def healpix(nside: int, phi0: str = "healpix", weights: str = "dz") -> Geometry:
    """HEALPix RING geometry.  ``phi0``: "healpix" (default) or "reference" (the reference's
    +1/2-pixel equatorial phi0, ring_tables_healpix.cu:25-27).  ``weights``: "dz" (the
    reference's ring weights_dz, ring_tables.py:39-40) or "uniform" (4*pi/npix per pixel)."""
    nside = int(nside)
    if nside < 1 or nside & (nside - 1):
        raise ValueError("nside must be a power of 2")
    dev = _current_device()
    key = ("healpix", nside, phi0, weights, dev)
    with _lock:
        g = _cache.get(key)
    if g is not None:
        return g
    out = ctypes.c_void_p()
    L.call("hb_geom_create_healpix", nside, L.HB_PHI0_HEALPIX if phi0 == "healpix" else L.HB_PHI0_REFERENCE,
           L.HB_WEIGHTS_DZ if weights == "dz" else L.HB_WEIGHTS_UNIFORM, ctypes.byref(out))
    t = host_ring_tables(nside, phi0)
    w = t["weights_dz"] if weights == "dz" else 2.0 * t["nphi"] / (12.0 * nside * nside)
    g = Geometry(out.value, nside, t["theta"], t["nphi"], t["phi0"], w, dev)
    with _lock:
        _cache[key] = g
    return g


def generic(theta, nphi, weights, phi0=None) -> Geometry:
    """Geometry of arbitrary rings (host arrays).  Cached by content."""
    theta = np.ascontiguousarray(np.asarray(theta, dtype=np.float64))
    nphi = np.ascontiguousarray(np.asarray(nphi, dtype=np.int32))
    weights = np.ascontiguousarray(np.asarray(weights, dtype=np.float64))
    phi0 = np.zeros_like(theta) if phi0 is None else np.ascontiguousarray(np.asarray(phi0, dtype=np.float64))
    if not (theta.size == nphi.size == weights.size == phi0.size):
        raise ValueError("theta, nphi, weights and phi0 must have one entry per ring")
    dev = _current_device()
    h = hashlib.sha1()
    for a in (theta, nphi, weights, phi0):
        h.update(a.tobytes())
    key = ("generic", h.hexdigest(), dev)
    with _lock:
        g = _cache.get(key)
    if g is not None:
        return g
    out = ctypes.c_void_p()
    L.call("hb_geom_create", theta.size, theta.ctypes.data, nphi.ctypes.data, phi0.ctypes.data,
           weights.ctypes.data, ctypes.byref(out))
    g = Geometry(out.value, 0, theta, nphi, phi0, weights, dev)
    with _lock:
        _cache[key] = g
    return g


def host_ring_tables(nside: int, phi0: str = "healpix") -> dict:
    """Host copy of the HEALPix ring tables (closed forms of ring_tables_healpix.cu:14-51)."""
    nside = int(nside)
    nr = 4 * nside - 1
    i = np.arange(1, nr + 1, dtype=np.int64)
    ip = np.minimum(i, 4 * nside - i)
    z = np.where(i < nside, 1.0 - (i * i).astype(np.float64) / (3.0 * float(nside * nside)),
                 np.where(i <= 3 * nside, (2 * nside - i).astype(np.float64) * (2.0 / (3.0 * nside)),
                          -(1.0 - (ip * ip).astype(np.float64) / (3.0 * float(nside * nside)))))
    nphi = np.where(ip < nside, 4 * ip, 4 * nside).astype(np.int32)
    dphi = 2.0 * math.pi / nphi
    s = (i - nside) & 1
    if phi0 == "healpix":
        p0 = np.where(ip < nside, 0.5 * dphi, np.where(s == 1, 0.0, 0.5 * dphi))
    else:
        p0 = np.where(ip < nside, 0.5 * dphi, (1.0 - 0.5 * s) * dphi)
    rs = np.zeros(nr + 1, dtype=np.int64)
    rs[1:] = np.cumsum(nphi)
    ze = np.empty(nr + 1)
    ze[0] = 1.0
    ze[1:-1] = 0.5 * (z[:-1] + z[1:])
    ze[-1] = -1.0
    return dict(z=z, theta=np.arccos(np.clip(z, -1.0, 1.0)), nphi=nphi, phi0=p0, ring_start=rs, z_edges=ze,
                weights_dz=ze[:-1] - ze[1:])


def detect_healpix(theta: np.ndarray, nphi: np.ndarray) -> int:
    """nside if (theta, nphi) is a full HEALPix RING grid, else 0."""
    nr = int(np.asarray(nphi).size)
    if (nr + 1) % 4:
        return 0
    nside = (nr + 1) // 4
    if nside < 1 or nside & (nside - 1):
        return 0
    t = host_ring_tables(nside)
    if not np.array_equal(np.asarray(nphi, dtype=np.int64), t["nphi"].astype(np.int64)):
        return 0
    if not np.allclose(np.asarray(theta, dtype=np.float64), t["theta"], rtol=0, atol=1e-12):
        return 0
    return nside
