"""Generate tests/golden/*.npz by running the REFERENCE's own SHT path on the CPU.

Run in the build container (needs the reference tree; nothing at test time reads it):
    python tests/golden/make_golden.py [/path/to/reference]

How the reference runs here (no CuPy, no GPU):
  * ``tests/golden/_cupy_shim`` provides a numpy-backed ``cupy`` module;
  * the reference's CUDA kernels ``build_ring_tables`` (ring_tables_healpix.cu) and
    ``plm_recurrence`` (legendre.cu) are compiled as host C++ by ``oracle/build_ref.sh`` into
    ``oracle/_ref/libhbref.so`` and patched in where the reference would load them with
    ``cp.RawModule`` (ring_tables.py:6-15, sht_raw.py:16-24);
  * ``np.math = math`` for sht_fallback.py:8 (numpy>=2 removed np.math);
  * isht.py imports ``_alm_norm``/``_compute_legendre_block`` from ``.sht`` which does not
    export them (isht.py:3): the generator sets them on the ``sht`` module before importing.
The input maps are made by the FP64 oracle's alm2map (healpy phi0) and stored in the
fixture, so the tests need neither the reference nor this script.
"""
import ctypes
import hashlib
import math
import os
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"

sys.path.insert(0, REPO)
from oracle import sht_oracle as O  # noqa: E402

np.math = math
sys.path.insert(0, os.path.join(HERE, "_cupy_shim"))
import cupy as cp  # noqa: E402  (the shim)

tmp = tempfile.mkdtemp()
os.symlink(REF, os.path.join(tmp, "hellblast"))
sys.path.insert(0, tmp)

lib = ctypes.CDLL(os.path.join(REPO, "oracle", "_ref", "libhbref.so"))
Dp = ctypes.POINTER(ctypes.c_double)


def host_ring_tables(grid, block, args):
    nside, z, th, nphi, ph, rs, ze = args
    lib.ref_build_ring_tables(ctypes.c_longlong(int(nside)), z.ctypes.data_as(Dp), th.ctypes.data_as(Dp),
                              nphi.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ph.ctypes.data_as(Dp),
                              rs.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)), ze.ctypes.data_as(Dp))


def host_legendre_block(x_cos, lmax, m):
    x = np.ascontiguousarray(np.asarray(x_cos, dtype=np.float64))
    P = np.zeros((x.size, lmax + 1))
    lib.ref_plm_recurrence(x.ctypes.data_as(Dp), ctypes.c_int(x.size), ctypes.c_int(lmax), ctypes.c_int(m),
                           P.ctypes.data_as(Dp))
    return P.view(cp.GArr)


import hellblast.ring_tables as rt  # noqa: E402
rt._get_fun = lambda src, fun: host_ring_tables
import hellblast.sht_raw as sht_raw  # noqa: E402
sht_raw._compute_legendre_block = host_legendre_block
import hellblast.sht_fallback as sht_fallback  # noqa: E402
import hellblast.sht as sht  # noqa: E402
sht._alm_norm = sht_raw._alm_norm
sht._compute_legendre_block = host_legendre_block
import hellblast.isht as isht  # noqa: E402
import hellblast.alm_ops as alm_ops  # noqa: E402
import hellblast.anafast  # noqa: E402,F401
anafast = sys.modules["hellblast.anafast"]  # the package rebinds the name `anafast` (__init__.py:127)
assert sht.map2alm_gpu is sht_raw.map2alm_gpu


def rings_of(flat, tabs):
    out = []
    nphi = tabs.nphi.get(); rs = tabs.ring_start.get()
    for r in range(tabs.Nr):
        out.append(np.asarray(flat[rs[r]:rs[r] + nphi[r]]).view(cp.GArr))
    return out


def case(name, nside, lmax, seed, m0_only=False):
    g = O.ring_tables(nside)
    cl = 1.0 / (np.arange(lmax + 1) + 1.0) ** 2
    cl[:2] = 0.0
    alm = O.synalm(cl, seed=seed)
    if m0_only:
        keep = np.zeros(alm.size, bool); keep[O.alm_index(lmax, np.arange(lmax + 1), 0)] = True
        alm[~keep] = 0.0
    mp = O.alm2map(alm, g, lmax)
    tabs = rt.HealpixRingTables(nside)
    rings = rings_of(mp, tabs)
    w = tabs.weights_dz()
    raw = np.asarray(sht_raw.map2alm_gpu(rings, tabs.theta_centers, tabs.nphi, w, lmax))
    fb = np.asarray(sht_fallback.map2alm_gpu(rings, tabs.theta_centers, tabs.nphi, w, lmax))
    cl_fb = np.asarray(alm_ops.alm2cl(fb, lmax=lmax))
    ana = np.asarray(anafast.anafast_ring(rings, tabs.theta_centers, tabs.nphi, w, lmax))
    out = dict(nside=nside, lmax=lmax, seed=seed, alm_in=alm, map=mp, ref_sht_raw=raw,
               ref_sht_fallback=fb, ref_alm2cl_fallback=cl_fb, ref_anafast_ring=ana,
               weights_dz=np.asarray(w))
    if m0_only:
        ref_alm = O.healpy_to_ref(alm, lmax)
        maprings = isht.alm2map_gpu(ref_alm.view(cp.GArr), tabs.theta_centers, tabs.nphi, lmax)
        out["ref_isht_map"] = np.concatenate([np.asarray(r) for r in maprings])
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print("wrote", name, {k: getattr(v, "shape", v) for k, v in out.items()})


def tables():
    out = {}
    for nside in (1, 2, 4, 8, 16, 32, 64):
        t = rt.HealpixRingTables(nside).dump_host()
        for k in ("z_centers", "theta_centers", "nphi", "phi_center0", "ring_start", "z_edges"):
            out[f"n{nside}_{k}"] = t[k]
    for nside in (128, 256, 512, 1024, 2048, 4096, 8192):
        t = rt.HealpixRingTables(nside).dump_host()
        h = hashlib.sha256(np.ascontiguousarray(t["nphi"]).tobytes() + np.ascontiguousarray(t["ring_start"]).tobytes())
        out[f"n{nside}_int_sha256"] = np.array(h.hexdigest())
        out[f"n{nside}_npix"] = np.array(t["npix"])
    np.savez_compressed(os.path.join(HERE, "ring_tables.npz"), **out)
    print("wrote ring_tables")


if __name__ == "__main__":
    tables()
    case("sht_nside8_lmax16", 8, 16, seed=0)
    case("sht_nside32_lmax64", 32, 64, seed=1)
    case("sht_nside32_lmax85", 32, 85, seed=2)
    case("sht_nside16_lmax40_m0", 16, 40, seed=3, m0_only=True)
