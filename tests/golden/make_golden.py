"""Generate tests/golden/*.npz by running the REFERENCE's own SHT path on the CPU.

Run in the build container (needs the reference tree; nothing at test time reads it):
    python tests/golden/make_golden.py [/path/to/reference]
(default: $HB_REFERENCE_DIR, else the build container's reference mount)

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
_ARGS = [a for a in sys.argv[1:] if not a.startswith("--")]
REF = _ARGS[0] if _ARGS else os.environ.get("HB_REFERENCE_DIR", "/root/reference")

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


def host_wigner_d_ms(theta, lmax, m, s):
    """The reference's wigner_d_ms_sum kernel (wigner_d_ms.cu:20-50) run as host code, in place
    of spin._wigner_d_ms (spin.py:19-26)."""
    th = np.ascontiguousarray(np.asarray(theta, dtype=np.float64))
    out = np.zeros((th.size, lmax + 1))
    lib.ref_wigner_d_ms_sum(th.ctypes.data_as(Dp), ctypes.c_int(th.size), ctypes.c_int(int(lmax)), ctypes.c_int(int(m)),
                            ctypes.c_int(int(s)), out.ctypes.data_as(Dp))
    return out.view(cp.GArr)


def closed_form_d(l, m1, m2, theta):
    """Wigner d^l_{m1 m2}(theta) from the textbook closed-form sum
    sum_k (-1)^(m1-m2+k) sqrt((l+m1)!(l-m1)!(l+m2)!(l-m2)!) / ((l+m2-k)! k! (m1-m2+k)! (l-m1-k)!)
    cos(theta/2)^(2l+m2-m1-2k) sin(theta/2)^(m1-m2+2k), evaluated with 40 significant digits.
    This is the function wigner_d_ms_sum sets out to compute with (m1, m2) = (m, s): its
    denominator is the one above, and the sign and the two powers are what the kernel gets wrong
    (wigner_d_ms.cu:42-45)."""
    import mpmath
    mpmath.mp.dps = 40
    t = mpmath.mpf(float(theta)) / 2
    c, sn = mpmath.cos(t), mpmath.sin(t)
    f = mpmath.factorial
    pre = mpmath.sqrt(f(l + m1) * f(l - m1) * f(l + m2) * f(l - m2))
    tot = mpmath.mpf(0)
    for k in range(0, 2 * l + 1):
        if l + m2 - k < 0 or m1 - m2 + k < 0 or l - m1 - k < 0:
            continue
        term = pre / (f(l + m2 - k) * f(k) * f(m1 - m2 + k) * f(l - m1 - k))
        tot += (-1) ** (m1 - m2 + k) * term * c ** (2 * l + m2 - m1 - 2 * k) * sn ** (m1 - m2 + 2 * k)
    return float(tot)


_d_cache = {}


def intended_wigner_d_ms(theta, lmax, m, s):
    """spin._wigner_d_ms with the Wigner d the reference intends, d^l_{m,s}(theta), l >= max(|m|,|s|)."""
    th = np.asarray(theta, dtype=np.float64)
    key = (th.tobytes(), int(lmax), int(m), int(s))
    if key not in _d_cache:
        out = np.zeros((th.size, lmax + 1))
        for l in range(max(abs(m), abs(s)), lmax + 1):
            for i, t in enumerate(th):
                out[i, l] = closed_form_d(l, int(m), int(s), t)
        _d_cache[key] = out
    return _d_cache[key].copy().view(cp.GArr)


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
import hellblast.spin as spin  # noqa: E402  (imports isht, patched above)


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


def spin_case(name, nside, lmax, seed, stock):
    """The reference's spin-2 analysis (map2alm_spin_gpu, eb_from_qu_gpu; spin.py:32-78) on Q/U
    maps of a Gaussian E/B draw, and its synthesis (qu_from_eb_gpu, spin.py:80-115) of an m = 0
    E/B input.  ``stock``: with the reference's own Wigner-d kernel, whose tables are stored
    too; otherwise with the closed-form d^l_{m,+-2} that kernel sets out to compute."""
    g = O.ring_tables(nside)
    cl = 1.0 / (np.arange(lmax + 1) + 2.0) ** 2
    cl[:2] = 0.0
    E_in = O.synalm(cl, seed=seed)
    B_in = O.synalm(0.3 * cl, seed=seed + 100)
    Q, U = O.alm2map_spin2(E_in, B_in, g, lmax)
    tabs = rt.HealpixRingTables(nside)
    w = tabs.weights_dz()
    th = np.asarray(tabs.theta_centers)
    spin._wigner_d_ms = host_wigner_d_ms if stock else intended_wigner_d_ms
    a2, am2 = spin.map2alm_spin_gpu(rings_of(Q, tabs), rings_of(U, tabs), tabs.theta_centers, tabs.nphi, w, lmax)
    E, B = spin.eb_from_qu_gpu(rings_of(Q, tabs), rings_of(U, tabs), tabs.theta_centers, tabs.nphi, w, lmax)
    out = dict(nside=nside, lmax=lmax, seed=seed, Q=Q, U=U, weights_dz=np.asarray(w), theta=th,
               ref_a2=np.asarray(a2), ref_am2=np.asarray(am2), ref_E=np.asarray(E), ref_B=np.asarray(B))
    if stock:
        # the d tables the reference's kernel produced, [m][ring][l] for s = +2 and s = -2
        out["ref_d_p2"] = np.stack([np.asarray(host_wigner_d_ms(th, lmax, m, 2)) for m in range(lmax + 1)])
        out["ref_d_m2"] = np.stack([np.asarray(host_wigner_d_ms(th, lmax, m, -2)) for m in range(lmax + 1)])
    else:
        # synthesis of an m = 0 input (where the reference's real-field Hermitian fill is harmless)
        keep = np.zeros(E_in.size, bool)
        keep[O.alm_index(lmax, np.arange(lmax + 1), 0)] = True
        E0 = np.where(keep, E_in, 0.0)
        B0 = np.where(keep, B_in, 0.0)
        cp.asrealarray = cp.real
        Qr, Ur = spin.qu_from_eb_gpu(O.healpy_to_ref(E0, lmax).view(cp.GArr), O.healpy_to_ref(B0, lmax).view(cp.GArr),
                                     tabs.theta_centers, tabs.nphi, lmax)
        out.update(E0_in=E0, B0_in=B0, ref_Q_m0=np.concatenate([np.asarray(r) for r in Qr]),
                   ref_U_m0=np.concatenate([np.asarray(r) for r in Ur]))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print("wrote", name, {k: getattr(v, "shape", v) for k, v in out.items()})


def pixel_case():
    """The reference's pixel-coordinate drivers (coords_ring.py, nested_pix2ang.py, nested_gpu.py)
    with their kernels (coords_ring.cu, nested_pix2ang.cu, nested_gpu.cu) run as host code."""
    U64 = ctypes.POINTER(ctypes.c_ulonglong)
    I32 = ctypes.POINTER(ctypes.c_int)
    LLp = ctypes.POINTER(ctypes.c_longlong)

    def arr(x):
        return np.ascontiguousarray(np.asarray(x))

    def k_ang2pix_ring(grid, block, args):
        th, ph, ridx, N, rs, nphi, ph0, out = (arr(a) if hasattr(a, "shape") else a for a in args)
        o = np.zeros(int(N), np.int64)
        lib.ref_ang2pix_ring_with_rings(th.ctypes.data_as(Dp), ph.ctypes.data_as(Dp), ridx.astype(np.int32).ctypes.data_as(I32),
                                        int(N), rs.astype(np.int64).ctypes.data_as(LLp),
                                        nphi.astype(np.int32).ctypes.data_as(I32), ph0.ctypes.data_as(Dp),
                                        o.ctypes.data_as(LLp))
        args[7][...] = o

    def k_pix2ang_ring(grid, block, args):
        ip, N, thc, rs, nphi, ph0, oth, oph = (arr(a) if hasattr(a, "shape") else a for a in args)
        t = np.zeros(int(N)); f = np.zeros(int(N))
        lib.ref_pix2ang_ring_batch(ip.astype(np.int64).ctypes.data_as(LLp), int(N), thc.ctypes.data_as(Dp),
                                   rs.astype(np.int64).ctypes.data_as(LLp), nphi.astype(np.int32).ctypes.data_as(I32),
                                   ph0.ctypes.data_as(Dp), t.ctypes.data_as(Dp), f.ctypes.data_as(Dp))
        args[6][...] = t
        args[7][...] = f

    def k_vec2pix_nest(grid, block, args):
        th, ph, N, nside, out = args
        o = np.zeros(int(N), np.uint64)
        lib.ref_vec2pix_nest_batch(arr(th).ctypes.data_as(Dp), arr(ph).ctypes.data_as(Dp), int(N), int(nside),
                                   o.ctypes.data_as(U64))
        out[...] = o

    def k_pix2ang_nest(grid, block, args):
        ip, N, nside, oth, oph = args
        t = np.zeros(int(N)); f = np.zeros(int(N))
        lib.ref_pix2ang_nest_batch(arr(ip).astype(np.uint64).ctypes.data_as(U64), int(N), int(nside),
                                   t.ctypes.data_as(Dp), f.ctypes.data_as(Dp))
        oth[...] = t
        oph[...] = f

    import hellblast.coords_ring as cr
    import hellblast.nested_gpu as ng
    import hellblast.nested_pix2ang as npa
    kern = {"ang2pix_ring_with_rings": k_ang2pix_ring, "pix2ang_ring_batch": k_pix2ang_ring,
            "vec2pix_nest_batch": k_vec2pix_nest, "pix2ang_nest_batch": k_pix2ang_nest}
    for mod in (cr, ng, npa):
        mod._get_fun = lambda src, fun: kern[fun]
    out = {}
    rng = np.random.default_rng(11)
    for nside in (1, 2, 4, 16, 1024):
        npix = 12 * nside * nside
        pix = np.arange(npix) if npix <= 3072 else np.sort(rng.choice(npix, 4000, replace=False))
        th_n, ph_n = npa.pix2ang_nest_gpu(nside, pix)
        mapper = cr.RingMapperGPU(nside)
        th_r, ph_r = mapper.pix2ang(pix)
        u = rng.uniform(-1.0, 1.0, 3000)
        th = np.arccos(u)
        ph = rng.uniform(0.0, 2.0 * np.pi, 3000)
        out.update({f"n{nside}_pix": pix, f"n{nside}_nest_theta": np.asarray(th_n), f"n{nside}_nest_phi": np.asarray(ph_n),
                    f"n{nside}_ring_theta": np.asarray(th_r), f"n{nside}_ring_phi": np.asarray(ph_r),
                    f"n{nside}_dir_theta": th, f"n{nside}_dir_phi": ph,
                    f"n{nside}_ref_ang2pix_ring": np.asarray(mapper.ang2pix(th, ph)),
                    f"n{nside}_ref_ang2pix_nest": np.asarray(ng.ang2pix_nest_gpu(th, ph, nside))})
    np.savez_compressed(os.path.join(HERE, "pixel_ref.npz"), **out)
    print("wrote pixel_ref", len(out))


def rotation_case():
    """The reference's z rotation of ref-layout alm (rotate_alm.py:5-19), its one rotation that is
    right as shipped (its Euler path's closed-form d is not a rotation matrix)."""
    import hellblast.rotate_alm as ra
    lmax = 20
    cl = 1.0 / (np.arange(lmax + 1) + 2.0) ** 2
    alm = O.synalm(cl, seed=9)
    ref = O.healpy_to_ref(alm, lmax)
    out = np.asarray(ra.rotate_alm_z(ref.view(cp.GArr), 0.7310, lmax))
    np.savez_compressed(os.path.join(HERE, "rotate_z_ref.npz"), lmax=lmax, alpha=0.7310, alm=alm, ref_out=out)
    print("wrote rotate_z_ref")


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
    if "--pixel-only" in sys.argv:
        pixel_case()
        sys.exit(0)
    if "--rotation-only" in sys.argv:
        rotation_case()
        sys.exit(0)
    # --spin-only: regenerate the spin-2 fixtures alone
    if "--spin-only" not in sys.argv:
        tables()
        case("sht_nside8_lmax16", 8, 16, seed=0)
        case("sht_nside32_lmax64", 32, 64, seed=1)
        case("sht_nside32_lmax85", 32, 85, seed=2)
        case("sht_nside16_lmax40_m0", 16, 40, seed=3, m0_only=True)
    spin_case("spin_stock_nside8_lmax20", 8, 20, seed=5, stock=True)
    spin_case("spin_dexact_nside8_lmax20", 8, 20, seed=6, stock=False)
    spin_case("spin_dexact_nside16_lmax40", 16, 40, seed=7, stock=False)
    pixel_case()
