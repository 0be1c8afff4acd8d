"""CPU tests of host-side logic: alm layouts and converters, geometry detection and host ring
tables, synalm's draw order, and the hellblast-style signatures' argument handling."""
import math

import numpy as np
import pytest
import torch


def test_healpy_index_and_size():
    from hellblast_b200 import alm_ops
    lmax = 7
    seen = set()
    for m in range(lmax + 1):
        for l in range(m, lmax + 1):
            seen.add(alm_ops.alm_index(lmax, l, m))
    assert seen == set(range(alm_ops.alm_size(lmax)))
    assert alm_ops.getlmax(alm_ops.alm_size(4095)) == 4095
    assert alm_ops.getlmax(alm_ops.alm_size(100, 30), mmax=30) == 100
    with pytest.raises(ValueError):
        alm_ops.getlmax(7)


def test_layout_round_trip_cpu(oracle):
    from hellblast_b200 import alm_ops
    lmax = 12
    rng = np.random.default_rng(0)
    a = rng.standard_normal(alm_ops.alm_size(lmax)) + 1j * rng.standard_normal(alm_ops.alm_size(lmax))
    t = torch.from_numpy(a)
    ref = alm_ops.healpy_to_ref(t, lmax)
    assert np.allclose(ref.numpy(), oracle.healpy_to_ref(a, lmax))
    back = alm_ops.ref_to_healpy(ref, lmax)
    assert np.array_equal(back.numpy(), a)
    # batched
    tb = torch.stack([t, 2 * t])
    assert np.array_equal(alm_ops.ref_to_healpy(alm_ops.healpy_to_ref(tb, lmax), lmax).numpy(), tb.numpy())


def test_almxfl_cpu():
    from hellblast_b200 import alm_ops
    lmax = 5
    a = torch.ones(alm_ops.alm_size(lmax), dtype=torch.complex128)
    fl = np.arange(lmax + 1, dtype=float)
    out = alm_ops.almxfl(a, fl)
    for m in range(lmax + 1):
        for l in range(m, lmax + 1):
            assert out[alm_ops.alm_index(lmax, l, m)] == l


def test_synalm_draw_order_matches_oracle(oracle):
    from hellblast_b200 import alm_ops
    lmax = 20
    cl = 1.0 / (np.arange(lmax + 1) + 1.0) ** 2
    cl[:2] = 0
    a = alm_ops.synalm(cl, seed=7, device="cpu").numpy()
    assert np.array_equal(a, oracle.synalm(cl, seed=7))


def test_host_ring_tables_match_oracle(oracle):
    from hellblast_b200 import geometry
    for nside in (1, 2, 8, 64, 512):
        for phi0 in ("healpix", "reference"):
            a = geometry.host_ring_tables(nside, phi0)
            b = oracle.ring_tables(nside, phi0=phi0)
            for k in ("z", "nphi", "phi0", "ring_start", "z_edges", "weights_dz"):
                assert np.array_equal(a[k], b[k]), (nside, phi0, k)
            # acos of numpy and of the C library may differ in the last bit
            assert np.allclose(a["theta"], b["theta"], rtol=0, atol=1e-15)


def test_detect_healpix():
    from hellblast_b200 import geometry
    t = geometry.host_ring_tables(16)
    assert geometry.detect_healpix(t["theta"], t["nphi"]) == 16
    assert geometry.detect_healpix(t["theta"][:-1], t["nphi"][:-1]) == 0
    th = t["theta"].copy(); th[3] += 1e-6
    assert geometry.detect_healpix(th, t["nphi"]) == 0


def test_nside_from_npix():
    from hellblast_b200 import transforms
    assert transforms.nside_from_npix(12 * 64 * 64) == 64
    with pytest.raises(ValueError):
        transforms.nside_from_npix(1000)


def test_precision_resolution():
    from hellblast_b200 import transforms
    assert transforms.resolve_precision(None, torch.float32) == torch.float32
    assert transforms.resolve_precision(None, torch.float64) == torch.float64
    assert transforms.resolve_precision("fp32", torch.float64) == torch.float32
    with pytest.raises(ValueError):
        transforms.resolve_precision("bf16", torch.float32)


def test_alias_phase_sign_is_exact_on_healpix_rings():
    """The ring kernels fold the aliases m0 + j n of a residue class with one phase product
    exp(i m0 phi0) when exp(i n phi0) is exactly +1 or -1 (else they take the per-alias phase).
    Both phi0 conventions put every HEALPix ring on the +-1 path: n phi0 / pi is an integer
    (0 or 1 mod 2) to within 1e-12, the tolerance of the device test."""
    from hellblast_b200 import geometry
    for phi0 in ("healpix", "reference"):
        for nside in (1, 2, 8, 64, 2048):
            t = geometry.host_ring_tables(nside, phi0)
            x = t["phi0"] / np.pi * t["nphi"]
            f = x - 2.0 * np.floor(0.5 * x)
            plus = (np.abs(f) < 1e-12) | (np.abs(f - 2.0) < 1e-12)
            minus = np.abs(f - 1.0) < 1e-12
            assert np.all(plus | minus), (phi0, nside)
            # the rings with a half-pixel shift (phi0 = pi / n) take s = -1
            assert np.array_equal(minus, np.abs(t["phi0"] * t["nphi"] - np.pi) < 1e-9), (phi0, nside)


def test_autotune_cache_round_trip(tmp_path, monkeypatch):
    """The autotune JSON cache stores and returns a result under its key (no GPU involved)."""
    from hellblast_b200 import batched
    monkeypatch.setenv("HB_AUTOTUNE_CACHE", str(tmp_path / "sub" / "tune.json"))
    key = (2048, 4095, 64, "NVIDIA B200")
    res = {"bf16": False, "wide": True, "candidates": [{"bf16": False, "wide": True, "ms": 140.0}]}
    batched._cache_store(key, res)
    assert batched._cache_load()[batched._cache_key(key)] == res
    batched._cache_store((1, 2, 3, "x"), {"bf16": True, "wide": False, "candidates": []})
    assert len(batched._cache_load()) == 2


def test_clear_caches_empties_plan_caches():
    import hellblast_b200 as hb
    from hellblast_b200 import batched, geometry
    geometry._cache[("probe",)] = object()
    batched._cache[("probe",)] = object()
    hb.clear_caches()
    assert not geometry._cache and not batched._cache
