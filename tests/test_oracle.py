"""CPU tests of the FP64 oracle: pinned against the reference's own outputs (golden fixtures
made by running the reference through tests/golden/make_golden.py), against scipy's spherical
harmonics, against the eth-operator definition of spin-2 harmonics, and for its internal
consistency (adjoints, round trips)."""
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN

CASES = ["sht_nside8_lmax16", "sht_nside32_lmax64", "sht_nside32_lmax85", "sht_nside16_lmax40_m0"]


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def relmax(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name", CASES)
def test_ref_compat_matches_reference(oracle, name):
    """Oracle in the reference's conventions == reference sht_fallback / sht_raw (<= 1e-12)."""
    d = load(name)
    nside, lmax = int(d["nside"]), int(d["lmax"])
    g = oracle.ring_tables(nside, phi0="reference")
    fb = oracle.map2alm_ref_compat(d["map"], g, lmax, flavour="fallback")
    raw = oracle.map2alm_ref_compat(d["map"], g, lmax, flavour="raw")
    assert relmax(oracle.healpy_to_ref(fb, lmax), d["ref_sht_fallback"]) < 1e-12
    assert relmax(oracle.healpy_to_ref(raw, lmax), d["ref_sht_raw"]) < 1e-12
    assert relmax(oracle.alm2cl(fb, lmax), d["ref_alm2cl_fallback"]) < 1e-12
    assert relmax(oracle.alm2cl(raw, lmax), d["ref_anafast_ring"]) < 1e-12


@pytest.mark.parametrize("name", CASES)
def test_correct_mode_m0_matches_reference(oracle, name):
    """Where the reference is right (m = 0 entries, no phi0 dependence), the corrected transform
    agrees with it."""
    d = load(name)
    nside, lmax = int(d["nside"]), int(d["lmax"])
    g = oracle.ring_tables(nside)
    a = oracle.map2alm(d["map"], g, lmax)
    l = np.arange(lmax + 1)
    assert relmax(a[oracle.alm_index(lmax, l, 0)], d["ref_sht_fallback"][l * (l + 1)]) < 1e-12


def test_isht_m0_matches_reference(oracle):
    d = load("sht_nside16_lmax40_m0")
    nside, lmax = int(d["nside"]), int(d["lmax"])
    g = oracle.ring_tables(nside)
    mp = oracle.alm2map(d["alm_in"], g, lmax, phase=False)
    assert relmax(mp, d["ref_isht_map"]) < 1e-12


def test_ring_tables_match_reference(oracle):
    import hashlib
    d = np.load(os.path.join(GOLDEN, "ring_tables.npz"))
    for nside in (1, 2, 4, 8, 16, 32, 64):
        g = oracle.ring_tables(nside, phi0="reference")
        assert np.array_equal(g["nphi"], d[f"n{nside}_nphi"])
        assert np.array_equal(g["ring_start"], d[f"n{nside}_ring_start"])
        for k, ref in (("z", "z_centers"), ("theta", "theta_centers"), ("phi0", "phi_center0"), ("z_edges", "z_edges")):
            assert np.array_equal(g[k], d[f"n{nside}_{ref}"]), (nside, k)
    for nside in (128, 256, 512, 1024, 2048, 4096, 8192):
        g = oracle.ring_tables(nside, phi0="reference")
        h = hashlib.sha256(g["nphi"].astype(np.int32).tobytes() + g["ring_start"].astype(np.int64).tobytes())
        assert h.hexdigest() == str(d[f"n{nside}_int_sha256"])


def test_healpix_phi0_is_half_pixel_off_reference(oracle):
    for nside in (2, 8, 64):
        a, b = oracle.ring_tables(nside), oracle.ring_tables(nside, phi0="reference")
        dphi = 2 * math.pi / a["nphi"]
        eq = (np.arange(1, 4 * nside) >= nside) & (np.arange(1, 4 * nside) <= 3 * nside)
        assert np.allclose((b["phi0"] - a["phi0"])[eq], 0.5 * dphi[eq], rtol=0, atol=1e-15)
        assert np.array_equal(a["phi0"][~eq], b["phi0"][~eq])


def test_lambda_vs_scipy(oracle):
    from scipy.special import sph_harm_y
    th = np.linspace(0.01, 3.13, 29)
    lmax = 60
    for m in (0, 1, 2, 9, 33, 60):
        lam = oracle.lambda_lm(lmax, m, np.cos(th), np.sin(th))
        for l in range(m, lmax + 1):
            assert np.max(np.abs(lam[:, l] - sph_harm_y(l, m, th, 0.0).real)) < 1e-12


def test_lambda_no_overflow_high_l(oracle):
    """Normalised recursion with log-scaled start: finite up to l = 8191 (the reference's
    factorial norms overflow above l + m ~ 170, sht_raw.py:26-28)."""
    th = np.array([1e-3, 0.3, 1.2, math.pi / 2])
    lam = oracle.lambda_lm(8191, 4000, np.cos(th), np.sin(th))
    assert np.all(np.isfinite(lam))
    assert np.max(np.abs(lam[:, 4000:])) < 100.0
    assert np.all(lam[0, :] == 0.0)  # lambda_{l,4000}(1e-3) underflows entirely


def _eth2(l, m, t, bar, h=1e-4):
    from scipy.special import sph_harm_y
    Y = lambda t: sph_harm_y(l, m, t, 0.0).real  # noqa: E731
    sgn = -1.0 if bar else 1.0

    def f1(t):
        d = (-Y(t + 2 * h) + 8 * Y(t + h) - 8 * Y(t - h) + Y(t - 2 * h)) / (12 * h)
        return -(d - sgn * m * Y(t) / np.sin(t))

    gfun = lambda t: f1(t) / np.sin(t)  # noqa: E731
    d = (-gfun(t + 2 * h) + 8 * gfun(t + h) - 8 * gfun(t - h) + gfun(t - 2 * h)) / (12 * h)
    return -np.sin(t) * (d - sgn * m * gfun(t) / np.sin(t))


def test_spin2_lambda_matches_eth_definition(oracle):
    """_{+-2}Y_lm = sqrt((l-2)!/(l+2)!) eth^2 / ethbar^2 Y_lm (Zaldarriaga & Seljak 1997)."""
    th = np.array([0.3, 0.9, 1.4, 2.2, 2.9])
    for l in range(2, 8):
        for m in range(0, l + 1):
            p2, m2 = oracle.spin2_lambda(l, m, th)
            nrm = math.sqrt(math.factorial(l - 2) / math.factorial(l + 2))
            assert np.max(np.abs(p2[:, l] - nrm * _eth2(l, m, th, bar=False))) < 1e-7
            assert np.max(np.abs(m2[:, l] - nrm * _eth2(l, m, th, bar=True))) < 1e-7


def test_oracle_adjoint_identities(oracle):
    nside, lmax = 8, 20
    g = oracle.ring_tables(nside)
    rng = np.random.default_rng(5)
    x = rng.standard_normal(g["npix"])
    n = oracle.alm_size(lmax)
    y = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    y[oracle.alm_index(lmax, np.arange(lmax + 1), 0)] = y[oracle.alm_index(lmax, np.arange(lmax + 1), 0)].real
    A = oracle.map2alm(x, g, lmax)
    lhs = np.sum(A.real * y.real + A.imag * y.imag)
    assert abs(lhs - np.dot(x, oracle.map2alm_adjoint(y, g, lmax))) < 1e-12 * abs(lhs)
    S = oracle.alm2map(y, g, lmax)
    St = oracle.alm2map_adjoint(x, g, lmax)
    assert abs(np.dot(S, x) - np.sum(St.real * y.real + St.imag * y.imag)) < 1e-12 * abs(np.dot(S, x))


def test_oracle_round_trip_converges(oracle):
    nside, lmax = 16, 31
    g = oracle.ring_tables(nside)
    cl = 1.0 / (np.arange(lmax + 1) + 1.0) ** 2
    alm = oracle.synalm(cl, seed=0)
    mp = oracle.alm2map(alm, g, lmax)
    w = oracle.uniform_weights(g)
    a = oracle.map2alm(mp, g, lmax, weights=w)
    errs = []
    for _ in range(3):
        a = a + oracle.map2alm(mp - oracle.alm2map(a, g, lmax), g, lmax, weights=w)
        errs.append(np.linalg.norm(a - alm) / np.linalg.norm(alm))
    assert errs[-1] < 5e-5 and errs[-1] < errs[0]


def test_alias_fold_exact_for_band_limited_ring(oracle):
    """A pure e^{i m phi} harmonic with m > nphi/2 on a small ring is folded onto m mod nphi."""
    g = oracle.generic_geometry([1.0], [8], phi0=[0.3])
    m = 11
    phi = 0.3 + 2 * math.pi * np.arange(8) / 8
    f = np.cos(m * phi)
    F = oracle.ring_analysis(f, g, mmax=16, weights=None)
    # DFT of the sampled cosine at bins (11 mod 8) = 3 and 5; phase e^{-i m phi0}
    ref = np.array([np.sum(f * np.exp(-1j * k * phi)) for k in range(17)])
    assert np.allclose(F[:, 0], ref, atol=1e-12)


def test_spin2_analysis_at_selected_m_matches_full(oracle):
    """The m-subset spin-2 analysis (used to spot-check transforms too large for the full
    oracle) reproduces the full analysis at those m."""
    nside, lmax = 16, 40
    g = oracle.ring_tables(nside)
    cl = 1.0 / (np.arange(lmax + 1) + 10.0) ** 2
    E = oracle.synalm(cl, seed=1)
    B = oracle.synalm(0.1 * cl, seed=2)
    Q, U = oracle.alm2map_spin2(E, B, g, lmax)
    E1, B1 = oracle.map2alm_spin2(Q, U, g, lmax)
    ms = [0, 1, 2, 3, 17, 40]
    Es, Bs = oracle.map2alm_spin2_ms(Q, U, g, lmax, ms)
    for j, m in enumerate(ms):
        idx = oracle.alm_index(lmax, np.arange(m, lmax + 1), m)
        np.testing.assert_allclose(Es[j, m:], E1[idx], rtol=0, atol=1e-13)
        np.testing.assert_allclose(Bs[j, m:], B1[idx], rtol=0, atol=1e-13)
