"""Spin-2 parity with the reference's own spin.py (map2alm_spin_gpu / eb_from_qu_gpu,
spin.py:32-78; qu_from_eb_gpu, spin.py:80-115), through fixtures made by running the reference
(tests/golden/make_golden.py, ``spin_case``).

Three fixtures:
  * ``spin_stock_nside8_lmax20``: the reference exactly as shipped, with its own Wigner-d kernel
    (wigner_d_ms.cu:20-50) run as host code.  That kernel does not compute d^l_{m,s}: its sign
    and its two powers of cos/sin(theta/2) are wrong (wigner_d_ms.cu:42-45; e.g. it returns 0 for
    d^2_{0,2} and -4.9 for d^4_{1,2}).  The fixture also stores the d tables it produced, and the
    oracle's restatement of the assembly around them (map2alm_spin2_ref_compat with those tables:
    FFT of Q +- iU over nphi, the m cut, per-ring bins m < nphi, weights, 2 pi sqrt((2l+1)/4pi),
    E/B) must reproduce the stock output exactly.
  * ``spin_dexact_nside{8,16}_lmax{20,40}``: the same reference code with its d generator
    replaced by the d^l_{m,+-2}(theta) it sets out to compute (the textbook closed-form sum with
    the kernel's own denominator, evaluated with 40 digits).  Every other line of spin.py runs as
    shipped.  These pin the oracle's and the CUDA kernels' spin-2 transforms.

Convention mapping (checked here, written out in transforms.map2alm_spin2):
  * the reference contracts a(+-2) with sqrt((2l+1)/4pi) d^l_{m,+-2}, where healpy (and this
    repository) uses d^l_{m,-+2}; both use E = -(a2 + a-2)/2, B = i (a2 - a-2)/2.  The difference
    is the U -> -U polarisation convention: E_ref(Q, U) = E(Q, -U), B_ref(Q, U) = -B(Q, -U);
  * the reference has no phi0 phase and no alias fold, keeps bins m < nphi_r of each ring and
    computes orders m <= max_r min(mmax, nphi_r // 2) only (spin.py:53,57,65);
  * its synthesis uses a2 = -(E - iB) (spin.py:84), so for the m = 0 input where its real-field
    spectrum fill is harmless, Q_ref = Q(E, B) and U_ref = -U(E, B).

Tolerances: oracle <= 1e-12; CUDA FP64 <= 1e-10 (max-abs over max-abs); CUDA FP32 <= 1e-5
(L2 norm).
"""
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN

DEXACT = ["spin_dexact_nside8_lmax20", "spin_dexact_nside16_lmax40"]


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def relmax(a, b):
    a = np.asarray(a); b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def rel2(a, b):
    a = np.asarray(a); b = np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _ref_cut(oracle, alm_hp, lmax, nside):
    """healpy-layout alm -> the reference's l(l+1)+m layout with its m cut (spin.py:53,57)."""
    out = oracle.healpy_to_ref(np.asarray(alm_hp), lmax)
    mcut = min(lmax, 2 * nside)
    ls = np.floor(np.sqrt(np.arange(out.size))).astype(int)
    ms = np.arange(out.size) - ls * (ls + 1)
    out[ms > mcut] = 0
    return out


# ------------------------------------------------------------------------------------ oracle
def test_oracle_assembly_reproduces_stock_reference(oracle):
    d = load("spin_stock_nside8_lmax20")
    nside, lmax = int(d["nside"]), int(d["lmax"])
    g = oracle.ring_tables(nside)
    a2, am2, E, B = oracle.map2alm_spin2_ref_compat(d["Q"], d["U"], g, lmax, weights=d["weights_dz"],
                                                    d_tables=(d["ref_d_p2"], d["ref_d_m2"]))
    for mine, ref in ((a2, "ref_a2"), (am2, "ref_am2"), (E, "ref_E"), (B, "ref_B")):
        assert relmax(mine, d[ref]) < 1e-12, ref


def test_oracle_d_recursion_matches_closed_form():
    """The oracle's spin-weighted recursion against the closed-form Wigner d (40 digits) on a
    sample of (theta, m, l), both s = +2 and s = -2."""
    mpmath = pytest.importorskip("mpmath")
    from oracle import sht_oracle as O
    mpmath.mp.dps = 40
    f = mpmath.factorial

    def d_closed(l, m1, m2, th):
        t = mpmath.mpf(th) / 2
        c, sn = mpmath.cos(t), mpmath.sin(t)
        pre = mpmath.sqrt(f(l + m1) * f(l - m1) * f(l + m2) * f(l - m2))
        tot = mpmath.mpf(0)
        for k in range(0, 2 * l + 1):
            if l + m2 - k < 0 or m1 - m2 + k < 0 or l - m1 - k < 0:
                continue
            tot += ((-1) ** (m1 - m2 + k) * pre / (f(l + m2 - k) * f(k) * f(m1 - m2 + k) * f(l - m1 - k))
                    * c ** (2 * l + m2 - m1 - 2 * k) * sn ** (m1 - m2 + 2 * k))
        return float(tot)

    lmax = 24
    th = np.array([0.05, 0.7, 1.3, math.pi / 2, 2.2, 3.09])
    nl = np.sqrt((2.0 * np.arange(lmax + 1) + 1.0) / (4.0 * math.pi))
    for m in (0, 1, 2, 3, 7, 24):
        lp2, lm2 = O.spin2_lambda(lmax, m, th)
        for i, t in enumerate(th):
            for l in range(max(m, 2), lmax + 1):
                assert abs(lm2[i, l] / nl[l] - d_closed(l, m, 2, t)) < 1e-12, (m, l, t, "+2")
                assert abs(lp2[i, l] / nl[l] - d_closed(l, m, -2, t)) < 1e-12, (m, l, t, "-2")


@pytest.mark.parametrize("name", DEXACT)
def test_oracle_matches_reference_with_exact_d(oracle, name):
    d = load(name)
    nside, lmax = int(d["nside"]), int(d["lmax"])
    g = oracle.ring_tables(nside)
    a2, am2, E, B = oracle.map2alm_spin2_ref_compat(d["Q"], d["U"], g, lmax, weights=d["weights_dz"])
    for mine, ref in ((a2, "ref_a2"), (am2, "ref_am2"), (E, "ref_E"), (B, "ref_B")):
        assert relmax(mine, d[ref]) < 1e-12, ref


@pytest.mark.parametrize("name", DEXACT)
def test_healpy_convention_mapping(oracle, name):
    """The healpy-convention oracle transform with (Q, -U), no phase, no fold, the m cut ==
    the reference's (E, -B); its synthesis of the m = 0 input == (Q_ref, -U_ref)."""
    d = load(name)
    nside, lmax = int(d["nside"]), int(d["lmax"])
    g = oracle.ring_tables(nside)
    E, B = oracle.map2alm_spin2(d["Q"], -d["U"], g, lmax, weights=d["weights_dz"], phase=False, fold=False)
    assert relmax(_ref_cut(oracle, E, lmax, nside), d["ref_E"]) < 1e-12
    assert relmax(-_ref_cut(oracle, B, lmax, nside), d["ref_B"]) < 1e-12
    Q, U = oracle.alm2map_spin2(d["E0_in"], d["B0_in"], g, lmax)
    assert relmax(Q, d["ref_Q_m0"]) < 1e-12
    assert relmax(-U, d["ref_U_m0"]) < 1e-12


# ------------------------------------------------------------------------------------- CUDA
@pytest.mark.gpu
@pytest.mark.parametrize("name", DEXACT)
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_cuda_spin_matches_reference(oracle, name, prec):
    """hellblast_b200.spin.eb_from_qu_gpu / map2alm_spin_gpu (ref_compat=True, ref layout) against
    the reference's eb_from_qu_gpu / map2alm_spin_gpu output."""
    import torch
    import hellblast_b200 as hb
    d = load(name)
    nside, lmax = int(d["nside"]), int(d["lmax"])
    tabs = hb.HealpixRingTables(nside, phi0="reference")
    dt = torch.float64 if prec == "fp64" else torch.float32
    Q = torch.from_numpy(d["Q"]).cuda().to(dt)
    U = torch.from_numpy(d["U"]).cuda().to(dt)
    rs = [int(x) for x in tabs.ring_start]
    qr = [Q[rs[r]:rs[r + 1]] for r in range(tabs.Nr)]
    ur = [U[rs[r]:rs[r + 1]] for r in range(tabs.Nr)]
    E, B = hb.spin.eb_from_qu_gpu(qr, ur, tabs.theta_centers, tabs.nphi, d["weights_dz"], lmax,
                                  ref_compat=True, alm_layout="ref_lsquare")
    a2, am2 = hb.spin.map2alm_spin_gpu(qr, ur, tabs.theta_centers, tabs.nphi, d["weights_dz"], lmax,
                                       ref_compat=True, alm_layout="ref_lsquare")
    got = [x.cpu().numpy().astype(np.complex128) for x in (E, B, a2, am2)]
    for mine, ref in zip(got, ("ref_E", "ref_B", "ref_a2", "ref_am2")):
        if prec == "fp64":
            assert relmax(mine, d[ref]) < 1e-10, ref
        else:
            assert rel2(mine, d[ref]) < 1e-5, ref


@pytest.mark.gpu
@pytest.mark.parametrize("name", DEXACT)
def test_cuda_spin_synthesis_m0_matches_reference(oracle, name):
    import torch
    import hellblast_b200 as hb
    d = load(name)
    nside, lmax = int(d["nside"]), int(d["lmax"])
    tabs = hb.HealpixRingTables(nside, phi0="reference")
    E0 = torch.from_numpy(oracle.healpy_to_ref(d["E0_in"], lmax)).cuda()
    B0 = torch.from_numpy(oracle.healpy_to_ref(d["B0_in"], lmax)).cuda()
    Q, U = hb.spin.qu_from_eb_gpu(E0, B0, tabs.theta_centers, tabs.nphi, lmax, flat=True, ref_compat=True,
                                  alm_layout="ref_lsquare")
    assert relmax(Q.cpu().numpy(), d["ref_Q_m0"]) < 1e-10
    assert relmax(U.cpu().numpy(), d["ref_U_m0"]) < 1e-10
