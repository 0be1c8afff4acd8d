"""alm rotations (hellblast_b200.rotate over hb_wigner_d / hb_rotate_alm; the reference's
rotate_alm_euler.py, wigner_full.py, wigner_fast.py + wigner_d_fast.cu, rotate_alm.py).

The reference's closed-form d^l_{mm'} raises cos and sin of beta/2 to the wrong powers
(wigner_full.py:28-37, wigner_d_fast.cu:38-44), so its Euler rotation is not a rotation; parity is
pinned instead to (1) the textbook closed form of d (40 digits) through the oracle, (2) the
reference's own z rotation (rotate_alm.py, golden fixture), which is what the Euler rotation must
reduce to at beta = 0, and (3) the field itself: the rotated alm synthesise f(R^-1 n),
R = Rz(alpha) Ry(beta) Rz(gamma) (an active rotation), checked by direct evaluation.
Tolerances: FP64, 1e-12 for d and 1e-11 for rotated alm (relative to the largest entry)."""
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN

BETAS = [0.0, 0.4, 1.9, math.pi, 4.0, -0.7]


def test_oracle_wigner_d_matches_closed_form(oracle):
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.dps = 40
    f = mpmath.factorial

    def dc(l, m1, m2, th):
        t = mpmath.mpf(th) / 2
        c, s = mpmath.cos(t), mpmath.sin(t)
        pre = mpmath.sqrt(f(l + m1) * f(l - m1) * f(l + m2) * f(l - m2))
        tot = mpmath.mpf(0)
        for k in range(0, 2 * l + 1):
            if l + m2 - k < 0 or m1 - m2 + k < 0 or l - m1 - k < 0:
                continue
            tot += ((-1) ** (m1 - m2 + k) * pre / (f(l + m2 - k) * f(k) * f(m1 - m2 + k) * f(l - m1 - k))
                    * c ** (2 * l + m2 - m1 - 2 * k) * s ** (m1 - m2 + 2 * k))
        return float(tot)
    for l in (0, 1, 2, 5, 11):
        for b in BETAS:
            D = oracle.wigner_d(l, b)
            want = np.array([[dc(l, m1, m2, b) for m2 in range(-l, l + 1)] for m1 in range(-l, l + 1)])
            assert np.max(np.abs(D - want)) < 1e-14


def test_oracle_rotation_is_the_active_rotation_of_the_field(oracle):
    lmax = 12
    alm = oracle.synalm(1.0 / (np.arange(lmax + 1) + 2.0) ** 2, seed=3)
    al, be, ga = 0.3, 1.1, -0.7
    rot = oracle.rotate_alm_euler(alm, lmax, al, be, ga)
    rng = np.random.default_rng(0)
    th = np.arccos(rng.uniform(-1, 1, 30))
    ph = rng.uniform(0, 2 * np.pi, 30)
    n = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], 1)

    def Rz(a):
        return np.array([[np.cos(a), -np.sin(a), 0], [np.sin(a), np.cos(a), 0], [0, 0, 1]])

    def Ry(b):
        return np.array([[np.cos(b), 0, np.sin(b)], [0, 1, 0], [-np.sin(b), 0, np.cos(b)]])
    q = n @ (Rz(al) @ Ry(be) @ Rz(ga))  # rows R^-1 n
    tq = np.arccos(np.clip(q[:, 2], -1, 1))
    pq = np.arctan2(q[:, 1], q[:, 0])
    assert np.max(np.abs(oracle.eval_alm(rot, lmax, th, ph) - oracle.eval_alm(alm, lmax, tq, pq))) < 1e-13


@pytest.mark.gpu
def test_gpu_wigner_d_vs_oracle(oracle):
    import torch
    from hellblast_b200 import rotate
    for l in (0, 1, 2, 5, 17, 64, 300):
        got = rotate.wigner_d_full(torch.tensor(BETAS, dtype=torch.float64), l).cpu().numpy()
        for i, b in enumerate(BETAS):
            assert np.max(np.abs(got[i] - oracle.wigner_d(l, b))) < 1e-12, (l, b)


@pytest.mark.gpu
def test_gpu_rotation_vs_oracle_and_reference_z_rotation(oracle):
    import torch
    from hellblast_b200 import rotate
    lmax = 64
    alms = np.stack([oracle.synalm(1.0 / (np.arange(lmax + 1) + 2.0) ** 2, seed=s) for s in (1, 2)])
    t = torch.from_numpy(alms).cuda()
    for (al, be, ga) in [(0.3, 1.1, -0.7), (2.0, 4.2, 0.1), (0.0, math.pi, 0.0)]:
        got = rotate.rotate_alm_euler(t, al, be, ga).cpu().numpy()
        for b in range(2):
            want = oracle.rotate_alm_euler(alms[b], lmax, al, be, ga)
            assert np.max(np.abs(got[b] - want)) < 1e-11 * np.max(np.abs(want))
    # beta = 0: the z rotation by alpha + gamma
    z = np.load(os.path.join(GOLDEN, "rotate_z_ref.npz"))
    L, a = int(z["lmax"]), float(z["alpha"])
    ref_out = z["ref_out"]
    za = torch.from_numpy(z["alm"]).cuda()
    got = rotate.rotate_alm_z(za, a).cpu().numpy()
    assert np.max(np.abs(oracle.healpy_to_ref(got, L) - ref_out)) < 1e-15
    got_e = rotate.rotate_alm_euler(za, 0.3, 0.0, a - 0.3).cpu().numpy()
    assert np.max(np.abs(oracle.healpy_to_ref(got_e, L) - ref_out)) < 1e-13
    got_ref = rotate.rotate_alm_z(torch.from_numpy(oracle.healpy_to_ref(z["alm"], L)).cuda(), a,
                                  alm_layout="ref_lsquare").cpu().numpy()
    assert np.max(np.abs(got_ref - ref_out)) < 1e-15


@pytest.mark.gpu
def test_gpu_rotation_large_lmax_invariants():
    """lmax 2047: C_l preserved and the inverse rotation R(-gamma, -beta, -alpha) recovers the
    input (1e-10)."""
    import torch
    import hellblast_b200 as hb
    from hellblast_b200 import rotate
    lmax = 2047
    a = hb.synalm(1.0 / (np.arange(lmax + 1) + 10.0) ** 2, lmax=lmax, seed=5, device="cuda")
    r = rotate.rotate_alm_euler(a, 0.9, 2.3, -1.4)
    back = rotate.rotate_alm_euler(r, 1.4, -2.3, -0.9)
    assert float(torch.linalg.norm(back - a) / torch.linalg.norm(a)) < 1e-10
    c0, c1 = hb.alm2cl(a), hb.alm2cl(r)
    assert float(torch.max(torch.abs(c1 - c0) / c0[2:].min())) < 1e-9
