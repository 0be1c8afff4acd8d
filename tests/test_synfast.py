"""synfast (hellblast_b200.synfast; the reference's synfast_tqu.py:28-128): the correlated T/E/B
draw against the oracle's per-l restatement of the reference's Cholesky algebra (same unit
normals, exact), its statistics, and the T/Q/U synthesis of filtered alm against the FP64
oracle (FP64 <= 1e-10, FP32 <= 1e-5)."""
import math

import numpy as np
import pytest
import torch


def _spectra(lmax):
    l = np.arange(lmax + 1, dtype=np.float64)
    tt = 1.0 / (l + 10.0) ** 2
    ee = 0.1 * tt
    bb = 0.01 * tt
    te = 0.25 * np.sqrt(tt * ee) * np.cos(l / 7.0)
    tt[:2] = ee[:2] = bb[:2] = te[:2] = 0.0
    te[5] = 2.0 * math.sqrt(tt[5] * ee[5])  # not positive definite at l = 5: L21 = 0 there
    return tt, ee, bb, te


def test_te_algebra_matches_oracle_restatement(oracle):
    from hellblast_b200 import synfast
    lmax = 40
    tt, ee, bb, te = _spectra(lmax)
    n = oracle.alm_size(lmax)
    rng = np.random.default_rng(3)
    z = [rng.standard_normal(n) + 1j * rng.standard_normal(n) for _ in range(3)]
    got = synfast.te_from_normals(tt, ee, bb, te, *(torch.from_numpy(x)[None] for x in z), lmax)
    want = oracle.synalm_te_from_normals(tt, ee, bb, te, *z, lmax)
    for g_, w_ in zip(got, want):
        assert np.max(np.abs(g_[0].numpy() - w_)) <= 1e-15 * max(1.0, np.max(np.abs(w_)))


@pytest.mark.gpu
def test_draw_statistics():
    """C_l^XY of 8 draws at lmax 300, binned over 20 l: within 5 sigma of the input."""
    from hellblast_b200 import alm_ops, synfast
    lmax = 300
    tt, ee, bb, te = _spectra(lmax)
    aT, aE, aB = synfast.synalm_te(tt, ee, bb, te, lmax, seed=11, nsims=8)
    est = {k: alm_ops.alm2cl(a, b).mean(0).cpu().numpy() for k, (a, b) in
           {"tt": (aT, None), "ee": (aE, None), "bb": (aB, None), "te": (aT, aE)}.items()}
    true = {"tt": tt, "ee": ee, "bb": bb, "te": te}
    for k in est:
        for lo in range(10, lmax - 19, 20):
            sl = slice(lo, lo + 20)
            nmodes = 8 * np.sum(2 * np.arange(lo, lo + 20) + 1)
            if k == "te":
                var = np.mean(tt[sl] * ee[sl] + te[sl] ** 2)
            else:
                var = 2 * np.mean(true[k][sl] ** 2)
            sigma = math.sqrt(var / nmodes)
            assert abs(np.mean(est[k][sl]) - np.mean(true[k][sl])) < 5 * sigma, (k, lo)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32", 1e-5)])
def test_synthesis_of_filtered_alm_vs_oracle(oracle, precision, tol):
    from hellblast_b200 import synfast
    nside, lmax, fwhm = 32, 80, 0.05
    tt, ee, bb, te = _spectra(lmax)
    aT, aE, aB = (a[0].cpu().numpy() for a in synfast.synalm_te(tt, ee, bb, te, lmax, seed=2))
    T, Q, U, fT, fE, fB = synfast.synfast_tqu({}, nside, lmax, fwhm=fwhm, alms=(aT, aE, aB), return_alm=True,
                                               precision=precision)
    sigma = fwhm / math.sqrt(8.0 * math.log(2.0))
    l = np.arange(lmax + 1)
    bl = np.exp(-0.5 * l * (l + 1) * sigma * sigma)
    ls = np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])
    g = oracle.ring_tables(nside)
    want_T = oracle.alm2map(aT * bl[ls], g, lmax)
    want_Q, want_U = oracle.alm2map_spin2(aE * bl[ls], aB * bl[ls], g, lmax)
    assert np.allclose(fT.cpu().numpy(), aT * bl[ls], rtol=0, atol=1e-15)
    for got, want in ((T, want_T), (Q, want_Q), (U, want_U)):
        got = got.double().cpu().numpy()
        assert np.linalg.norm(got - want) / np.linalg.norm(want) < tol


@pytest.mark.gpu
def test_noise_and_shapes():
    from hellblast_b200 import synfast
    nside, lmax = 16, 40
    tt, ee, bb, te = _spectra(lmax)
    cls = {"tt": tt, "ee": ee, "bb": bb, "te": te}
    T0, Q0, U0 = synfast.synfast_tqu(cls, nside, seed=5)
    T1, Q1, U1 = synfast.synfast_tqu(cls, nside, seed=5, sigmaT=2.0, sigmaQ=3.0, sigmaU=4.0)
    assert T0.shape == (12 * nside * nside,)
    for a, b, s in ((T0, T1, 2.0), (Q0, Q1, 3.0), (U0, U1, 4.0)):
        d = (b - a).double()
        assert abs(float(d.std()) - s) < 0.1 * s
    T, Q, U = synfast.synfast_tqu({"tt": tt}, nside, seed=1, nsims=3)
    assert T.shape == (3, 12 * nside * nside) and float(Q.abs().max()) == 0.0
    with pytest.raises(ValueError):
        synfast.synfast_tqu({"tt": tt, "ee": ee}, nside)
