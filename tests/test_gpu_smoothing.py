"""GPU tests of the smoothing pipeline (map2alm -> almxfl -> alm2map; smoothing.py and beams.py
of the reference): FP64 against the oracle, and the batched path whose filter is fused into the
tensor-core analysis store against the per-map FP64 pipeline."""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hb():
    import hellblast_b200
    return hellblast_b200


def test_gaussian_beam_formula(hb):
    lmax, fwhm = 64, 0.05
    sigma = fwhm / math.sqrt(8 * math.log(2))
    l = np.arange(lmax + 1)
    ref = np.exp(-0.5 * l * (l + 1) * sigma ** 2)
    got = hb.smoothing.gaussian_beam_fl(lmax, fwhm).cpu().numpy()
    np.testing.assert_allclose(got, ref, rtol=1e-14)


def test_smooth_map_fp64_vs_oracle(hb, oracle):
    nside, lmax, fwhm = 16, 40, 0.2
    g = oracle.ring_tables(nside)
    cl = 1.0 / (np.arange(lmax + 1) + 1.0) ** 2
    m = oracle.alm2map(oracle.synalm(cl, seed=11), g, lmax)
    bl = hb.smoothing.gaussian_beam_fl(lmax, fwhm).cpu().numpy()
    a = oracle.map2alm(m, g, lmax)
    ls = np.concatenate([np.arange(mm, lmax + 1) for mm in range(lmax + 1)])
    ref = oracle.alm2map(a * bl[ls], g, lmax)
    got = hb.smoothing.smooth_map(torch.from_numpy(m).cuda(), nside, lmax=lmax, fwhm=fwhm).cpu().numpy()
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-10


def test_smooth_batch_fused_filter(hb):
    """float32 batch: the filter applied inside the batched map2alm store equals almxfl of the
    FP64 per-map pipeline (within the FP32 / split tolerance)."""
    nside, lmax, nmaps, fwhm = 32, 63, 6, 0.1
    cl = 1.0 / (np.arange(lmax + 1) + 10.0) ** 2
    a = torch.stack([hb.synalm(cl, lmax=lmax, seed=30 + i, device="cuda") for i in range(nmaps)])
    maps = hb.hp_compat.alm2map(a, nside, lmax=lmax)
    got = hb.smoothing.smooth_map(maps.float(), nside, lmax=lmax, fwhm=fwhm)
    ref = torch.stack([hb.smoothing.smooth_map(maps[i], nside, lmax=lmax, fwhm=fwhm) for i in range(nmaps)])
    assert got.shape == ref.shape and got.dtype == torch.float32
    assert float(torch.linalg.norm(got.double() - ref) / torch.linalg.norm(ref)) < 1e-5
    # and the fused alm against almxfl of the unfused batched map2alm
    bp = hb.batched.plan(nside, lmax, nmaps)
    fl = hb.smoothing.gaussian_beam_fl(lmax, fwhm)
    fused = bp.map2alm(maps.float(), fl=fl.float()).reshape(nmaps, -1)
    plain = hb.almxfl(bp.map2alm(maps.float()).reshape(nmaps, -1), fl.float(), lmax=lmax)
    assert float(torch.linalg.norm(fused - plain) / torch.linalg.norm(plain)) < 1e-6
