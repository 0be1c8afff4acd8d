"""GPU tests of the FP32 ring-FFT stage alone (hb_ring_analysis / hb_ring_synthesis through the
C ABI) against the oracle's numpy ring FFTs (sht_raw.py:38-43 and isht.py:16-24 of the
reference, with the phi0 phase and alias fold).

On HEALPix grids the equatorial belt and the polar rings from ring index 64 on run on the
pair-packed kernels (one complex FFT per ring pair; Bluestein for the polar rings, whose nphi = 4i
is not a power of two), the smaller polar rings on the general ring kernels.  The polar rings
with 2048 < nphi < 8192 (nside >= 513) run split in four quarter-length Bluestein transforms
(ring_quad_*_kernel); the nside 1024 and 2048 cases cover both of those classes.  The cases cover
both conventions of phi0 (HEALPix: s = 0 or 1 in phi0 = s pi / nphi; the reference's: s = 1 or
2), the unpaired equator ring, the flags, and the three alias regimes (mmax < nphi/2,
nphi/2 <= mmax < nphi, mmax >= nphi).  Tolerance: 1e-5 relative (L2), FP32.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.fixture(scope="module")
def hb():
    import hellblast_b200
    return hellblast_b200


def rel2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _pairs(g):
    """ring index of the north / south ring of each pair of a HEALPix grid (south -1: unpaired)."""
    nr = g["nr"]
    npairs = (nr + 1) // 2
    north = np.arange(npairs)
    south = nr - 1 - north
    south[south == north] = -1
    return north, south


CASES = [(128, "healpix", 200, 0), (256, "healpix", 767, 0), (256, "reference", 767, 0), (256, "healpix", 1500, 0),
         (256, "healpix", 767, 1), (256, "reference", 300, 2), (256, "healpix", 1100, 3),
         (1024, "healpix", 2047, 0), (2048, "healpix", 4095, 0), (2048, "reference", 4095, 2)]


def _nmaps(nside):
    return 2 if nside <= 256 else 1


@pytest.mark.parametrize("nside,phi0,lmax,flags", CASES)
def test_ring_analysis_fp32_vs_oracle(hb, oracle, nside, phi0, lmax, flags):
    from hellblast_b200 import _lib as L
    from hellblast_b200 import geometry as G
    g = G.healpix(nside, phi0=phi0)
    p = G.plan(g, lmax, precision=64)
    go = oracle.ring_tables(nside, phi0=phi0)
    nmaps = _nmaps(nside)
    rng = np.random.default_rng(nside + lmax + flags)
    maps = rng.standard_normal((nmaps, g.npix)).astype(np.float32)
    F = torch.empty(nmaps, lmax + 1, g.npairs, 2, dtype=torch.complex64, device="cuda")
    L.call("hb_ring_analysis", p.handle, 32, nmaps, torch.from_numpy(maps).cuda().data_ptr(), None, F.data_ptr(), flags,
           torch.cuda.current_stream().cuda_stream)
    F = F.cpu().numpy()
    north, south = _pairs(go)
    for b in range(nmaps):
        ref = oracle.ring_analysis(maps[b].astype(np.float64), go, lmax, weights=go["weights_dz"],
                                   phase=not (flags & L.HB_F_NOPHASE), fold=not (flags & L.HB_F_NOFOLD))
        want = np.zeros((lmax + 1, g.npairs, 2), dtype=np.complex128)
        want[:, :, 0] = ref[:, north]
        has = south >= 0
        want[:, has, 1] = ref[:, south[has]]
        assert rel2(F[b], want) < TOL
        assert np.all(F[b][:, ~has, 1] == 0)


@pytest.mark.parametrize("nside,phi0,lmax,flags", [c for c in CASES if not (c[3] & 2)])
def test_ring_synthesis_fp32_vs_oracle(hb, oracle, nside, phi0, lmax, flags):
    from hellblast_b200 import _lib as L
    from hellblast_b200 import geometry as G
    g = G.healpix(nside, phi0=phi0)
    p = G.plan(g, lmax, precision=64)
    go = oracle.ring_tables(nside, phi0=phi0)
    nmaps = _nmaps(nside)
    rng = np.random.default_rng(3 * nside + lmax + flags)
    Gm = (rng.standard_normal((nmaps, lmax + 1, g.npairs, 2)) + 1j * rng.standard_normal((nmaps, lmax + 1, g.npairs, 2)))
    Gm = Gm.astype(np.complex64)
    north, south = _pairs(go)
    has = south >= 0
    Gm[:, :, ~has, 1] = 0  # the unpaired equator's south slot is not data
    out = torch.empty(nmaps, g.npix, dtype=torch.float32, device="cuda")
    L.call("hb_ring_synthesis", p.handle, 32, nmaps, torch.from_numpy(Gm).cuda().data_ptr(), out.data_ptr(), flags,
           torch.cuda.current_stream().cuda_stream)
    out = out.cpu().numpy()
    for b in range(nmaps):
        Go = np.zeros((lmax + 1, go["nr"]), dtype=np.complex128)
        Go[:, north] = Gm[b, :, :, 0]
        Go[:, south[has]] = Gm[b, :, has, 1].T
        ref = oracle.ring_synthesis(Go, go, phase=not (flags & L.HB_F_NOPHASE))
        assert rel2(out[b].astype(np.float64), ref) < TOL


def test_unpaired_south_slot_garbage_is_ignored(hb, oracle):
    """The south slot of the unpaired equator pair may hold anything (here NaN): the equator ring
    and every other ring come out finite and equal to the clean input's."""
    from hellblast_b200 import _lib as L
    from hellblast_b200 import geometry as G
    nside, lmax = 256, 600
    g = G.healpix(nside)
    p = G.plan(g, lmax, precision=64)
    rng = np.random.default_rng(11)
    Gm = (rng.standard_normal((1, lmax + 1, g.npairs, 2)) + 1j * rng.standard_normal((1, lmax + 1, g.npairs, 2)))
    Gm = Gm.astype(np.complex64)
    eq = g.npairs - 1
    clean = Gm.copy()
    clean[:, :, eq, 1] = 0
    dirty = Gm.copy()
    dirty[:, :, eq, 1] = np.nan
    outs = []
    for x in (clean, dirty):
        out = torch.empty(1, g.npix, dtype=torch.float32, device="cuda")
        L.call("hb_ring_synthesis", p.handle, 32, 1, torch.from_numpy(x).cuda().data_ptr(), out.data_ptr(), 0,
               torch.cuda.current_stream().cuda_stream)
        outs.append(out.cpu().numpy())
    assert np.all(np.isfinite(outs[1]))
    assert np.array_equal(outs[0], outs[1])
