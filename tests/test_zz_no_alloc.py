"""hb_map2alm_f32_noalloc (FP32 map2alm with a static device scratch, no allocation) against
hb_map2alm_f32 with a caller workspace, both called through the C ABI.  Collected last so it
also runs after every other test has used the library in the same process."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

# Both entry points run the same kernels in the same order; the tolerance only allows for
# nothing more than FP32 rounding differences.
TOL = 1e-6
SCRATCH = 64 << 20  # HB_NOALLOC_SCRATCH_BYTES


@pytest.fixture(scope="module")
def lib():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA GPU")
    from hellblast_b200 import _lib as L
    from hellblast_b200 import geometry as G
    return L, G


def _maps(nmaps, npix, seed):
    g = torch.Generator().manual_seed(seed)
    return torch.randn(nmaps, npix, generator=g, dtype=torch.float32).cuda()


def _with_workspace(L, plan, maps, nalm):
    nmaps = maps.shape[0]
    ws = torch.empty(plan.workspace_bytes(32, nmaps), dtype=torch.uint8, device="cuda")
    alm = torch.empty(nmaps, nalm, dtype=torch.complex64, device="cuda")
    L.call("hb_map2alm_f32", plan.handle, nmaps, maps.data_ptr(), None, alm.data_ptr(), ws.data_ptr(), ws.numel(),
           0, torch.cuda.current_stream().cuda_stream)
    return alm


def _no_alloc(L, plan, maps, nalm):
    nmaps = maps.shape[0]
    alm = torch.empty(nmaps, nalm, dtype=torch.complex64, device="cuda")
    L.call("hb_map2alm_f32_noalloc", plan.handle, nmaps, maps.data_ptr(), None, alm.data_ptr(), 0,
           torch.cuda.current_stream().cuda_stream)
    return alm


def _rel(a, b):
    return float(torch.linalg.norm((a - b).to(torch.complex128)) / torch.linalg.norm(b.to(torch.complex128)))


def test_no_alloc_matches_workspace_entry_point_two_calls(lib):
    L, G = lib
    # call 1: nside 256, lmax 511, 16 maps = exactly the 64 MiB of scratch
    g1 = G.healpix(256)
    p1 = G.plan(g1, 511, precision=32)
    assert p1.workspace_bytes(32, 16) == SCRATCH
    nalm1 = int(L.lib().hb_alm_size(511, 511))
    m1 = _maps(16, g1.npix, 1)
    a1 = _no_alloc(L, p1, m1, nalm1)
    # call 2 right after: a different geometry and size, so the scratch still holds call 1's
    # entries beyond what call 2 writes
    g2 = G.healpix(64)
    p2 = G.plan(g2, 150, 120, precision=32)
    nalm2 = int(L.lib().hb_alm_size(150, 120))
    m2 = _maps(3, g2.npix, 2)
    a2 = _no_alloc(L, p2, m2, nalm2)
    torch.cuda.synchronize()
    r1 = _with_workspace(L, p1, m1, nalm1)
    r2 = _with_workspace(L, p2, m2, nalm2)
    torch.cuda.synchronize()
    assert np.isfinite(a1.abs().max().item()) and np.isfinite(a2.abs().max().item())
    assert _rel(a1, r1) < TOL
    assert _rel(a2, r2) < TOL
    # and once more on call 1's input after call 2 changed the scratch
    a3 = _no_alloc(L, p1, m1, nalm1)
    torch.cuda.synchronize()
    assert _rel(a3, r1) < TOL


def test_no_alloc_unpaired_rings_after_a_larger_call(lib):
    """A generic grid with an odd ring count and no mirror symmetry: every ring is unpaired, so
    the south half of each F(m, pair) entry is the kernel's own zero, not a value left in the
    shared scratch by the larger call made just before."""
    L, G = lib
    g1 = G.healpix(256)
    p1 = G.plan(g1, 511, precision=32)
    nalm1 = int(L.lib().hb_alm_size(511, 511))
    a1 = _no_alloc(L, p1, _maps(16, g1.npix, 3), nalm1)
    rng = np.random.default_rng(7)
    nr = 37
    theta = np.sort(rng.uniform(0.05, 3.0, nr))
    nphi = 2 * rng.integers(8, 120, nr)
    w = rng.uniform(0.01, 0.1, nr)
    g2 = G.generic(theta, nphi, w, phi0=rng.uniform(0.0, 0.3, nr))
    p2 = G.plan(g2, 90, precision=32)
    nalm2 = int(L.lib().hb_alm_size(90, 90))
    m2 = _maps(5, int(nphi.sum()), 4)
    for _ in range(2):
        a2 = _no_alloc(L, p2, m2, nalm2)
        torch.cuda.synchronize()
        r2 = _with_workspace(L, p2, m2, nalm2)
        torch.cuda.synchronize()
        assert np.isfinite(a1.abs().max().item())
        assert _rel(a2, r2) < TOL
        a1 = _no_alloc(L, p1, _maps(16, g1.npix, 5), nalm1)  # dirty the scratch again


def test_no_alloc_rejects_calls_beyond_the_scratch(lib):
    L, G = lib
    g = G.healpix(256)
    p = G.plan(g, 511, precision=32)
    assert p.workspace_bytes(32, 17) > SCRATCH
    maps = torch.zeros(17, g.npix, dtype=torch.float32, device="cuda")
    alm = torch.empty(17, int(L.lib().hb_alm_size(511, 511)), dtype=torch.complex64, device="cuda")
    rc = L.lib().hb_map2alm_f32_noalloc(p.handle, 17, maps.data_ptr(), None, alm.data_ptr(), 0,
                                        torch.cuda.current_stream().cuda_stream)
    assert rc == L.HB_ERR_INVALID
    assert "static scratch" in L.lib().hb_last_error_string().decode()
    with pytest.raises(ValueError):
        L.call("hb_map2alm_f32_noalloc", None, 1, maps.data_ptr(), None, alm.data_ptr(), 0, None)
    small = G.plan(G.healpix(8), 8, precision=32)
    rc = L.lib().hb_map2alm_f32_noalloc(small.handle, 65536, maps.data_ptr(), None, alm.data_ptr(), 0,
                                        torch.cuda.current_stream().cuda_stream)
    assert rc == L.HB_ERR_INVALID
    assert "nmaps" in L.lib().hb_last_error_string().decode()
