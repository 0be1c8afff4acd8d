"""GPU tests of the spin-2 transforms and of the differentiable path: parity with the FP64
oracle, exact adjoints (dot-product tests, a dense transform matrix at small nside), and
central finite differences in FP64."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
TOL32 = 1e-5


def relmax(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def rel2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def npy(t):
    return t.detach().cpu().numpy()


@pytest.fixture(scope="module")
def hb():
    import hellblast_b200
    return hellblast_b200


def _eb(oracle, lmax, seed):
    cl = 1.0 / (np.arange(lmax + 1) + 10.0) ** 2
    cl[:2] = 0.0
    E = oracle.synalm(cl, seed=seed)
    B = oracle.synalm(0.1 * cl, seed=seed + 100)
    return E, B


@pytest.mark.parametrize("nside,lmax", [(2, 7), (8, 23), (32, 95), (16, 120)])
def test_spin2_fp64_vs_oracle(hb, oracle, nside, lmax):
    g = oracle.ring_tables(nside)
    E, B = _eb(oracle, lmax, nside)
    Q, U = oracle.alm2map_spin2(E, B, g, lmax)
    q, u = hb.hp_compat.alm2map_spin(torch.from_numpy(E).cuda(), torch.from_numpy(B).cuda(), nside=nside, lmax=lmax)
    assert relmax(npy(q), Q) < TOL64 and relmax(npy(u), U) < TOL64
    E1, B1 = oracle.map2alm_spin2(Q, U, g, lmax)
    e, b = hb.hp_compat.map2alm_spin(torch.from_numpy(Q).cuda(), torch.from_numpy(U).cuda(), lmax=lmax)
    assert relmax(npy(e), E1) < TOL64 and relmax(npy(b), B1) < TOL64


@pytest.mark.parametrize("nside,lmax", [(16, 47), (128, 383)])
def test_spin2_fp32_vs_oracle(hb, oracle, nside, lmax):
    g = oracle.ring_tables(nside)
    E, B = _eb(oracle, lmax, nside + 1)
    Q, U = oracle.alm2map_spin2(E, B, g, lmax)
    q, u = hb.hp_compat.alm2map_spin(torch.from_numpy(E).cuda().to(torch.complex64),
                                     torch.from_numpy(B).cuda().to(torch.complex64), nside=nside, lmax=lmax)
    assert rel2(npy(q), Q) < TOL32 and rel2(npy(u), U) < TOL32
    E1, B1 = oracle.map2alm_spin2(Q, U, g, lmax)
    e, b = hb.hp_compat.map2alm_spin(torch.from_numpy(Q).cuda().float(), torch.from_numpy(U).cuda().float(), lmax=lmax)
    assert rel2(npy(e), E1) < TOL32 and rel2(npy(b), B1) < TOL32


def test_spin_wrappers_reference_names(hb, oracle):
    nside, lmax = 8, 16
    g = oracle.ring_tables(nside)
    E, B = _eb(oracle, lmax, 3)
    Q, U = oracle.alm2map_spin2(E, B, g, lmax)
    tabs = hb.HealpixRingTables(nside)
    a2, am2 = hb.map2alm_spin_gpu(torch.from_numpy(Q).cuda(), torch.from_numpy(U).cuda(), tabs.theta_centers,
                                  tabs.nphi, tabs.weights_dz(), lmax)
    e, b = hb.eb_from_qu_gpu(torch.from_numpy(Q).cuda(), torch.from_numpy(U).cuda(), tabs.theta_centers,
                             tabs.nphi, tabs.weights_dz(), lmax)
    # E = -(a2 + a-2)/2, B = i (a2 - a-2)/2  (spin.py:76-77)
    assert relmax(npy(-(a2 + am2) / 2), npy(e)) < 1e-14
    assert relmax(npy(1j * (a2 - am2) / 2), npy(b)) < 1e-14
    Qr, Ur = hb.qu_from_eb_gpu(e, b, tabs.theta_centers, tabs.nphi, lmax)
    assert len(Qr) == tabs.Nr
    E1, B1 = oracle.map2alm_spin2(Q, U, g, lmax)
    Q1, U1 = oracle.alm2map_spin2(E1, B1, g, lmax)
    assert relmax(npy(torch.cat(Qr)), Q1) < TOL64 and relmax(npy(torch.cat(Ur)), U1) < TOL64


def _rand_alm(hb, lmax, seed, dtype=torch.complex128):
    g = torch.Generator().manual_seed(seed)
    n = hb.alm_size(lmax)
    a = torch.complex(torch.randn(n, generator=g, dtype=torch.float64), torch.randn(n, generator=g, dtype=torch.float64))
    return a.to(dtype).cuda()


def _dot_c(a, b):
    return float((a.real * b.real + a.imag * b.imag).sum())


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_adjoint_dot_products(hb, prec):
    nside, lmax = 32, 80
    rt = torch.float64 if prec == "fp64" else torch.float32
    ct = torch.complex128 if prec == "fp64" else torch.complex64
    tol = 1e-12 if prec == "fp64" else 1e-5
    g = hb.geometry.healpix(nside)
    pid = hb.geometry.plan(g, lmax, precision=32 if prec == "fp32" else 64).pid
    x = torch.randn(1, g.npix, dtype=torch.float64, generator=torch.Generator().manual_seed(0)).to(rt).cuda()
    y = _rand_alm(hb, lmax, 1, ct)[None]
    A_x = torch.ops.hb.map2alm(x, pid, None, 0)
    At_y = torch.ops.hb.map2alm_adjoint(y, pid, None, 0)
    lhs, rhs = _dot_c(A_x, y), float((x * At_y).sum())
    assert abs(lhs - rhs) <= tol * abs(lhs)
    S_y = torch.ops.hb.alm2map(y, pid, 0)
    St_x = torch.ops.hb.alm2map_adjoint(x, pid, 0)
    # imaginary parts of m = 0 do not enter a real map: drop them from y for the identity
    y0 = y.clone()
    y0[:, :lmax + 1] = y0[:, :lmax + 1].real.to(ct)
    lhs, rhs = float((torch.ops.hb.alm2map(y0, pid, 0) * x).sum()), _dot_c(St_x, y0)
    assert abs(lhs - rhs) <= tol * abs(lhs)
    assert torch.all(St_x[:, :lmax + 1].imag == 0)
    del S_y


def test_spin_adjoint_dot_products(hb):
    nside, lmax = 16, 40
    g = hb.geometry.healpix(nside)
    pid = hb.geometry.plan(g, lmax, precision=64, spin=True).pid
    gen = torch.Generator().manual_seed(3)
    Q = torch.randn(1, g.npix, dtype=torch.float64, generator=gen).cuda()
    U = torch.randn(1, g.npix, dtype=torch.float64, generator=gen).cuda()
    e, b = _rand_alm(hb, lmax, 4)[None], _rand_alm(hb, lmax, 5)[None]
    E, B = torch.ops.hb.map2alm_spin2(Q, U, pid, None, 0)
    gQ, gU = torch.ops.hb.map2alm_spin2_adjoint(e, b, pid, None, 0)
    lhs = _dot_c(E, e) + _dot_c(B, b)
    rhs = float((Q * gQ).sum() + (U * gU).sum())
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
    q, u = torch.ops.hb.alm2map_spin2(e, b, pid, 0)
    ge, gb = torch.ops.hb.alm2map_spin2_adjoint(Q, U, pid, 0)
    # l < 2 and the m = 0 imaginary parts do not enter Q/U
    mask = torch.ones_like(e.real)
    for m in range(0, 2):
        for l in range(m, 2):
            mask[:, hb.alm_index(lmax, l, m)] = 0
    e0 = e * mask
    b0 = b * mask
    e0[:, :lmax + 1] = e0[:, :lmax + 1].real.to(e.dtype)
    b0[:, :lmax + 1] = b0[:, :lmax + 1].real.to(e.dtype)
    q0, u0 = torch.ops.hb.alm2map_spin2(e0, b0, pid, 0)
    lhs = float((q0 * Q).sum() + (u0 * U).sum())
    rhs = _dot_c(ge, e0) + _dot_c(gb, b0)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
    del q, u


def test_dense_matrix_small_nside(hb, oracle):
    """Build alm2map and map2alm as explicit matrices at nside 2 (column by column through the
    GPU kernels) and check the adjoint kernels reproduce their transposes exactly."""
    nside, lmax = 2, 5
    g = hb.geometry.healpix(nside)
    pid = hb.geometry.plan(g, lmax).pid
    n = hb.alm_size(lmax)
    npix = g.npix
    # real coordinates of alm: Re(a_lm) for all, Im(a_lm) for m > 0
    coords = [(k, 0) for k in range(n)] + [(k, 1) for k in range(lmax + 1, n)]
    eye = torch.zeros(len(coords), n, dtype=torch.complex128, device="cuda")
    for j, (k, part) in enumerate(coords):
        eye[j, k] = 1.0 if part == 0 else 1j
    S = torch.ops.hb.alm2map(eye, pid, 0).T  # [npix, ncoord]
    pix = torch.eye(npix, dtype=torch.float64, device="cuda")
    St = torch.ops.hb.alm2map_adjoint(pix, pid, 0)  # [npix, n] complex
    St_real = torch.stack([St[:, k].real if part == 0 else St[:, k].imag for (k, part) in coords], 1)
    assert torch.allclose(St_real, S, rtol=0, atol=1e-13)
    A = torch.ops.hb.map2alm(pix, pid, None, 0)  # [npix, n]: row i = alm of unit pixel i
    A_real = torch.stack([A[:, k].real if part == 0 else A[:, k].imag for (k, part) in coords], 1)  # [npix, nc]
    At = torch.ops.hb.map2alm_adjoint(eye, pid, None, 0)  # [ncoord, npix]
    assert torch.allclose(At.T, A_real, rtol=0, atol=1e-13)
    # and the matrices agree with the oracle
    go = oracle.ring_tables(nside)
    ref = np.stack([oracle.alm2map(npy(eye[j]), go, lmax) for j in range(len(coords))], 1)
    assert np.allclose(npy(S), ref, rtol=0, atol=1e-13)


def test_autograd_finite_differences_fp64(hb):
    """Central differences of a C_l loss through map2alm (nside 8, lmax 16, FP64)."""
    nside, lmax = 8, 16
    gen = torch.Generator().manual_seed(11)
    m = torch.randn(1, 12 * nside * nside, dtype=torch.float64, generator=gen).cuda().requires_grad_(True)
    tgt = torch.rand(1, lmax + 1, dtype=torch.float64, generator=gen).cuda() + 0.5

    def loss(x):
        alm = hb.autograd.map2alm(x, nside, lmax)
        cl = hb.autograd.alm2cl(alm, lmax)
        return (((cl - tgt) / tgt) ** 2).sum()

    L = loss(m)
    L.backward()
    g = m.grad.detach().clone()
    rng = np.random.default_rng(0)
    for i in rng.choice(m.shape[1], 8, replace=False):
        h = 1e-5
        e = torch.zeros_like(m); e[0, i] = h
        with torch.no_grad():
            fd = (loss(m + e) - loss(m - e)) / (2 * h)
        assert abs(float(fd) - float(g[0, i])) <= 1e-6 * max(1.0, abs(float(fd)))


def test_autograd_alm2map_and_spin_gradcheck(hb):
    nside, lmax = 2, 4
    a = _rand_alm(hb, lmax, 7)[None].requires_grad_(True)

    def f(x):
        return hb.autograd.alm2map(x, nside, lmax)

    # gradcheck perturbs Re and Im independently; the m = 0 Im parts have zero derivative
    assert torch.autograd.gradcheck(f, (a,), eps=1e-6, atol=1e-8)
    Q = torch.randn(1, 48, dtype=torch.float64).cuda().requires_grad_(True)
    U = torch.randn(1, 48, dtype=torch.float64).cuda().requires_grad_(True)
    assert torch.autograd.gradcheck(lambda q, u: hb.autograd.map2alm_spin(q, u, nside, lmax), (Q, U), eps=1e-6,
                                    atol=1e-8)
    e = _rand_alm(hb, lmax, 8)[None].requires_grad_(True)
    b = _rand_alm(hb, lmax, 9)[None].requires_grad_(True)
    assert torch.autograd.gradcheck(lambda x, y: hb.autograd.alm2map_spin(x, y, nside, lmax), (e, b), eps=1e-6,
                                    atol=1e-8)
