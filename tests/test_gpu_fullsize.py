"""Full-size configurations checked against the FP64 oracle, not against this repository's own
FP64 path: the oracle computes the same transforms restricted to a random subset of harmonic
orders m (oracle.map2alm_ms / oracle.alm2map_ms: full ring FFTs, Legendre work for those m
only), which is exact for the entries it returns.

* plain scalar transforms at nside 1024, lmax 2047 (C_l = (l+10)^-2, seed 1), FP64 and FP32;
* the batched split-precision pair at nside 2048, lmax 4095 (both tile widths);
* the differentiable path at nside 2048, lmax 4095: dot-product adjoint identities of the
  scalar and spin-2 transforms at full size, and central finite differences of the T + E/B
  power-spectrum loss at nside 32, lmax 63 in FP64.

Tolerances: FP64 <= 1e-10 relative (max-abs over max-abs of the subset), FP32 and the batched
split <= 1e-5 relative (L2 over the subset).
"""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
TOL32 = 1e-5


@pytest.fixture(scope="module")
def hb():
    import hellblast_b200
    return hellblast_b200


def relmax(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def rel2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _subset(oracle, alm, lmax, ms):
    """healpy-layout alm -> [len(ms), lmax + 1] rows (l < m zero), like oracle.map2alm_ms."""
    out = np.zeros((len(ms), lmax + 1), dtype=np.complex128)
    for j, m in enumerate(ms):
        out[j, m:] = alm[oracle.alm_index(lmax, np.arange(m, lmax + 1), int(m))]
    return out


def _keep_only(oracle, alm, lmax, ms):
    keep = np.zeros(alm.size, bool)
    for m in ms:
        keep[oracle.alm_index(lmax, np.arange(m, lmax + 1), int(m))] = True
    return np.where(keep, alm, 0)


def test_plain_nside1024_vs_oracle_m_subset(hb, oracle):
    nside, lmax = 1024, 2047
    g = oracle.ring_tables(nside)
    cl = 1.0 / (np.arange(lmax + 1) + 10.0) ** 2
    a = hb.synalm(cl, lmax=lmax, seed=1, device="cuda")  # complex128
    a_h = a.cpu().numpy()
    rng = np.random.default_rng(1)
    # alm2map: only a few orders present, so the oracle synthesises the whole map exactly
    ms_map = np.unique(np.concatenate([[0, 1, lmax], rng.choice(lmax + 1, 5, replace=False)]))
    a_sub = _keep_only(oracle, a_h, lmax, ms_map)
    ref_map = oracle.alm2map_ms(a_h, g, lmax, ms_map)
    m64 = hb.hp_compat.alm2map(torch.from_numpy(a_sub).cuda(), nside, lmax=lmax).cpu().numpy()
    m32 = hb.hp_compat.alm2map(torch.from_numpy(a_sub).cuda().to(torch.complex64), nside, lmax=lmax)
    assert relmax(m64, ref_map) < TOL64
    assert rel2(m32.double().cpu().numpy(), ref_map) < TOL32
    # map2alm of the full band-limited map, compared on 32 random orders
    full64 = hb.hp_compat.alm2map(a, nside, lmax=lmax)
    ms = np.sort(rng.choice(lmax + 1, 32, replace=False))
    x64 = full64.cpu().numpy()
    ref64 = oracle.map2alm_ms(x64, g, lmax, ms)
    b64 = hb.hp_compat.map2alm(full64, lmax=lmax).cpu().numpy()
    assert relmax(_subset(oracle, b64, lmax, ms), ref64) < TOL64
    full32 = full64.float()
    ref32 = oracle.map2alm_ms(full32.double().cpu().numpy(), g, lmax, ms)
    b32 = hb.hp_compat.map2alm(full32, lmax=lmax).cpu().numpy().astype(np.complex128)
    assert rel2(_subset(oracle, b32, lmax, ms), ref32) < TOL32


@pytest.mark.parametrize("wide", [False, True])
def test_batched_nside2048_vs_oracle_m_subset(hb, oracle, wide):
    nside, lmax, nmaps = 2048, 4095, 4
    g = oracle.ring_tables(nside)
    cl = 1.0 / (np.arange(lmax + 1) + 10.0) ** 2
    rng = np.random.default_rng(2)
    ms_map = np.unique(np.concatenate([[0, lmax], rng.choice(lmax + 1, 4, replace=False)]))
    a = torch.stack([hb.synalm(cl, lmax=lmax, seed=30 + i, device="cuda", dtype=torch.complex64)
                     for i in range(nmaps)])
    a0 = a[0].cpu().numpy().astype(np.complex128)
    a[0] = torch.from_numpy(_keep_only(oracle, a0, lmax, ms_map)).cuda().to(torch.complex64)
    maps = hb.batched.alm2map(a, nside, lmax, wide=wide)
    back = hb.batched.map2alm(maps, nside, lmax, wide=wide)
    torch.cuda.synchronize()
    assert hb.batched.plan(nside, lmax, nmaps, wide=wide).status() == 0
    # alm2map of map 0 (a few orders) against the oracle's whole map
    ref_map = oracle.alm2map_ms(a0, g, lmax, ms_map)
    assert rel2(maps[0].double().cpu().numpy(), ref_map) < TOL32
    # map2alm of map 1 (all orders present) on 16 random orders, against the oracle's
    # analysis of the same float32 map
    ms = np.sort(rng.choice(lmax + 1, 16, replace=False))
    x1 = maps[1].double().cpu().numpy()
    ref = oracle.map2alm_ms(x1, g, lmax, ms)
    got = _subset(oracle, back[1].cpu().numpy().astype(np.complex128), lmax, ms)
    assert rel2(got, ref) < TOL32


def _rand_alm(hb, lmax, seed, dtype=torch.complex128):
    gen = torch.Generator().manual_seed(seed)
    n = hb.alm_size(lmax)
    a = torch.complex(torch.randn(n, generator=gen, dtype=torch.float64),
                      torch.randn(n, generator=gen, dtype=torch.float64))
    return a.to(dtype).cuda()


def _dot_c(a, b):
    return float((a.real.double() * b.real.double() + a.imag.double() * b.imag.double()).sum())


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_adjoint_dot_products_nside2048(hb, prec):
    """<A x, y> = <x, A^T y> for map2alm and alm2map (scalar) and for the spin-2 map2alm at
    nside 2048, lmax 4095.  FP64: 1e-10; FP32: 1e-4 (each side carries its own FP32 transform
    error, about 5e-6 of the full product)."""
    nside, lmax = 2048, 4095
    rt = torch.float64 if prec == "fp64" else torch.float32
    ct = torch.complex128 if prec == "fp64" else torch.complex64
    tol = 1e-10 if prec == "fp64" else 1e-4
    g = hb.geometry.healpix(nside)
    gen = torch.Generator().manual_seed(0)
    x = torch.randn(1, g.npix, dtype=torch.float64, generator=gen).to(rt).cuda()
    y = _rand_alm(hb, lmax, 1, ct)[None]
    y[:, :lmax + 1] = y[:, :lmax + 1].real.to(ct)  # m = 0 imaginary parts do not enter a real map
    pid = hb.geometry.plan(g, lmax, precision=32 if prec == "fp32" else 64).pid
    lhs, rhs = _dot_c(torch.ops.hb.map2alm(x, pid, None, 0), y), float((x.double() * torch.ops.hb.map2alm_adjoint(
        y, pid, None, 0).double()).sum())
    assert abs(lhs - rhs) <= tol * abs(lhs), (lhs, rhs)
    lhs, rhs = float((torch.ops.hb.alm2map(y, pid, 0).double() * x.double()).sum()), _dot_c(
        torch.ops.hb.alm2map_adjoint(x, pid, 0), y)
    assert abs(lhs - rhs) <= tol * abs(lhs), (lhs, rhs)
    spid = hb.geometry.plan(g, lmax, precision=32 if prec == "fp32" else 64, spin=True).pid
    U = torch.randn(1, g.npix, dtype=torch.float64, generator=gen).to(rt).cuda()
    e, b = y, _rand_alm(hb, lmax, 2, ct)[None]
    E, B = torch.ops.hb.map2alm_spin2(x, U, spid, None, 0)
    lhs = _dot_c(E, e) + _dot_c(B, b)
    del E, B
    gQ, gU = torch.ops.hb.map2alm_spin2_adjoint(e, b, spid, None, 0)
    rhs = float((x.double() * gQ.double()).sum() + (U.double() * gU.double()).sum())
    assert abs(lhs - rhs) <= tol * abs(lhs), (lhs, rhs)


def test_tqu_power_loss_finite_differences_nside32(hb):
    """The config's differentiable loss, sum over TT, EE, BB of sum_l (C_l^est - C_l^tgt)^2 /
    C_l^tgt^2 with C^tgt = 1.1 C^true, backpropagated to T, Q and U through the adjoint kernels
    at nside 32, lmax 63 in FP64, against central differences on random pixels."""
    nside, lmax = 32, 63
    l = np.arange(lmax + 1, dtype=np.float64)
    cl_tt = 1.0 / (l + 10.0) ** 2
    aT = hb.synalm(cl_tt, lmax=lmax, seed=2, device="cuda")
    aE = hb.synalm(0.1 * cl_tt, lmax=lmax, seed=3, device="cuda")
    aB = hb.synalm(0.01 * cl_tt, lmax=lmax, seed=4, device="cuda")
    with torch.no_grad():
        T = hb.autograd.alm2map(aT[None], nside, lmax)
        Q, U = hb.autograd.alm2map_spin(aE[None], aB[None], nside, lmax)
        tgt = [1.1 * hb.autograd.alm2cl(x[None], lmax)[:, 2:] for x in (aT, aE, aB)]

    def loss(t, q, u):
        cl_t = hb.autograd.alm2cl(hb.autograd.map2alm(t, nside, lmax), lmax)[:, 2:]
        e, b = hb.autograd.map2alm_spin(q, u, nside, lmax)
        cl_e = hb.autograd.alm2cl(e, lmax)[:, 2:]
        cl_b = hb.autograd.alm2cl(b, lmax)[:, 2:]
        return sum((((c - t0) / t0) ** 2).sum() for c, t0 in zip((cl_t, cl_e, cl_b), tgt))

    leaves = [x.clone().requires_grad_(True) for x in (T, Q, U)]
    L = loss(*leaves)
    L.backward()
    rng = np.random.default_rng(5)
    for k in range(3):
        grad = leaves[k].grad.detach()
        scale = float(leaves[k].detach().abs().max())
        for i in rng.choice(12 * nside * nside, 6, replace=False):
            h = 1e-4 * scale
            xs = [x.detach().clone() for x in leaves]
            xp = [x.clone() for x in xs]; xp[k][0, i] += h
            xm = [x.clone() for x in xs]; xm[k][0, i] -= h
            with torch.no_grad():
                fd = float((loss(*xp) - loss(*xm)) / (2 * h))
            assert abs(fd - float(grad[0, i])) <= 1e-6 * max(abs(fd), 1e-3 * float(grad.abs().max())), (k, i)
