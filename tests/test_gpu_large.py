"""Large-workload GPU checks of the north-star configurations that do not fit the smaller
parity tests: the differentiable spin-2 power-spectrum loss on 8 Q/U map pairs at nside 4096,
lmax 8191 (forward map2alm_spin + alm2cl, backward through the adjoint kernels with lambda
recomputed), spot-checked against the FP64 oracle on 64 random m; and an uneven batch of 512
maps of four resolutions in one batched plan."""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
TOL = 1e-5


@pytest.fixture(scope="module")
def hb():
    import hellblast_b200
    return hellblast_b200


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_large_spin2_differentiable_nside4096(hb, oracle):
    nside, lmax, nmaps = 4096, 8191, 8
    l = np.arange(lmax + 1, dtype=np.float64)
    cl_e = 1.0 / (l + 10.0) ** 2
    E = torch.stack([hb.synalm(cl_e, lmax=lmax, seed=4 + 2 * i, device="cuda", dtype=torch.complex64)
                     for i in range(nmaps)])
    B = torch.stack([hb.synalm(0.05 * cl_e, lmax=lmax, seed=5 + 2 * i, device="cuda", dtype=torch.complex64)
                     for i in range(nmaps)])
    with torch.no_grad():
        Q, U = hb.autograd.alm2map_spin(E, B, nside, lmax)
        tgt_e = 1.1 * hb.autograd.alm2cl(E, lmax)
        tgt_b = 1.1 * hb.autograd.alm2cl(B, lmax)
    del E, B
    Q.requires_grad_(True)
    U.requires_grad_(True)
    e, b = hb.autograd.map2alm_spin(Q, U, nside, lmax)
    ce, cb = hb.autograd.alm2cl(e, lmax), hb.autograd.alm2cl(b, lmax)
    loss = (((ce - tgt_e) / tgt_e)[:, 2:] ** 2).sum() + (((cb - tgt_b) / tgt_b)[:, 2:] ** 2).sum()
    loss.backward()
    assert torch.isfinite(loss) and torch.isfinite(Q.grad).all() and torch.isfinite(U.grad).all()
    assert float(Q.grad.abs().max()) > 0 and float(U.grad.abs().max()) > 0
    # FP64 oracle on 64 random m of map 0 (the same FP32 maps, analysed in FP64)
    rng = np.random.default_rng(4)
    ms = np.sort(rng.choice(lmax + 1, size=64, replace=False))
    g = oracle.ring_tables(nside)
    q0, u0 = Q[0].detach().double().cpu().numpy(), U[0].detach().double().cpu().numpy()
    Eo, Bo = oracle.map2alm_spin2_ms(q0, u0, g, lmax, ms)
    e0, b0 = e[0].detach().cpu().numpy().astype(np.complex128), b[0].detach().cpu().numpy().astype(np.complex128)
    got_e = np.concatenate([e0[oracle.alm_index(lmax, np.arange(max(m, 2), lmax + 1), m)] for m in ms])
    got_b = np.concatenate([b0[oracle.alm_index(lmax, np.arange(max(m, 2), lmax + 1), m)] for m in ms])
    ref_e = np.concatenate([Eo[j, max(m, 2):] for j, m in enumerate(ms)])
    ref_b = np.concatenate([Bo[j, max(m, 2):] for j, m in enumerate(ms)])
    assert rel(got_e, ref_e) < TOL and rel(got_b, ref_b) < TOL, (rel(got_e, ref_e), rel(got_b, ref_b))


def test_uneven_batch_512_maps_one_plan(hb):
    """512 maps, nside drawn uniformly from {128, 256, 512, 1024} (seed 3), lmax = 2 nside - 1,
    C_l = (l+1)^-2, all in one batched plan (one persistent launch per direction); two or three
    maps of each resolution checked against the FP64 transforms."""
    hb.clear_caches()  # the nside 4096 plans above are no longer needed
    rng = np.random.default_rng(3)
    nsides = rng.choice([128, 256, 512, 1024], size=512)
    counts = {int(ns): int((nsides == ns).sum()) for ns in (128, 256, 512, 1024)}
    specs = [(hb.geometry.healpix(ns), 2 * ns - 1, None, k) for ns, k in counts.items() if k]
    bp = hb.batched.BatchedPlan(specs)
    alms, order = [], []
    for ns, k in counts.items():
        lmax = 2 * ns - 1
        cl = 1.0 / (np.arange(lmax + 1) + 1.0) ** 2
        one = [hb.synalm(cl, lmax=lmax, seed=1000 * ns + i, device="cuda", dtype=torch.complex64)
               for i in range(min(k, 4))]
        alms.append(torch.stack([one[i % len(one)] for i in range(k)]))
        order.append((ns, k))
    flat = torch.cat([a.reshape(-1) for a in alms])
    maps = bp.alm2map(flat)
    back = bp.map2alm(maps)
    torch.cuda.synchronize()
    assert bp.status() == 0
    mofs = aofs = 0
    checked = 0
    for (ns, k), a in zip(order, alms):
        npix, nalm = 12 * ns * ns, a.shape[1]
        for i in range(0, k, max(1, k // 2)):
            a64 = a[i].to(torch.complex128)
            m64 = hb.hp_compat.alm2map(a64, ns, lmax=2 * ns - 1)
            b64 = hb.hp_compat.map2alm(m64, lmax=2 * ns - 1)
            mi = maps[mofs + i * npix: mofs + (i + 1) * npix].double()
            bi = back[aofs + i * nalm: aofs + (i + 1) * nalm].to(torch.complex128)
            assert float(torch.linalg.norm(mi - m64) / torch.linalg.norm(m64)) < TOL
            assert float(torch.linalg.norm(bi - b64) / torch.linalg.norm(b64)) < TOL
            checked += 1
        mofs += k * npix
        aofs += k * nalm
    assert checked >= 8
