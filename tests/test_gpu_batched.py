"""GPU tests of the batched split-precision tensor-core path (tcgen05, BF16 hi+lo three-pass,
FP32 accumulation): against the FP64 path (itself pinned to the oracle) at <= 1e-5 relative,
against the plain FP32 path, several batch widths, several geometries in one launch."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-5


def rel(a, b):
    a = a.to(torch.complex128) if a.is_complex() else a.double()
    b = b.to(torch.complex128) if b.is_complex() else b.double()
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


@pytest.fixture(scope="module")
def hb():
    import hellblast_b200
    return hellblast_b200


def _batch(hb, lmax, nmaps, seed=0):
    cl = 1.0 / (np.arange(lmax + 1) + 10.0) ** 2
    return torch.stack([hb.synalm(cl, lmax=lmax, seed=seed + i, device="cuda") for i in range(nmaps)])


@pytest.mark.parametrize("bf16", [False, True])
@pytest.mark.parametrize("nside,nmaps", [(8, 1), (16, 3), (64, 20), (128, 64)])
def test_batched_alm2map_and_map2alm_vs_fp64(hb, nside, nmaps, bf16):
    lmax = 2 * nside - 1
    a64 = _batch(hb, lmax, nmaps)
    m64 = hb.hp_compat.alm2map(a64, nside, lmax=lmax)
    mb = hb.batched.alm2map(a64.to(torch.complex64), nside, lmax, bf16=bf16)
    bp = hb.batched.plan(nside, lmax, nmaps, bf16=bf16)
    assert bp.status() == 0
    assert mb.shape == m64.shape and mb.dtype == torch.float32
    assert rel(mb, m64) < TOL
    b64 = hb.hp_compat.map2alm(m64, lmax=lmax)
    bb = hb.batched.map2alm(m64.float(), nside, lmax, bf16=bf16)
    assert bp.status() == 0
    assert rel(bb, b64) < TOL
    # and against the plain FP32 path on the same inputs
    m32 = hb.hp_compat.alm2map(a64.to(torch.complex64), nside, lmax=lmax)
    assert rel(mb, m32) < 2 * TOL


def test_batched_high_lmax_small_nside(hb):
    """lmax well above 2 nside: aliasing fold and underflowing polar lambda_mm in the batch."""
    nside, lmax, nmaps = 16, 100, 5
    a64 = _batch(hb, lmax, nmaps, seed=3)
    m64 = hb.hp_compat.alm2map(a64, nside, lmax=lmax)
    mb = hb.batched.alm2map(a64.to(torch.complex64), nside, lmax)
    assert rel(mb, m64) < TOL
    b64 = hb.hp_compat.map2alm(m64, lmax=lmax)
    bb = hb.batched.map2alm(m64.float(), nside, lmax)
    assert rel(bb, b64) < TOL


def test_batched_several_geometries_one_launch(hb):
    """Uneven batch: maps of different nside/lmax in one persistent launch per direction."""
    specs = [(16, 31, 3), (32, 63, 70), (8, 15, 2)]
    geoms = [(hb.geometry.healpix(ns), lm, None, k) for ns, lm, k in specs]
    bp = hb.batched.BatchedPlan(geoms)
    alms = [_batch(hb, lm, k, seed=10 * i) for i, (ns, lm, k) in enumerate(specs)]
    flat = torch.cat([a.to(torch.complex64).reshape(-1) for a in alms])
    maps = bp.alm2map(flat)
    assert bp.status() == 0
    ofs = 0
    refs = []
    for (ns, lm, k), a in zip(specs, alms):
        ref = hb.hp_compat.alm2map(a, ns, lmax=lm)
        n = ref.numel()
        assert rel(maps[ofs:ofs + n].reshape(ref.shape), ref) < TOL
        refs.append(ref)
        ofs += n
    back = bp.map2alm(torch.cat([r.float().reshape(-1) for r in refs]))
    assert bp.status() == 0
    ofs = 0
    for (ns, lm, k), r in zip(specs, refs):
        ref = hb.hp_compat.map2alm(r, lmax=lm)
        n = ref.numel()
        assert rel(back[ofs:ofs + n].reshape(ref.shape), ref) < TOL
        ofs += n


def test_batched_vs_oracle_small(hb, oracle):
    nside, lmax = 8, 20
    g = oracle.ring_tables(nside)
    cl = 1.0 / (np.arange(lmax + 1) + 1.0) ** 2
    alms = np.stack([oracle.synalm(cl, seed=s) for s in range(4)])
    ref = np.stack([oracle.alm2map(a, g, lmax) for a in alms])
    out = hb.batched.alm2map(torch.from_numpy(alms).cuda().to(torch.complex64), nside, lmax).double().cpu().numpy()
    assert np.linalg.norm(out - ref) / np.linalg.norm(ref) < TOL
    back = hb.batched.map2alm(torch.from_numpy(ref).cuda().float(), nside, lmax).cpu().numpy()
    refa = np.stack([oracle.map2alm(r, g, lmax) for r in ref])
    assert np.linalg.norm(back - refa) / np.linalg.norm(refa) < TOL


@pytest.mark.parametrize("nside,wide", [(1024, False), (2048, False), (2048, True)])
def test_batched_pair_accuracy_at_full_size(hb, nside, wide):
    """The north-star bar: the batched pair (IEEE-half hi+lo; 32- or 64-map groups) within 1e-5
    of FP64 at lmax = 2 nside - 1, 8 maps (first and last checked)."""
    lmax, nmaps = 2 * nside - 1, 8
    a64 = _batch(hb, lmax, nmaps, seed=7)
    mb = hb.batched.alm2map(a64.to(torch.complex64), nside, lmax, wide=wide)
    bb = hb.batched.map2alm(mb, nside, lmax, wide=wide)
    errs = []
    for i in (0, nmaps - 1):
        m64 = hb.hp_compat.alm2map(a64[i], nside, lmax=lmax)
        b64 = hb.hp_compat.map2alm(m64, lmax=lmax)
        errs.append((rel(mb[i], m64), rel(bb[i], b64)))
        del m64, b64
    assert hb.batched.plan(nside, lmax, nmaps, wide=wide).status() == 0
    assert all(e[0] < TOL and e[1] < TOL for e in errs), errs


def test_batched_graph_replay_matches_direct_calls(hb):
    """A batched step captured as one CUDA graph (several geometries, both directions) reproduces
    the direct calls bit for bit, twice in a row."""
    specs = [(16, 31, 5), (32, 63, 40)]
    bp = hb.batched.BatchedPlan([(hb.geometry.healpix(ns), lm, None, k) for ns, lm, k in specs])
    alm = torch.cat([_batch(hb, lm, k, seed=20 + i).to(torch.complex64).reshape(-1)
                     for i, (ns, lm, k) in enumerate(specs)])
    ref_maps = bp.alm2map(alm)
    ref_alm = bp.map2alm(ref_maps)
    maps = torch.empty_like(ref_maps)
    out = torch.empty_like(ref_alm)
    bp.capture(alm, maps, out)
    for _ in range(2):
        maps.zero_()
        out.zero_()
        bp.replay()
        torch.cuda.synchronize()
        assert bp.status() == 0
        assert torch.equal(maps, ref_maps)
        assert torch.equal(out, ref_alm)


def test_autotune_picks_a_measured_configuration_within_tolerance(hb):
    nside, lmax, nmaps = 32, 63, 40
    t = hb.batched.autotune(nside, lmax, nmaps)
    assert len(t["candidates"]) == 4 and all(c["ms"] > 0 for c in t["candidates"])
    chosen = [c for c in t["candidates"] if (c["bf16"], c["wide"]) == (t["bf16"], t["wide"])][0]
    assert chosen["ok"] and chosen["rel_err"] <= TOL
    assert chosen["ms"] == min(c["ms"] for c in t["candidates"] if c["ok"])
    a = _batch(hb, lmax, nmaps, seed=5).to(torch.complex64)
    bp = hb.batched.plan(nside, lmax, nmaps, tuned=True)
    assert (bp.bf16, bp.wide) == (t["bf16"], t["wide"])
    m = bp.alm2map(a).reshape(nmaps, -1)
    assert rel(m, hb.hp_compat.alm2map(a.to(torch.complex128), nside, lmax=lmax)) < TOL


def test_bounded_wait_expires_and_context_stays_usable(hb):
    """Failure detection without a GPU fault: with a 20 ms wait bound, the synthesis loader of
    CTA 0 withholds its first batch-tile copy (hb_batched_fault_test); the waits on that stage
    run out, the kernel records an error code and returns.  The host reads the code, clears it,
    and the same plan then runs clean and correct."""
    import time
    nside, lmax, nmaps = 32, 63, 40
    a = _batch(hb, lmax, nmaps, seed=9).to(torch.complex64)
    bp = hb.batched.BatchedPlan([(hb.geometry.healpix(nside), lmax, None, nmaps)])
    bp.fault_test(wait_s=0.02, withhold_copy=True)
    t0 = time.perf_counter()
    bp.alm2map(a.reshape(-1))
    torch.cuda.synchronize()
    assert time.perf_counter() - t0 < 5.0  # bounded: a few wait limits, not a hang
    code = bp.status()
    assert code != 0
    bp.reset_status()
    bp.fault_test(wait_s=2.0, withhold_copy=False)
    m = bp.alm2map(a.reshape(-1)).reshape(nmaps, -1)
    torch.cuda.synchronize()
    assert bp.status() == 0
    assert rel(m, hb.hp_compat.alm2map(a.to(torch.complex128), nside, lmax=lmax)) < TOL
