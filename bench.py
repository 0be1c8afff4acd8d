"""Benchmark: map2alm+alm2map pairs/s at nside 2048, lmax 4095 on B200.

One step = one alm2map + map2alm pair for each map of the batch (synthetic Gaussian alm,
C_l = (l+10)^-2, float32 maps of 50,331,648 pixels: every input is larger than the 126 MB L2).
N GPUs: independent maps per rank (weak scaling, no data-path collective), timed on the device
with CUDA events, max over ranks.  Prints one JSON line on rank 0.

  python bench.py [--gpus N --steps K --warmup W --mode plain|batched --nmaps B]
  python bench.py --impl reference   # the CPU restatement of the reference path (oracle port)
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "map2alm+alm2map/s, nside 2048 lmax 4095: batched vs plain, rel err ≤1e-5 vs FP64"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--mode", default="batched", choices=["plain", "batched", "msharded"],
                   help="batched: tensor-core batch per GPU (replicas); plain: FP32 per-map path; msharded: "
                        "each map's transform split over the GPUs by ring pairs and orders m (one all-to-all "
                        "per direction, strong scaling)")
    p.add_argument("--nside", type=int, default=2048)
    p.add_argument("--lmax", type=int, default=None)
    p.add_argument("--nmaps", type=int, default=None, help="maps per GPU (default 64 batched, 1 plain)")
    p.add_argument("--split", default=None, choices=["f16", "bf16"],
                   help="16-bit type of the hi+lo split (default: chosen by the autotuner)")
    p.add_argument("--wide", default=None, action="store_true",
                   help="groups of 64 maps, MMA N = 128 (default: chosen by the autotuner)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-extras", action="store_true",
                   help="skip the plain-path and differentiable-path legs of the batched line")
    p.add_argument("--plain-maps", type=int, default=4, help="maps timed one per call on the plain FP32 path")
    p.add_argument("--cpu-sample-m", type=int, default=12)
    return p.parse_args()


def n_lm(lmax, mmax=None):
    mmax = lmax if mmax is None else mmax
    return mmax * (2 * lmax + 1 - mmax) // 2 + lmax + 1


class Clocks:
    """Samples nvidia-smi SM clocks and throttle reasons while the timed region runs."""
    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                self.samples.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        sm = [float(s[0]) for s in self.samples if len(s) >= 7 and s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if len(s) >= 7 and s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples if len(s) >= 7 for i in range(4) if s[3 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ----------------------------------------------------------------------------- CPU side
def cpu_baseline(nside, lmax, sample_m):
    """The FP64 oracle (C restatement of the reference path, OpenMP on all host cores) on a
    bounded sample: ring FFTs of the whole map, Legendre work for m = 0..sample_m-1, scaled
    to all m by the Legendre work ratio.  Returns pairs/s and a description."""
    from oracle import sht_oracle as O
    g = O.ring_tables(nside)
    cl = 1.0 / (np.arange(lmax + 1) + 10.0) ** 2
    ms = sample_m - 1
    rng = np.random.default_rng(1)
    alm = (rng.standard_normal(n_lm(lmax, ms)) + 1j * rng.standard_normal(n_lm(lmax, ms))) * math.sqrt(cl[0])
    t0 = time.perf_counter()
    G = O.legendre_synthesis(alm, g, lmax, ms)
    t1 = time.perf_counter()
    mp = O.ring_synthesis(G, g)
    t2 = time.perf_counter()
    F = O.ring_analysis(mp, g, ms, weights=g["weights_dz"])
    t3 = time.perf_counter()
    O.legendre_analysis(F, g, lmax)
    t4 = time.perf_counter()
    leg_sample = (t1 - t0) + (t4 - t3)
    fft = (t2 - t1) + (t3 - t2)
    ratio = n_lm(lmax) / n_lm(lmax, ms)
    per_pair = leg_sample * ratio + fft
    cores = os.cpu_count()
    return 1.0 / per_pair, {
        "cores": cores, "kind": "port",
        "sample": (f"FP64 oracle (oracle/sht_oracle.c, OpenMP {cores} threads + numpy FFT) at nside {nside}, "
                   f"lmax {lmax}: ring FFTs of the full map ({fft:.1f} s) + Legendre for m<{sample_m} "
                   f"({leg_sample:.1f} s) scaled x{ratio:.0f} to all m"),
        "seconds": t4 - t0}


def reference_pair_steps(nside, lmax, nsteps, seed=1):
    """One full FP64 alm2map + map2alm pair of the oracle (the CPU restatement of the reference's
    path: numpy ring FFTs, C + OpenMP Legendre work) cut into ``nsteps`` consecutive steps in
    dependency order, so that the steps together do exactly one pair:
      A: Legendre synthesis G(m, ring) for a set of orders m (sets balanced by l-range length);
      B: ring synthesis and ring analysis of a block of rings (blocks balanced by pixel count;
         the block's FFTs run on a thread pool);
      D: Legendre analysis a_lm for a set of orders.
    Returns (list of callables, the warm-up callables, a function returning the pair's result)."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import sht_oracle as O
    g = O.ring_tables(nside)
    nr, npix, mmax = g["nr"], int(g["npix"]), lmax
    cl = 1.0 / (np.arange(lmax + 1) + 10.0) ** 2
    alm = O.synalm(cl, lmax=lmax, seed=seed)
    units = max(nsteps, 3)
    na = max(1, int(round(0.4 * units)))
    nb = max(1, units - 2 * na)
    # orders: greedy balance of the l-range lengths over na sets
    msets = [[] for _ in range(na)]
    load = np.zeros(na)
    for m in range(mmax + 1):  # descending cost
        j = int(np.argmin(load))
        msets[j].append(m)
        load[j] += lmax - m + 1
    msets = [np.array(sorted(x), dtype=np.int64) for x in msets]
    rs = g["ring_start"]
    cuts = [int(np.searchsorted(rs, npix * k / nb)) for k in range(nb)] + [nr]
    rblocks = [(cuts[k], cuts[k + 1]) for k in range(nb) if cuts[k + 1] > cuts[k]]
    G = np.zeros((mmax + 1, nr), dtype=np.complex128)
    F = np.zeros((mmax + 1, nr), dtype=np.complex128)
    mp = np.zeros(npix)
    out = np.zeros((mmax + 1, lmax + 1), dtype=np.complex128)
    w = g["weights_dz"]
    threads = os.cpu_count() or 1

    def A(ms):
        return lambda: G.__setitem__(ms, O.legendre_synthesis_ms(O.alm_rows(alm, lmax, ms), g, lmax, ms))

    def ring_block(r0, r1):
        sg = O.ring_subset(g, r0, r1)
        mp[rs[r0]:rs[r1]] = O.ring_synthesis(G[:, r0:r1], sg)
        F[:, r0:r1] = O.ring_analysis(mp[rs[r0]:rs[r1]], sg, mmax, weights=w[r0:r1])

    def B(r0, r1):
        step = max(1, (r1 - r0 + 4 * threads - 1) // (4 * threads))
        subs = [(a, min(a + step, r1)) for a in range(r0, r1, step)]

        def run():
            with ThreadPoolExecutor(threads) as ex:
                list(ex.map(lambda ab: ring_block(*ab), subs))
        return run

    def D(ms):
        return lambda: out.__setitem__(ms, O.legendre_analysis_ms(F[ms], g, lmax, ms))

    work = [A(ms) for ms in msets] + [B(*rb) for rb in rblocks] + [D(ms) for ms in msets]
    steps = [[] for _ in range(nsteps)]
    for i, f in enumerate(work):  # consecutive units per step, in order
        steps[i * nsteps // len(work)].append(f)
    steps = [(lambda fs: (lambda: [f() for f in fs]))(fs) for fs in steps]

    def result():
        got = np.concatenate([out[m, m:] for m in range(mmax + 1)])
        return float(np.linalg.norm(got - alm) / np.linalg.norm(alm))
    return steps, [A(ms) for ms in msets], result


def run_reference(args):
    """The reference arm: the FP64 oracle (the CPU restatement of the reference's SHT path; the
    reference's own path is CuPy-only and overflows above lmax 85) on the host cores.  The
    --steps K steps together perform exactly one full alm2map + map2alm pair at the bench's
    nside and lmax (reference_pair_steps); --warmup W runs W of the Legendre synthesis units
    untimed first.  value = one pair / the K steps' total time."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    lmax = 2 * args.nside - 1 if args.lmax is None else args.lmax
    K = max(1, args.steps)
    steps, warm, result = reference_pair_steps(args.nside, lmax, K)
    for i in range(args.warmup):
        warm[i % len(warm)]()
    times = []
    for f in steps:
        t0 = time.perf_counter()
        f()
        times.append(time.perf_counter() - t0)
    total = sum(times)
    v = 1.0 / total
    cores = os.cpu_count()
    sample = (f"one full FP64 pair (oracle: C + OpenMP Legendre on {cores} threads, numpy ring FFTs on a "
              f"{cores}-thread pool) at nside {args.nside}, lmax {lmax}, cut into {K} steps in dependency "
              f"order (Legendre synthesis by order sets, ring FFTs by ring blocks, Legendre analysis by "
              f"order sets); {total:.1f} s in total")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "pairs/s", "n_gpus": args.gpus,
        "steps": K, "warmup": args.warmup, "ms_per_step": 1000.0 * total / K, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (Gaussian alm, C_l=(l+10)^-2)",
        "config": {"workload": f"scalar map2alm+alm2map pair, nside {args.nside}, lmax {lmax}, float64, CPU, "
                               "one map per pair", "nside": args.nside, "lmax": lmax},
        "cpu_baseline": {"value": v, "unit": "pairs/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "round_trip_rel_err": result(),
        "step_seconds": [round(t, 3) for t in times],
    }), flush=True)


# ----------------------------------------------------------------------------- GPU side
def hbm_bytes_ring_fft(nmaps, mmax, npairs, npix, itemsize=4):
    """Algorithmic HBM bytes of one ring-FFT pass over `nmaps` maps (either direction): the
    Fourier coefficients (mmax + 1) x npairs x (north, south) complex read or written once, and
    every map pixel written or read once."""
    return nmaps * ((mmax + 1) * npairs * 2 * 2 * itemsize + npix * itemsize)


def load_traffic():
    """DRAM bytes per launch measured by ncu (profiles/traffic_*.txt: `stage bytes` lines)."""
    out = {}
    d = os.path.join(ROOT, "profiles")
    for name in sorted(os.listdir(d)) if os.path.isdir(d) else []:
        if not (name.startswith("traffic_") and name.endswith(".txt")):
            continue
        with open(os.path.join(d, name)) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 2 and not line.startswith("#"):
                    try:
                        out[parts[0]] = float(parts[1])
                    except ValueError:
                        pass
    return out


def plain_leg(hb, L, G, nside, lmax, nmaps, alm_h, dev, st, reps=3):
    """The plain FP32 per-map form (the comparison the metric names): alm2map + map2alm of one
    map per call through the FP32 Legendre and ring-FFT kernels, `nmaps` maps, `reps` times."""
    import torch
    g = G.healpix(nside)
    plan = G.plan(g, lmax, precision=32)
    ws = torch.empty(plan.workspace_bytes(32, 1), dtype=torch.uint8, device=dev)
    alm = alm_h[:nmaps].to(dev)
    maps = torch.empty(nmaps, 12 * nside * nside, dtype=torch.float32, device=dev)
    out = torch.empty_like(alm)
    sp = st.cuda_stream

    def run():
        for i in range(nmaps):
            L.call("hb_alm2map_f32", plan.handle, 1, alm[i].data_ptr(), maps[i].data_ptr(), ws.data_ptr(),
                   ws.numel(), 0, sp)
            L.call("hb_map2alm_f32", plan.handle, 1, maps[i].data_ptr(), None, out[i].data_ptr(), ws.data_ptr(),
                   ws.numel(), 0, sp)
    run()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        run()
    e1.record(st)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / (reps * nmaps)
    del ws, maps, out
    return 1000.0 / ms, ms


def diff_leg(hb, nside, lmax, dev, st, reps=3):
    """The differentiable path: the T + E/B power-spectrum loss sum_XX sum_l (C_l - 1.1 C_l^true)^2 /
    (1.1 C_l^true)^2 of one float32 T, Q, U map set (TT (l+10)^-2, EE 0.1 TT, BB 0.01 TT), forward
    alone and forward + backward through the adjoint kernels.  Returns (forward ms, ratio)."""
    import torch
    from hellblast_b200 import autograd
    l = np.arange(lmax + 1, dtype=np.float64)
    cl = 1.0 / (l + 10.0) ** 2
    aT, aE, aB = (hb.synalm(c, lmax=lmax, seed=s, device=dev, dtype=torch.complex64)[None]
                  for c, s in ((cl, 2), (0.1 * cl, 3), (0.01 * cl, 4)))
    with torch.no_grad():
        T = autograd.alm2map(aT, nside, lmax)
        Q, U = autograd.alm2map_spin(aE, aB, nside, lmax)
        tgt = [1.1 * autograd.alm2cl(x, lmax) for x in (aT, aE, aB)]

    def loss_of(t, q, u):
        e, b = autograd.map2alm_spin(q, u, nside, lmax)
        cls = [autograd.alm2cl(autograd.map2alm(t, nside, lmax), lmax), autograd.alm2cl(e, lmax),
               autograd.alm2cl(b, lmax)]
        return sum((((c - ct) / ct)[:, 2:] ** 2).sum() for c, ct in zip(cls, tgt))

    def fwd():
        with torch.no_grad():
            loss_of(T, Q, U)

    def fwd_bwd():
        t, q, u = (x.clone().requires_grad_(True) for x in (T, Q, U))
        loss_of(t, q, u).backward()

    res = []
    for fn in (fwd, fwd_bwd):
        fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            fn()
        e1.record(st)
        torch.cuda.synchronize(dev)
        res.append(e0.elapsed_time(e1) / reps)
    return res[0], res[1] / res[0]


def run_msharded(args):
    """--mode msharded: one FP32 alm2map + map2alm of B maps per step, every map split over the
    ranks (distributed.MShardedSHT: ring-pair blocks for the FFTs, zig-zag order sets for the
    Legendre work, one NCCL all-to-all per direction).  value = B pairs / step time (max over
    ranks); e2e copies the alm in from pinned host memory and this rank's result out each step."""
    import datetime
    import torch
    import torch.distributed as dist
    import hellblast_b200 as hb
    from hellblast_b200 import distributed as D

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    nside = args.nside
    lmax = 2 * nside - 1 if args.lmax is None else args.lmax
    B = args.nmaps if args.nmaps is not None else 4
    st = torch.cuda.current_stream(dev)
    cl = 1.0 / (np.arange(lmax + 1) + 10.0) ** 2
    alm_h = torch.stack([hb.synalm(cl, lmax=lmax, seed=i, device="cpu", dtype=torch.complex64) for i in range(B)])
    alm = alm_h.to(dev)
    ms = D.MShardedSHT(nside, lmax, precision=32)
    n_fft = ms.lg.fft_launches(32) if ms.lg is not None else 0

    def step(a):
        return ms.map2alm(ms.alm2map(a))

    for _ in range(args.warmup):
        out = step(alm)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    with Clocks(local) as clk:
        t0 = torch.cuda.Event(enable_timing=True); t1 = torch.cuda.Event(enable_timing=True)
        t0.record(st)
        for _ in range(args.steps):
            out = step(alm)
        t1.record(st)
        torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    ms_t = t0.elapsed_time(t1)
    # accuracy: this rank's orders of map 0 against the single-GPU FP64 pair
    a64 = alm_h[0].to(dev, torch.complex128)
    b64 = hb.hp_compat.map2alm(hb.hp_compat.alm2map(a64, nside, lmax=lmax), lmax=lmax)
    from hellblast_b200 import alm_ops
    mine = torch.isin(alm_ops._m_of_index(lmax, lmax, str(dev)), torch.as_tensor(ms.layout.msets[rank], device=dev))
    err = float(torch.linalg.norm((out[0].to(torch.complex128) - b64)[mine]) / torch.linalg.norm(b64[mine]))
    pin_in = alm_h.pin_memory()
    pin_out = torch.empty_like(pin_in).pin_memory()
    e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    e0.record(st)
    for _ in range(args.steps):
        r = step(pin_in.to(dev, non_blocking=True))
        pin_out.copy_(r, non_blocking=True)
    e1.record(st)
    torch.cuda.synchronize(dev)
    ms_e = e0.elapsed_time(e1)
    if world > 1:
        tt = torch.tensor([ms_t, ms_e], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms_t, ms_e = (float(x) for x in tt.tolist())
        dist.destroy_process_group()
    if rank != 0:
        return
    print(json.dumps({
        "metric": METRIC, "value": args.steps * B / (ms_t * 1e-3), "unit": "pairs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_t / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic (Gaussian alm, C_l=(l+10)^-2)",
        "config": {"workload": f"scalar map2alm+alm2map pair, nside {nside}, lmax {lmax}, float32, {B} maps per "
                               f"step, each split over {world} GPUs by ring pairs and orders m", "nside": nside,
                   "lmax": lmax, "maps_per_step": B, "mode": "msharded", "parallelism": f"m-sharded x{world}",
                   "l2": "inputs larger than L2 (one map 201 MB at nside 2048)"},
        "rel_err_vs_fp64_rank0_orders": err,
        "e2e": {"value": args.steps * B / (ms_e * 1e-3), "unit": "pairs/s", "h2d_bytes_per_step": int(pin_in.numel() * 8),
                "d2h_bytes_per_step": int(pin_out.numel() * 8), "api": "distributed.MShardedSHT from pinned host alm"},
        "gpu_launches": args.steps * (2 + 2 * n_fft),
        "clocks": clk.summary(),
    }), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.mode == "msharded":
        return run_msharded(args)
    import torch
    import torch.distributed as dist
    import hellblast_b200 as hb
    from hellblast_b200 import _lib as L
    from hellblast_b200 import geometry as G

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    nside = args.nside
    lmax = 2 * nside - 1 if args.lmax is None else args.lmax
    mmax = lmax
    nalm = n_lm(lmax)
    npix = 12 * nside * nside
    P = 2 * nside
    B = args.nmaps if args.nmaps is not None else (64 if args.mode == "batched" else 1)
    g = G.healpix(nside)
    st = torch.cuda.current_stream(dev)
    sp = st.cuda_stream

    # synthetic Gaussian alm, C_l = (l+10)^-2, seeded per rank and map (independent maps)
    cl = 1.0 / (np.arange(lmax + 1) + 10.0) ** 2
    alm_h = torch.stack([hb.synalm(cl, lmax=lmax, seed=1000 * rank + i, device="cpu", dtype=torch.complex64)
                         for i in range(min(B, 4))])
    alm_h = alm_h.repeat((B + alm_h.shape[0] - 1) // alm_h.shape[0], 1)[:B].contiguous()
    alm = alm_h.to(dev)
    maps = torch.empty(B, npix, dtype=torch.float32, device=dev)
    alm_out = torch.empty_like(alm)

    # FP32-pipe peak measured on this GPU (FFMA probe)
    probe_out = torch.empty(148 * 8 * 256, dtype=torch.float32, device=dev)
    iters = 20000
    L.call("hb_probe_fp32", 148 * 8, 256, 2000, probe_out.data_ptr(), sp)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    L.call("hb_probe_fp32", 148 * 8, 256, iters, probe_out.data_ptr(), sp)
    e1.record(st)
    torch.cuda.synchronize(dev)
    fp32_peak = 148 * 8 * 256 * iters * 8 * 2 / (e0.elapsed_time(e1) * 1e-3) / 1e12
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    bf16_peak = float(peaks.get("bf16_tflops", 1590.0))
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))

    if args.mode == "plain":
        plan = G.plan(g, lmax, mmax, precision=32)
        n_launch = 2 + 2 * g.fft_launches(32)
        ws = torch.empty(plan.workspace_bytes(32, B), dtype=torch.uint8, device=dev)

        def step(ev=None):
            if ev: ev[0].record(st)
            L.call("hb_legendre_synthesis", plan.handle, 32, B, alm.data_ptr(), ws.data_ptr(), sp)
            if ev: ev[1].record(st)
            L.call("hb_ring_synthesis", plan.handle, 32, B, ws.data_ptr(), maps.data_ptr(), 0, sp)
            if ev: ev[2].record(st)
            L.call("hb_ring_analysis", plan.handle, 32, B, maps.data_ptr(), None, ws.data_ptr(), 0, sp)
            if ev: ev[3].record(st)
            L.call("hb_legendre_analysis", plan.handle, 32, B, ws.data_ptr(), alm_out.data_ptr(), sp)
            if ev: ev[4].record(st)

        def stage_times(evs):
            s = np.array([[ev[i].elapsed_time(ev[i + 1]) for i in range(4)] for ev in evs]).mean(0)
            return {"legendre_synthesis": s[0], "ring_synthesis": s[1], "ring_analysis": s[2],
                    "legendre_analysis": s[3]}
        def make_ev():
            return [torch.cuda.Event(enable_timing=True) for _ in range(5)]
    else:
        tune = None
        if args.split is None and args.wide is None:  # measured choice: fastest within 1e-5 of FP64
            tune = hb.batched.autotune(nside, lmax, B)
            bf16, wide = tune["bf16"], tune["wide"]
        else:
            bf16, wide = args.split == "bf16", bool(args.wide)
        bp = hb.batched.plan(nside, lmax, B, bf16=bf16, wide=wide)
        alm_flat, maps_flat, out_flat = alm.reshape(-1), maps.reshape(-1), alm_out.reshape(-1)
        # the whole step (both directions, every kernel) as one CUDA graph
        bp.capture(alm_flat, maps_flat, out_flat)
        stage_acc = []

        def step(ev=None):
            if ev is None:
                bp.replay(st)
                return
            bp.profile(True)  # separately timed step with events between the kernels
            bp.alm2map(alm_flat, out=maps_flat)
            bp.map2alm(maps_flat, out=out_flat)
            stage_acc.append(bp.stage_ms())
            bp.profile(False)

        def stage_times(evs):
            keys = stage_acc[0].keys()
            return {k: float(np.mean([s[k] for s in stage_acc])) for k in keys}
        groups = (B + (63 if wide else 31)) // (64 if wide else 32)
        n_launch = 2 * groups + 2 + 2 * g.fft_launches(32)  # operand preps, tensor kernels, ring FFT classes

        def make_ev():
            return True

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    if args.mode == "plain":
        evs = [make_ev() for _ in range(args.steps)]
    with Clocks(local) as clk:
        torch.cuda.synchronize(dev)
        t0 = torch.cuda.Event(enable_timing=True); t1 = torch.cuda.Event(enable_timing=True)
        t0.record(st)
        for k in range(args.steps):
            step(evs[k] if args.mode == "plain" else None)
        t1.record(st)
        torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    ms = t0.elapsed_time(t1)
    if args.mode == "batched":  # stage breakdown from one extra, separately timed step
        step(True)
        torch.cuda.synchronize(dev)
        stages = stage_times(None)
        assert bp.status() == 0, f"tensor-core pipeline reported error {bp.status()}"
    else:
        stages = stage_times(evs)
    if world > 1:
        tt = torch.tensor([ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    value = world * args.steps * B / (ms * 1e-3)

    # accuracy of map 0 of the pair vs the FP64 pair on the same input
    a64 = alm_h[0].to(dev, torch.complex128)
    m64 = hb.hp_compat.alm2map(a64, nside, lmax=lmax)
    b64 = hb.hp_compat.map2alm(m64, lmax=lmax)
    relerr = float(torch.linalg.norm(alm_out[0].to(torch.complex128) - b64) / torch.linalg.norm(b64))
    del m64, b64

    # end to end through the public API: pinned host alm in, host alm out, copies timed
    alm_pin = alm_h.pin_memory()
    out_pin = torch.empty_like(alm_pin).pin_memory()

    if args.mode == "plain":
        def e2e_run(k):
            for _ in range(k):
                a = alm_pin.to(dev, non_blocking=True)
                m = hb.hp_compat.alm2map(a, nside, lmax=lmax)
                r = hb.hp_compat.map2alm(m, lmax=lmax)
                out_pin.copy_(r, non_blocking=True)
    else:
        # batches streamed from pinned host memory: copies in / out overlap the transforms
        pipe = hb.batched.HostPipeline(bp, dev)

        def e2e_run(k):
            pipe.run([alm_pin] * k, [out_pin] * k)
            pipe.wait_on(st)

    # the streamed batches overlap copies with transforms; the first copy in and the last copy
    # out (about one step's time together) are not hidden, so this leg streams at least 16
    # batches, as a pipeline of batches would in production
    e2e_steps = args.steps if args.mode == "plain" else max(args.steps, 16)
    e2e_run(max(1, args.warmup))
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    t2 = torch.cuda.Event(enable_timing=True); t3 = torch.cuda.Event(enable_timing=True)
    t2.record(st)
    if args.mode != "plain":
        for s_ in (pipe.s_in, pipe.s_run, pipe.s_out):
            s_.wait_stream(st)
    e2e_run(e2e_steps)
    t3.record(st)
    torch.cuda.synchronize(dev)
    ms_e2e = t2.elapsed_time(t3)
    if world > 1:
        tt = torch.tensor([ms_e2e], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms_e2e = float(tt.item())
    e2e = world * e2e_steps * B / (ms_e2e * 1e-3)

    logical = 8.0 * nalm * P  # per map per direction: 4 recursion + 4 contraction flop per (l, m, pair)
    if args.mode == "plain":
        t_dom = (stages["legendre_synthesis"] + stages["legendre_analysis"]) * 1e-3
        achieved = 2 * logical * B / t_dom / 1e12
        roof = {"bound": "fp32", "kernel": "leg_synthesis_kernel + leg_analysis_kernel", "achieved": achieved,
                "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak, "traffic": None,
                "peak_source": "FFMA probe (hb_probe_fp32) on this GPU in this run",
                "flop_per_launch": logical * B}
    else:
        t_dom = (stages["tensor_synthesis"] + stages["tensor_analysis"]) * 1e-3
        alg = (4.0 * B + 4.0) * nalm * P          # logical: contraction per map + shared recursion
        ex = bp.executed_mma_flop()               # MMAs actually issued (3 split passes, Re/Im columns,
        executed = 0.5 * (ex["synthesis"] + ex["analysis"])  # padding of the last group, evanescent skip)
        achieved = 2 * alg / t_dom / 1e12
        tensor = {"bound": "tensor", "kernel": "synth_tc_kernel + anal_tc_kernel", "achieved": achieved,
                  "peak": bf16_peak, "unit": "TFLOP/s", "frac": achieved / bf16_peak,
                  "traffic": None,
                  "peak_source": ("MEASURED_PEAKS.json bf16_tflops (burst), of measured" if peaks
                                  else "fallback 1590 TFLOP/s, of fallback"),
                  "flop_per_launch": alg,
                  "tensor_flop_executed_per_launch": executed,
                  "tensor_achieved_executed": 2 * executed / t_dom / 1e12,
                  "tensor_frac_executed": 2 * executed / t_dom / 1e12 / bf16_peak}
        # the ring FFTs (one launch per FFT-length class and direction; a "launch" below is the
        # whole direction, all its class launches) and the tile preps: HBM-bound
        traffic = load_traffic()
        fft_bytes = hbm_bytes_ring_fft(B, mmax, g.npairs, npix)
        hbm_src = "MEASURED_PEAKS.json hbm_gbs, of measured" if peaks else "fallback 6650 GB/s, of fallback"
        stage_roof = {"tensor_legendre": tensor}
        for key, kern in (("ring_synthesis", "ring_quad_synthesis_kernel + ring_pair_synthesis_kernel + "
                                             "ring_synthesis_kernel<float>"),
                          ("ring_analysis", "ring_quad_analysis_kernel + ring_pair_analysis_kernel + "
                                            "ring_analysis_kernel<float>")):
            ach = fft_bytes / (stages[key] * 1e-3) / 1e9
            stage_roof[key] = {"bound": "hbm", "kernel": kern + " (all FFT-length classes of one direction)",
                               "achieved": ach, "peak": hbm_peak, "unit": "GB/s", "frac": ach / hbm_peak,
                               "traffic": traffic.get(f"{key}_nside{nside}_maps{B}"), "peak_source": hbm_src,
                               "bytes_per_launch": fft_bytes, "ms": stages[key]}
        # the preps read their operand once and write the hi/lo tiles, which hold as many bytes
        for key, kern, nbytes in (("prep_alm", "prep_alm_tiles_kernel", 2 * 8 * B * nalm),
                                  ("prep_f", "prep_f_tiles_kernel", 2 * hbm_bytes_ring_fft(B, mmax, g.npairs, 0))):
            ach = nbytes / (stages[key] * 1e-3) / 1e9
            stage_roof[key] = {"bound": "hbm", "kernel": kern, "achieved": ach, "peak": hbm_peak, "unit": "GB/s",
                               "frac": ach / hbm_peak, "traffic": traffic.get(f"{key}_nside{nside}_maps{B}"),
                               "peak_source": hbm_src, "bytes_per_launch": nbytes, "ms": stages[key]}
        tensor["ms"] = stages["tensor_synthesis"] + stages["tensor_analysis"]
        dom = max(stage_roof, key=lambda k: stage_roof[k]["ms"])
        roof = dict(stage_roof[dom])
        roof["stage"] = dom
    out = {
        "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (Gaussian alm, C_l=(l+10)^-2)",
        "config": {"workload": (f"scalar map2alm+alm2map pair, nside {nside}, lmax {lmax}, float32 maps, "
                                + (f"batched hi+lo split-{'BF16' if bf16 else 'F16'} tcgen05 path"
                                   f" ({'64' if wide else '32'} maps per group"
                                   f"{', autotuned' if tune else ''}), " if args.mode == "batched"
                                   else "plain per-map FP32 path, ") + f"{B} maps per GPU per step"),
                   "nside": nside, "lmax": lmax, "maps_per_gpu": B, "mode": args.mode,
                   "l2": "inputs larger than L2 (one map 201 MB, one alm 67 MB)",
                   "parallelism": f"replicas x{world}"},
        "rel_err_vs_fp64": relerr,
        "stages_ms": stages,
        "roofline": roof,
        "e2e": {"value": e2e, "unit": "pairs/s", "h2d_bytes_per_step": int(alm_pin.numel() * 8),
                "d2h_bytes_per_step": int(out_pin.numel() * 8), "steps": e2e_steps,
                "api": ("hp_compat.alm2map / map2alm per step" if args.mode == "plain"
                        else "batched.HostPipeline: pinned host alm in, copies overlapped with the transforms")},
        "gpu_launches": args.steps * n_launch,
        "clocks": clk.summary(),
    }
    if args.mode == "batched":
        out["stages_roofline"] = stage_roof
    if args.mode == "batched" and not args.no_extras:
        del maps, alm_out
        if args.mode == "batched":
            del pipe
        torch.cuda.empty_cache()
        pv, pms = plain_leg(hb, L, G, nside, lmax, min(args.plain_maps, B), alm_h, dev, st)
        out["plain_value"] = pv
        out["plain_ms_per_map"] = pms
        out["batched_over_plain"] = value / world / pv
        f_ms, ratio = diff_leg(hb, nside, lmax, dev, st)
        out["diff_forward_ms"] = f_ms
        out["diff_fwd_bwd_over_fwd"] = ratio
    if args.mode == "batched" and tune is not None:
        out["autotune"] = [{k: (round(v, 8) if isinstance(v, float) else v) for k, v in c.items()}
                           for c in tune["candidates"]]
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, info = cpu_baseline(nside, lmax, args.cpu_sample_m)
        out["cpu_baseline"] = {"value": v, "unit": "pairs/s", "cores": info["cores"], "kind": info["kind"],
                               "sample": info["sample"]}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
