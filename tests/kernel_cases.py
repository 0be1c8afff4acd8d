"""Seeded, self-contained invocations of each kernel family, timed with CUDA events on the
launching stream: the command line a user (or an ncu capture) runs to time or profile one part
of the transform in isolation.

    python tests/kernel_cases.py CASE [--nside N] [--lmax L] [--nmaps B] [--reps R]

CASE is one of
  ring_tables  hb_ring_tables (HealpixRingTables, ring_tables.py:17-37 of the reference)
  plain        FP32 alm2map + map2alm per map (leg_*_kernel, ring_*_kernel)
  spin         FP32 spin-2 alm2map + map2alm (spin_*_kernel)
  alm2cl       hb_alm2cl on B alm vectors (alm_ops.py:19-32)
  ring         FP32 ring synthesis + ring analysis alone (hb_ring_synthesis / hb_ring_analysis;
               ring_pair_*, ring_quad_* and ring_*_kernel<float>) on B maps of Gaussian G(m)
  batched      batched split-precision alm2map + map2alm (synth_tc/anal_tc + ring FFTs)
  diff         the differentiable T/Q/U power-spectrum loss: forward, and forward + backward
               through the adjoint kernels; prints both times and their ratio

Inputs: Gaussian alm with C_l = (l+10)^-2 (EE = 0.1 TT, BB = 0.01 TT), numpy seed 2.  One JSON
line per case on stdout.
"""
from __future__ import annotations

import argparse
import json

import os
import sys

import numpy as np
import torch

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from hellblast_b200 import _lib as L  # noqa: E402
from hellblast_b200 import alm_ops, autograd, batched, ops  # noqa: E402
from hellblast_b200 import geometry as G  # noqa: E402
from hellblast_b200.ring_tables import HealpixRingTables  # noqa: E402


def _time(fn, reps, warmup, st):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    for a, b in ev:
        a.record(st)
        fn()
        b.record(st)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev]


def _alm(lmax, nmaps, scale=1.0, seed=2):
    cl = scale / (np.arange(lmax + 1) + 10.0) ** 2
    one = alm_ops.synalm(cl, lmax=lmax, seed=seed, device="cuda", dtype=torch.complex64)
    return one.expand(nmaps, -1).contiguous()


def run(case: str, nside: int, lmax: int, nmaps: int, reps: int, warmup: int, wide: bool = False,
        bf16: bool = False) -> dict:
    dev = torch.device("cuda", torch.cuda.current_device())
    st = torch.cuda.current_stream(dev)
    out = {"case": case, "nside": nside, "lmax": lmax, "nmaps": nmaps}
    if case == "ring_tables":
        ms = _time(lambda: HealpixRingTables(nside, device=dev), reps, warmup, st)
    elif case in ("plain", "spin"):
        g = G.healpix(nside)
        spin = case == "spin"
        p = G.plan(g, lmax, lmax, precision=32, spin=spin)
        a = _alm(lmax, nmaps)
        if spin:
            b = _alm(lmax, nmaps, 0.1, seed=3)
            fn = lambda: ops.map2alm_spin2(*ops.alm2map_spin2(a, b, p.pid, 0), p.pid, None, 0)  # noqa: E731
        else:
            fn = lambda: ops.map2alm(ops.alm2map(a, p.pid, 0), p.pid, None, 0)  # noqa: E731
        ms = _time(fn, reps, warmup, st)
    elif case == "alm2cl":
        a = _alm(lmax, nmaps)
        ms = _time(lambda: ops.alm2cl(a, None, lmax, lmax), reps, warmup, st)
        out["bytes_read"] = a.numel() * a.element_size()
    elif case == "ring":
        g = G.healpix(nside)
        p = G.plan(g, lmax, precision=64)
        torch.manual_seed(2)
        Gm = torch.randn(nmaps, lmax + 1, g.npairs, 2, dtype=torch.complex64, device=dev)
        Gm[:, :, g.npairs - 1, 1] = 0  # the unpaired equator's south slot is not data
        mp = torch.empty(nmaps, g.npix, dtype=torch.float32, device=dev)
        F = torch.empty_like(Gm)
        sp = st.cuda_stream

        def fn():
            L.call("hb_ring_synthesis", p.handle, 32, nmaps, Gm.data_ptr(), mp.data_ptr(), 0, sp)
            L.call("hb_ring_analysis", p.handle, 32, nmaps, mp.data_ptr(), None, F.data_ptr(), 0, sp)
        ms = _time(fn, reps, warmup, st)
    elif case == "batched":
        bp = batched.plan(nside, lmax, nmaps, wide=wide, bf16=bf16)
        a = _alm(lmax, nmaps).reshape(-1)
        mp = torch.empty(bp.total_pix, dtype=torch.float32, device=dev)
        r = torch.empty_like(a)
        ms = _time(lambda: (bp.alm2map(a, out=mp), bp.map2alm(mp, out=r)), reps, warmup, st)
        if bp.status() != 0:
            raise RuntimeError(f"tensor-core pipeline reported error {bp.status()}")
    elif case == "diff":
        aT, aE, aB = _alm(lmax, 1), _alm(lmax, 1, 0.1, 3), _alm(lmax, 1, 0.01, 4)
        T = autograd.alm2map(aT, nside, lmax).detach()
        Q, U = (x.detach() for x in autograd.alm2map_spin(aE, aB, nside, lmax))
        with torch.no_grad():
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

        ms_f = _time(fwd, reps, warmup, st)
        ms = _time(fwd_bwd, reps, warmup, st)
        out["forward_ms"] = float(np.median(ms_f))
        out["ratio_fwd_bwd_over_fwd"] = float(np.median(ms)) / out["forward_ms"]
    else:
        raise ValueError(f"unknown case {case}")
    out["ms"] = [round(x, 4) for x in ms]
    out["median_ms"] = float(np.median(ms))
    return out


def main(argv=None):
    p = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    p.add_argument("case", choices=["ring_tables", "plain", "spin", "alm2cl", "ring", "batched", "diff"])
    p.add_argument("--nside", type=int, default=1024)
    p.add_argument("--lmax", type=int, default=None)
    p.add_argument("--nmaps", type=int, default=1)
    p.add_argument("--reps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=1)
    p.add_argument("--wide", action="store_true", help="batched: 64-map groups (MMA N = 128)")
    p.add_argument("--bf16", action="store_true", help="batched: BF16 hi+lo split (default IEEE half)")
    a = p.parse_args(argv)
    if not torch.cuda.is_available():
        raise SystemExit("kernel_cases needs a CUDA device (there is no CPU path)")
    L.lib()
    lmax = 2 * a.nside - 1 if a.lmax is None else a.lmax
    print(json.dumps(run(a.case, a.nside, lmax, a.nmaps, a.reps, a.warmup, a.wide, a.bf16)), flush=True)


if __name__ == "__main__":
    main()
