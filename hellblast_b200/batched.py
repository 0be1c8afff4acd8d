"""Batched split-precision transforms (16-bit hi+lo three-pass products on the tcgen05 tensor
cores, FP32 accumulation in TMEM): many maps of one or several (nside, lmax) in one persistent
launch per direction.  Wraps hb_batched_plan_* of the C ABI.

The default split is IEEE half with exact power-of-two per-m scaling (``bf16=True``: BF16).
Maps run in groups of 32 with four TMEM accumulator sets per output tile (``wide=True``: groups
of 64 with two sets, fewer recursion passes, about twice the accumulation error)."""
from __future__ import annotations

import ctypes
import threading

import torch

from . import _lib as L
from . import geometry as G
from .ops import alm_size

_cache: dict[tuple, "BatchedPlan"] = {}
_lock = threading.Lock()


class BatchedPlan:
    """``specs``: list of (geometry, lmax, mmax, nmaps).  Inputs/outputs are flat CUDA tensors
    holding the maps (float32) or alm (complex64, healpy layout) of all specs back to back."""

    def __init__(self, specs, bf16: bool = False, wide: bool = False):
        self.specs = [(g, int(lmax), int(lmax if mmax is None else mmax), int(n)) for g, lmax, mmax, n in specs]
        self.plans = [G.plan(g, lmax, mmax, precision=32) for g, lmax, mmax, _ in self.specs]
        n = len(self.plans)
        arr = (ctypes.c_void_p * n)(*[p.handle.value for p in self.plans])
        nm = (ctypes.c_int * n)(*[s[3] for s in self.specs])
        out = ctypes.c_void_p()
        flags = (L.HB_BATCHED_BF16 if bf16 else 0) | (L.HB_BATCHED_WIDE if wide else 0)
        L.call("hb_batched_plan_create", arr, nm, n, flags, ctypes.byref(out))
        self.bf16 = bf16
        self.wide = wide
        self.handle = out
        self.nbytes = int(L.lib().hb_batched_plan_bytes(out))
        self.total_pix = sum(g.npix * k for g, _, _, k in self.specs)
        self.total_alm = sum(alm_size(l, m) * k for _, l, m, k in self.specs)

    def alm2map(self, alm: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        alm = alm.reshape(-1).contiguous()
        if alm.dtype != torch.complex64 or alm.numel() != self.total_alm or not alm.is_cuda:
            raise ValueError(f"alm must be a CUDA complex64 tensor of {self.total_alm} elements")
        out = torch.empty(self.total_pix, dtype=torch.float32, device=alm.device) if out is None else out
        L.call("hb_batched_alm2map", self.handle, alm.data_ptr(), out.data_ptr(),
               torch.cuda.current_stream(alm.device).cuda_stream)
        return out

    def map2alm(self, maps: torch.Tensor, out: torch.Tensor | None = None, fl: torch.Tensor | None = None) -> torch.Tensor:
        """maps -> alm; with ``fl`` (a per-l filter, >= max lmax + 1 values) every alm(l, m) is
        multiplied by fl[l] in the tensor-core kernel's store (almxfl fused)."""
        maps = maps.reshape(-1).contiguous()
        if maps.dtype != torch.float32 or maps.numel() != self.total_pix or not maps.is_cuda:
            raise ValueError(f"maps must be a CUDA float32 tensor of {self.total_pix} elements")
        out = torch.empty(self.total_alm, dtype=torch.complex64, device=maps.device) if out is None else out
        if fl is not None:
            fl = torch.as_tensor(fl, dtype=torch.float32, device=maps.device).contiguous()
            if fl.numel() < max(s[1] for s in self.specs) + 1:
                raise ValueError("fl needs at least lmax + 1 entries")
        L.call("hb_batched_map2alm_fl", self.handle, maps.data_ptr(), out.data_ptr(),
               None if fl is None else fl.data_ptr(), torch.cuda.current_stream(maps.device).cuda_stream)
        return out

    def capture(self, alm: torch.Tensor | None, maps: torch.Tensor, out: torch.Tensor | None) -> None:
        """Record alm2map(alm -> maps) then map2alm(maps -> out) (either direction may be None)
        into a CUDA graph owned by the plan; ``replay()`` then runs the whole step as one graph
        launch.  The tensors' storage is baked into the graph: keep them alive and in place."""
        for t, dt, n in ((alm, torch.complex64, self.total_alm), (maps, torch.float32, self.total_pix),
                         (out, torch.complex64, self.total_alm)):
            if t is not None and (t.dtype != dt or t.numel() != n or not t.is_cuda or not t.is_contiguous()):
                raise ValueError("capture: buffers must be contiguous CUDA tensors of the plan's sizes")
        self._graph_buffers = (alm, maps, out)
        L.call("hb_batched_graph_capture", self.handle, None if alm is None else alm.data_ptr(), maps.data_ptr(),
               None if out is None else out.data_ptr())

    def replay(self, stream: torch.cuda.Stream | None = None) -> None:
        st = torch.cuda.current_stream() if stream is None else stream
        L.call("hb_batched_graph_launch", self.handle, st.cuda_stream)

    def profile(self, enable: bool = True) -> None:
        L.call("hb_batched_profile", self.handle, 1 if enable else 0)

    def stage_ms(self) -> dict:
        ms = (ctypes.c_float * 6)()
        L.call("hb_batched_stage_ms", self.handle, ms)
        keys = ("prep_alm", "tensor_synthesis", "ring_synthesis", "ring_analysis", "prep_f", "tensor_analysis")
        return dict(zip(keys, [float(v) for v in ms]))

    def executed_mma_flop(self) -> dict:
        """Tensor-core FLOP one alm2map / one map2alm call executes (after the evanescent skip):
        the work of 12 MMAs of 128 x N x 16 per live chunk (issued as 4 of width 2N and 4 of width N)."""
        ch = (ctypes.c_int64 * 2)()
        n = ctypes.c_int(0)
        L.call("hb_batched_work", self.handle, ch, ctypes.byref(n))
        per_chunk = 12 * 2 * 128 * n.value * 16
        return {"synthesis": ch[0] * per_chunk, "analysis": ch[1] * per_chunk, "mma_n": n.value}

    def status(self) -> int:
        code = ctypes.c_int(0)
        L.call("hb_batched_status", self.handle, ctypes.byref(code))
        return code.value

    def reset_status(self) -> None:
        L.call("hb_batched_reset_status", self.handle)

    def fault_test(self, wait_s: float = 2.0, withhold_copy: bool = False) -> None:
        """Failure-detection test hook: bound of every tensor-core pipeline wait, and whether the
        synthesis loader of CTA 0 withholds its first batch-tile copy (hb_batched_fault_test)."""
        L.call("hb_batched_fault_test", self.handle, int(wait_s * 1e9), 1 if withhold_copy else 0)

    def __del__(self):  # pragma: no cover
        try:
            if self.handle:
                L.lib().hb_batched_plan_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


def plan(nside: int, lmax: int, nmaps: int, mmax: int | None = None, weights: str = "dz",
         bf16: bool = False, wide: bool = False, tuned: bool = False) -> BatchedPlan:
    """Cached single-geometry batched plan (HEALPix nside, lmax, nmaps maps).  ``bf16`` selects
    the BF16 hi+lo split instead of the default IEEE-half hi+lo split, ``wide`` groups of 64 maps;
    ``tuned`` takes both from ``autotune(nside, lmax, nmaps)`` (measured on first use)."""
    if tuned:
        t = autotune(nside, lmax, nmaps)
        bf16, wide = t["bf16"], t["wide"]
    key = (int(nside), int(lmax), mmax, int(nmaps), weights, bool(bf16), bool(wide), torch.cuda.current_device())
    with _lock:
        bp = _cache.get(key)
    if bp is None:
        bp = BatchedPlan([(G.healpix(nside, weights=weights), lmax, mmax, nmaps)], bf16=bf16, wide=wide)
        with _lock:
            _cache[key] = bp
    return bp


def alm2map(alm: torch.Tensor, nside: int, lmax: int, mmax: int | None = None, bf16: bool = False,
            wide: bool = False) -> torch.Tensor:
    """[nmaps, nalm] complex64 -> [nmaps, npix] float32 through the tensor-core path."""
    nmaps = alm.shape[0]
    return plan(nside, lmax, nmaps, mmax, bf16=bf16, wide=wide).alm2map(alm).reshape(nmaps, -1)


def map2alm(maps: torch.Tensor, nside: int, lmax: int, mmax: int | None = None, bf16: bool = False,
            wide: bool = False) -> torch.Tensor:
    """[nmaps, npix] float32 -> [nmaps, nalm] complex64 through the tensor-core path."""
    nmaps = maps.shape[0]
    return plan(nside, lmax, nmaps, mmax, bf16=bf16, wide=wide).map2alm(maps).reshape(nmaps, -1)


class HostPipeline:
    """Streams batches held in pinned host memory through a batched plan: alm2map + map2alm of
    batch i runs on a compute stream while batch i+1 is copied in and batch i-1's alm is copied
    out on two copy streams (two device buffer sets, CUDA events between the streams).

    ``run(inputs, outputs)`` takes lists of pinned complex64 host tensors of the plan's alm size
    (outputs receive map2alm(alm2map(input))); it returns after queueing all work, and
    ``synchronize()`` waits for the last copy out."""

    def __init__(self, bp: BatchedPlan, device=None):
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.bp = bp
        self.dev = dev
        self.s_in, self.s_run, self.s_out = (torch.cuda.Stream(dev) for _ in range(3))
        self.alm = [torch.empty(bp.total_alm, dtype=torch.complex64, device=dev) for _ in range(2)]
        self.res = [torch.empty(bp.total_alm, dtype=torch.complex64, device=dev) for _ in range(2)]
        self.maps = torch.empty(bp.total_pix, dtype=torch.float32, device=dev)
        self.in_ready = [torch.cuda.Event() for _ in range(2)]
        self.ran = [torch.cuda.Event() for _ in range(2)]
        self.copied = [torch.cuda.Event() for _ in range(2)]
        self.used = [False, False]

    def run(self, inputs, outputs):
        for x in list(inputs) + list(outputs):
            if x.is_cuda or x.dtype != torch.complex64 or x.numel() != self.bp.total_alm or not x.is_pinned():
                raise ValueError("HostPipeline.run takes pinned complex64 host tensors of the plan's alm size")
        for i, (hin, hout) in enumerate(zip(inputs, outputs)):
            s = i & 1
            if self.used[s]:  # buffer set s is free once batch i-2 ran and was copied out
                self.s_in.wait_event(self.ran[s])
            with torch.cuda.stream(self.s_in):
                self.alm[s].copy_(hin.reshape(-1), non_blocking=True)
                self.in_ready[s].record(self.s_in)
            self.s_run.wait_event(self.in_ready[s])
            if self.used[s]:
                self.s_run.wait_event(self.copied[s])
            with torch.cuda.stream(self.s_run):
                self.bp.alm2map(self.alm[s], out=self.maps)
                self.bp.map2alm(self.maps, out=self.res[s])
                self.ran[s].record(self.s_run)
            self.s_out.wait_event(self.ran[s])
            with torch.cuda.stream(self.s_out):
                hout.reshape(-1).copy_(self.res[s], non_blocking=True)
                self.copied[s].record(self.s_out)
            self.used[s] = True

    def wait_on(self, stream: torch.cuda.Stream) -> None:
        """Make `stream` wait for everything queued so far (for timing with events on it)."""
        for s in (self.s_in, self.s_run, self.s_out):
            stream.wait_stream(s)

    def synchronize(self) -> None:
        self.s_out.synchronize()


_tuned: dict[tuple, dict] = {}


def autotune_cache_path() -> str:
    """JSON file that keeps autotune results across processes: $HB_AUTOTUNE_CACHE, else
    ~/.cache/hellblast_b200/autotune.json."""
    import os
    return os.environ.get("HB_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "hellblast_b200", "autotune.json"))


def _cache_key(key: tuple) -> str:
    return "|".join(str(k) for k in key) + "|" + L.lib().hb_version().decode()


def _cache_load() -> dict:
    import json
    try:
        with open(autotune_cache_path()) as f:
            d = json.load(f)
        return d if isinstance(d, dict) else {}
    except (OSError, ValueError):
        return {}


def _cache_store(key: tuple, result: dict) -> None:
    """Add one result to the JSON cache (rewritten atomically; failures to write are ignored:
    the cache only saves time)."""
    import json
    import os
    import tempfile
    path = autotune_cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        d = _cache_load()
        d[_cache_key(key)] = result
        fd, tmp = tempfile.mkstemp(dir=os.path.dirname(path), suffix=".tmp")
        with os.fdopen(fd, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass


def autotune(nside: int, lmax: int, nmaps: int, tol: float = 1e-5, reps: int = 2, seed: int = 0,
             candidates=((False, False), (False, True), (True, False), (True, True)), use_cache: bool = True) -> dict:
    """Chooses the batched tile configuration for (nside, lmax, nmaps) on this GPU by measurement.

    Each candidate (bf16, wide) is a 16-bit split type (IEEE half with power-of-two scaling, or
    BF16) and an MMA tile width (N = 64: 32 maps per recursion pass, or N = 128: 64 maps per
    pass).  For each, a plan is built, one alm2map + map2alm pair over `nmaps` synthetic maps is
    timed with CUDA events (after a warm-up), and map 0's pair error against the FP64 transforms
    is measured.  The fastest candidate with error <= tol wins; the result (with every
    candidate's time and error) is cached per (nside, lmax, nmaps, device) in the process and in
    a JSON file (autotune_cache_path(), keyed also by the library version; ``use_cache=False``
    measures afresh), and ``plan(..., tuned=True)`` uses it.  The candidates' plans are released again (each holds its operand
    tiles)."""
    from .alm_ops import synalm
    from . import hp_compat
    dev = torch.device("cuda", torch.cuda.current_device())
    key = (int(nside), int(lmax), int(nmaps), torch.cuda.get_device_name(dev))
    if key in _tuned:
        return _tuned[key]
    if use_cache:
        hit = _cache_load().get(_cache_key(key))
        if isinstance(hit, dict) and {"bf16", "wide", "candidates"} <= set(hit):
            _tuned[key] = hit
            return hit
    cl = 1.0 / (torch.arange(lmax + 1, dtype=torch.float64) + 10.0) ** 2
    a64 = synalm(cl.numpy(), lmax=lmax, seed=seed, device=dev)
    m64 = hp_compat.alm2map(a64, nside, lmax=lmax)
    ref = hp_compat.map2alm(m64, lmax=lmax)
    alm = a64.to(torch.complex64).expand(nmaps, -1).contiguous().reshape(-1)
    results = []
    for bf16, wide in candidates:
        bp = BatchedPlan([(G.healpix(nside), lmax, None, nmaps)], bf16=bf16, wide=wide)
        maps = torch.empty(bp.total_pix, dtype=torch.float32, device=dev)
        out = torch.empty_like(alm)
        bp.alm2map(alm, out=maps)
        bp.map2alm(maps, out=out)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            bp.alm2map(alm, out=maps)
            bp.map2alm(maps, out=out)
        e1.record()
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / reps
        got = out[: ref.numel()].to(torch.complex128)
        err = float(torch.linalg.norm(got - ref) / torch.linalg.norm(ref))
        ok = bp.status() == 0 and err <= tol
        results.append({"bf16": bf16, "wide": wide, "ms": ms, "rel_err": err, "ok": ok})
        del bp, maps, out
        torch.cuda.empty_cache()
    good = [r for r in results if r["ok"]]
    best = min(good, key=lambda r: r["ms"]) if good else min(results, key=lambda r: r["rel_err"])
    _tuned[key] = {"bf16": best["bf16"], "wide": best["wide"], "candidates": results}
    if use_cache:
        _cache_store(key, _tuned[key])
    return _tuned[key]
