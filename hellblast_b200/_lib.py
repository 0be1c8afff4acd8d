"""Loader for the C-ABI library ``hellblast_b200/_lib/libhbsht.so`` (include/hbsht.h).

There is no fallback: if the library is missing or fails to load, every transform raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libhbsht.so")

HB_OK = 0
HB_ERR_INVALID = -1
HB_ERR_UNSUPPORTED = -2
HB_ERR_CUDA = -3
HB_ERR_WORKSPACE = -4
HB_ERR_ALLOC = -5

HB_PHI0_HEALPIX = 0
HB_PHI0_REFERENCE = 1
HB_WEIGHTS_DZ = 0
HB_WEIGHTS_UNIFORM = 1
HB_F_NOPHASE = 1
HB_F_NOFOLD = 2
HB_F_NO2PI = 4
HB_PIX_NEST = 1
HB_PIX_REFERENCE = 2

_lock = threading.Lock()
_lib = None

vp = ctypes.c_void_p
i32 = ctypes.c_int
i64 = ctypes.c_int64
sz = ctypes.c_size_t

# name -> (restype, argtypes)
SIGNATURES = {
    "hb_last_error_string": (ctypes.c_char_p, []),
    "hb_version": (ctypes.c_char_p, []),
    "hb_alm_size": (i64, [i32, i32]),
    "hb_ring_tables": (i32, [i64, i32, vp, vp, vp, vp, vp, vp, vp, vp]),
    "hb_geom_create_healpix": (i32, [i64, i32, i32, ctypes.POINTER(vp)]),
    "hb_geom_create": (i32, [i64, vp, vp, vp, vp, ctypes.POINTER(vp)]),
    "hb_geom_destroy": (i32, [vp]),
    "hb_geom_fft_launches": (i32, [vp, i32, ctypes.POINTER(i32)]),
    "hb_geom_info": (i32, [vp, ctypes.POINTER(i64), ctypes.POINTER(i64), ctypes.POINTER(i64), ctypes.POINTER(i64)]),
    "hb_plan_create": (i32, [vp, i32, i32, i32, ctypes.POINTER(vp)]),
    "hb_plan_destroy": (i32, [vp]),
    "hb_plan_bytes": (sz, [vp]),
    "hb_sht_workspace_size": (sz, [vp, i32, i32]),
    "hb_spin2_workspace_size": (sz, [vp, i32, i32]),
    "hb_alm2cl_f32": (i32, [i32, i32, i32, vp, vp, vp, vp]),
    "hb_alm2cl_f64": (i32, [i32, i32, i32, vp, vp, vp, vp]),
    "hb_ring_analysis": (i32, [vp, i32, i32, vp, vp, vp, i32, vp]),
    "hb_ring_synthesis": (i32, [vp, i32, i32, vp, vp, i32, vp]),
    "hb_legendre_analysis": (i32, [vp, i32, i32, vp, vp, vp]),
    "hb_legendre_synthesis": (i32, [vp, i32, i32, vp, vp, vp]),
    "hb_legendre_analysis_ms": (i32, [vp, i32, i32, i32, vp, vp, vp, vp]),
    "hb_ring2nest": (i32, [i64, i64, vp, vp, vp, vp]),
    "hb_nest2ring": (i32, [i64, i64, vp, vp, vp, vp]),
    "hb_pix2ang": (i32, [i64, i32, vp, i64, vp, vp, vp, vp, vp]),
    "hb_ang2pix": (i32, [i64, i32, vp, vp, i64, vp, vp, vp, vp, vp]),
    "hb_reorder": (i32, [i64, i32, i32, i32, vp, vp, vp]),
    "hb_wigner_d": (i32, [i32, i32, vp, vp, vp]),
    "hb_rotate_alm": (i32, [i32, i32, vp, vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, vp]),
    "hb_legendre_synthesis_ms": (i32, [vp, i32, i32, i32, vp, vp, vp, vp]),
    "hb_probe_fp32": (i32, [i32, i32, i32, vp, vp]),
    "hb_batched_plan_create": (i32, [ctypes.POINTER(vp), ctypes.POINTER(i32), i32, i32, ctypes.POINTER(vp)]),
    "hb_batched_plan_destroy": (i32, [vp]),
    "hb_batched_plan_bytes": (sz, [vp]),
    "hb_batched_alm2map": (i32, [vp, vp, vp, vp]),
    "hb_batched_map2alm": (i32, [vp, vp, vp, vp]),
    "hb_batched_map2alm_fl": (i32, [vp, vp, vp, vp, vp]),
    "hb_batched_status": (i32, [vp, ctypes.POINTER(i32)]),
    "hb_batched_fault_test": (i32, [vp, ctypes.c_uint64, i32]),
    "hb_batched_reset_status": (i32, [vp]),
    "hb_batched_profile": (i32, [vp, i32]),
    "hb_batched_stage_ms": (i32, [vp, ctypes.POINTER(ctypes.c_float)]),
    "hb_batched_graph_capture": (i32, [vp, vp, vp, vp]),
    "hb_batched_work": (i32, [vp, ctypes.POINTER(i64), ctypes.POINTER(i32)]),
    "hb_batched_graph_launch": (i32, [vp, vp]),
}
for _p in ("f32", "f64"):
    SIGNATURES[f"hb_map2alm_{_p}"] = (i32, [vp, i32, vp, vp, vp, vp, sz, i32, vp])
    SIGNATURES[f"hb_alm2map_{_p}"] = (i32, [vp, i32, vp, vp, vp, sz, i32, vp])
    SIGNATURES[f"hb_alm2map_adjoint_{_p}"] = (i32, [vp, i32, vp, vp, vp, sz, i32, vp])
    SIGNATURES[f"hb_map2alm_adjoint_{_p}"] = (i32, [vp, i32, vp, vp, vp, vp, sz, i32, vp])
    SIGNATURES[f"hb_map2alm_spin2_{_p}"] = (i32, [vp, i32, vp, vp, vp, vp, vp, vp, sz, i32, vp])
    SIGNATURES[f"hb_alm2map_spin2_{_p}"] = (i32, [vp, i32, vp, vp, vp, vp, vp, sz, i32, vp])
    SIGNATURES[f"hb_alm2map_spin2_adjoint_{_p}"] = (i32, [vp, i32, vp, vp, vp, vp, vp, sz, i32, vp])
    SIGNATURES[f"hb_map2alm_spin2_adjoint_{_p}"] = (i32, [vp, i32, vp, vp, vp, vp, vp, vp, sz, i32, vp])
SIGNATURES["hb_map2alm_f32_noalloc"] = (i32, [vp, i32, vp, vp, vp, i32, vp])

HB_PLAN_FP32 = 1
HB_PLAN_SPIN2_FP32 = 2
HB_BATCHED_BF16 = 1
HB_BATCHED_WIDE = 2


class HBError(RuntimeError):
    """A C-ABI call returned an error status."""


def lib():
    """Load libhbsht.so once; raise if it is absent (no CPU fallback exists)."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise ImportError(
                        f"hellblast_b200: CUDA library {LIB_PATH} is missing; build it with "
                        "`python -c 'import __graft_entry__ as g; g.build()'` or `make -C hellblast_b200/csrc`")
                L = ctypes.CDLL(LIB_PATH)
                for name, (res, args) in SIGNATURES.items():
                    f = getattr(L, name)
                    f.restype = res
                    f.argtypes = args
                _lib = L
    return _lib


def check(rc: int, what: str) -> None:
    if rc == HB_OK:
        return
    msg = lib().hb_last_error_string().decode(errors="replace")
    if rc == HB_ERR_INVALID:
        raise ValueError(f"{what}: {msg}")
    if rc == HB_ERR_UNSUPPORTED:
        raise NotImplementedError(f"{what}: {msg}")
    raise HBError(f"{what} failed ({rc}): {msg}")


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args), name)
