"""CPU tests of the drop-in boundary: the C-ABI library loads, exports every entry point that
include/hbsht.h declares, and rejects bad arguments on the host (no GPU work is launched)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "hbsht.h")


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"HB_API\s+[^;(]*?\b(hb_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    from hellblast_b200 import _lib as L
    lib = L.lib()
    syms = declared_symbols()
    assert len(syms) >= 28
    for s in syms:
        assert hasattr(lib, s), s
        assert s in L.SIGNATURES, f"{s} missing from the Python loader"


def test_exported_symbols_match_nm():
    import subprocess
    from hellblast_b200 import _lib as L
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (hb_[a-z0-9_]+)", out))
    assert set(declared_symbols()) <= exported
    # nothing else leaks out of the shared object under the hb_ prefix
    assert exported <= set(declared_symbols())


def test_alm_size_and_version():
    from hellblast_b200 import _lib as L
    lib = L.lib()
    assert lib.hb_alm_size(4095, 4095) == 4096 * 4097 // 2
    assert lib.hb_alm_size(10, 3) == 3 * (21 - 3) // 2 + 11
    assert lib.hb_alm_size(3, 4) == -1
    assert b"sm_100a" in lib.hb_version()


def test_host_side_argument_errors():
    from hellblast_b200 import _lib as L
    lib = L.lib()
    out = ctypes.c_void_p()
    assert lib.hb_geom_create_healpix(3, 0, 0, ctypes.byref(out)) == L.HB_ERR_INVALID
    assert b"power of 2" in lib.hb_last_error_string()
    assert lib.hb_geom_create_healpix(8, 7, 0, ctypes.byref(out)) == L.HB_ERR_INVALID
    assert lib.hb_ring_tables(6, 0, None, None, None, None, None, None, None, None) == L.HB_ERR_INVALID
    assert lib.hb_map2alm_f32(None, 1, None, None, None, None, 0, 0, None) == L.HB_ERR_INVALID
    assert b"null plan" in lib.hb_last_error_string()
    assert lib.hb_plan_create(None, 10, 10, 0, ctypes.byref(out)) == L.HB_ERR_INVALID
    assert lib.hb_alm2cl_f64(-1, 0, 1, None, None, None, None) == L.HB_ERR_INVALID
    th = np.array([0.5, 4.0]); nphi = np.array([4, 3], dtype=np.int32); w = np.ones(2)
    assert lib.hb_geom_create(2, th.ctypes.data, nphi.ctypes.data, None, w.ctypes.data,
                              ctypes.byref(out)) == L.HB_ERR_INVALID


def test_python_raises_on_error_status():
    from hellblast_b200 import _lib as L
    with pytest.raises(ValueError, match="power of 2"):
        L.call("hb_geom_create_healpix", 5, 0, 0, ctypes.byref(ctypes.c_void_p()))


def test_ops_reject_cpu_tensors():
    import torch
    import hellblast_b200 as hb
    with pytest.raises(ValueError, match="CUDA"):
        torch.ops.hb.alm2cl(torch.zeros(1, 6, dtype=torch.complex128), None, 2, 2)


def test_registered_torch_ops():
    import torch
    import hellblast_b200  # noqa: F401
    for name in ("map2alm", "alm2map", "map2alm_adjoint", "alm2map_adjoint", "map2alm_spin2", "alm2map_spin2",
                 "map2alm_spin2_adjoint", "alm2map_spin2_adjoint", "alm2cl"):
        assert hasattr(torch.ops.hb, name)
