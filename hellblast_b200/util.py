"""Array interchange: torch CUDA tensors are the native type; CuPy arrays arrive and leave
through DLPack; numpy arrays are copied to the current CUDA device."""
from __future__ import annotations

import numpy as np
import torch


def _is_cupy(x) -> bool:
    return type(x).__module__.split(".")[0] == "cupy"


def as_tensor(x, dtype=None) -> torch.Tensor:
    """Tensor view/copy of x (torch tensor, CuPy array via DLPack, numpy, list).  Host arrays
    move to the current CUDA device; torch tensors keep their device (the transform ops then
    reject CPU tensors: there is no CPU path)."""
    if isinstance(x, torch.Tensor):
        t = x
    elif _is_cupy(x):
        t = torch.from_dlpack(x)
    else:
        t = torch.from_numpy(np.ascontiguousarray(np.asarray(x)))
        if torch.cuda.is_available():
            t = t.to("cuda")
    if dtype is not None and t.dtype != dtype:
        t = t.to(dtype)
    return t


def like_input(t: torch.Tensor, ref):
    """Return t as a CuPy array (DLPack) when ref was one, else as a torch tensor."""
    if _is_cupy(ref):
        import cupy  # noqa: F401  (only reachable when the caller already uses CuPy)
        return cupy.from_dlpack(t)
    return t


def flatten_rings(rings, dtype=None) -> torch.Tensor:
    """A list of per-ring arrays (the reference's input form, sht_raw.py:38-40) or a flat
    array -> one contiguous flat CUDA tensor."""
    if isinstance(rings, (list, tuple)):
        parts = [as_tensor(r) for r in rings]
        t = torch.cat([p.reshape(-1) for p in parts])
    else:
        t = as_tensor(rings)
    if dtype is not None and t.dtype != dtype:
        t = t.to(dtype)
    return t.contiguous()


def host_array(x, dtype) -> np.ndarray:
    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy().astype(dtype)
    if _is_cupy(x):
        return np.asarray(x.get(), dtype=dtype)
    return np.asarray(x, dtype=dtype)
