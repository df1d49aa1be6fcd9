"""Device-memory plumbing: torch tensors carry the buffers, the CUDA engine does the math."""

from __future__ import annotations

import ctypes

import numpy as np
import torch


def require_cuda() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("pyftle_b200 needs a CUDA device (sm_100a); none is visible")
    return torch.device("cuda", torch.cuda.current_device())


def as_device_f64(x, *, copy: bool = False) -> torch.Tensor:
    """Contiguous float64 CUDA tensor holding x (numpy array, sequence or tensor)."""
    dev = require_cuda()
    if isinstance(x, torch.Tensor):
        pinned = (not x.is_cuda) and x.is_pinned()
        t = x.to(device=dev, dtype=torch.float64, non_blocking=pinned)
        if copy and t.data_ptr() == x.data_ptr():
            t = t.clone()
        return t.contiguous()
    arr = np.ascontiguousarray(np.asarray(x, dtype=np.float64))
    return torch.from_numpy(arr).to(dev, non_blocking=False)


def to_host(x) -> np.ndarray:
    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy()
    return np.asarray(x)


def ptr(t: torch.Tensor | None) -> ctypes.c_void_p:
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def stream_ptr(stream: torch.cuda.Stream | None = None) -> ctypes.c_void_p:
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)
