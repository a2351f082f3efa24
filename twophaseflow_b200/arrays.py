"""Array plumbing between the reference's array types and device memory.

Inputs may be torch CUDA tensors (zero-copy), objects exposing
``__cuda_array_interface__`` (e.g. CuPy arrays; zero-copy through torch), or
host NumPy arrays (copied to the device through pinned memory; results are
copied back and returned as NumPy, matching the reference's CPU backend).
"""

from __future__ import annotations

import numpy as np


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("twophaseflow_b200 needs a CUDA device; no CPU fallback exists")
    return torch


class DeviceView:
    """A device tensor plus how to hand results back in the caller's type."""

    __slots__ = ("tensor", "host")

    def __init__(self, tensor, host: bool):
        self.tensor = tensor
        self.host = host

    def out(self, t):
        if self.host:
            return t.cpu().numpy()
        return t


def to_device(data, dtype=None, device=None) -> DeviceView:
    torch = _torch()
    dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
    if isinstance(data, torch.Tensor):
        t = data
        host = not t.is_cuda
        if host:
            t = t.pin_memory().to(dev, non_blocking=True) if t.device.type == "cpu" else t.to(dev)
    elif hasattr(data, "__cuda_array_interface__"):
        t = torch.as_tensor(data, device=dev)
        host = False
    else:
        arr = np.ascontiguousarray(np.asarray(data))
        t = torch.from_numpy(arr)
        t = t.pin_memory().to(dev, non_blocking=True)
        host = True
    if dtype is not None and t.dtype != dtype:
        t = t.to(dtype)
    if not t.is_contiguous():
        t = t.contiguous()
    return DeviceView(t, host)


def line_split(shape, axis):
    """(outer, n, inner) of a C-order array viewed along ``axis``."""
    outer = 1
    for s in shape[:axis]:
        outer *= int(s)
    inner = 1
    for s in shape[axis + 1:]:
        inner *= int(s)
    return outer, int(shape[axis]), inner
