"""Array plumbing at the Python boundary: numpy (the reference's array type)
or torch tensors in, device tensors for the kernels, results back in the
caller's type.  No arithmetic happens here."""
from __future__ import annotations

import numpy as np
import torch

from .runtime import require_cuda


def is_numpy(a) -> bool:
    return isinstance(a, np.ndarray)


def to_device(a, dtype=None, device=None) -> torch.Tensor:
    require_cuda()
    if isinstance(a, torch.Tensor):
        t = a
        if device is None:
            device = t.device if t.is_cuda else torch.device("cuda", torch.cuda.current_device())
        if dtype is None:
            dtype = t.dtype if t.dtype in (torch.float32, torch.float64) else torch.float64
        return t.to(device=device, dtype=dtype)
    arr = np.asarray(a)
    if dtype is None:
        dtype = torch.float32 if arr.dtype == np.float32 else torch.float64
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device())
    return torch.as_tensor(np.ascontiguousarray(arr), dtype=dtype).to(device)


def like_input(t: torch.Tensor, ref):
    """Return t as numpy if ref is numpy, else as a tensor on ref's device."""
    if is_numpy(ref):
        return t.detach().cpu().numpy().astype(ref.dtype if ref.dtype in (np.float32, np.float64) else np.float64)
    return t
