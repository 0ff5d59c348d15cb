"""Device plumbing: PyTorch provides CUDA memory and streams, nothing else."""
from __future__ import annotations

import numpy as np


def torch():
    import torch as _t
    return _t


def require_cuda(device=None):
    """The CUDA device to run on; raises when no GPU is usable (no CPU fallback)."""
    t = torch()
    if not t.cuda.is_available():
        raise RuntimeError('ehss_b200 needs a CUDA device (B200, sm_100a); none is available')
    if isinstance(device, t.device):
        return device if device.index is not None else t.device('cuda', t.cuda.current_device())
    return t.device('cuda', t.cuda.current_device() if device is None else int(device))


def stream_handle(device=None):
    t = torch()
    return t.cuda.current_stream(device).cuda_stream


def to_device(a, dtype, device):
    """Copy a host array to a new contiguous device tensor."""
    t = torch()
    arr = np.ascontiguousarray(a, dtype=dtype)
    host = t.from_numpy(arr)
    return host.to(device, non_blocking=False)


def empty(shape, dtype, device):
    return torch().empty(shape, dtype=dtype, device=device)


def ptr(x):
    return None if x is None else x.data_ptr()
