"""Host <-> device plumbing for the reference-signature entry points.

Every public function accepts either numpy arrays (the reference's calling
convention: host arrays in, host arrays out, transfers inside the call) or
CUDA torch tensors (the resident form: nothing leaves the device).
"""

from __future__ import annotations

import numpy as np

from . import _lib


def check_device(device, who):
    if device not in (None, 'cuda') and not str(device).startswith('cuda'):
        raise ValueError(
            f"{who}: steam_b200 computes on CUDA only (device={device!r}); "
            f"there is no host path in this package")
    return _lib.require_cuda(who)


def is_tensor(a) -> bool:
    try:
        import torch
    except ImportError:  # pragma: no cover
        return False
    return isinstance(a, torch.Tensor)


def to_device(a, dtype=None, copy=False):
    """(tensor, host_array_or_None).  Numpy input is uploaded (contiguous);
    tensors must already live on a CUDA device."""
    import torch
    if is_tensor(a):
        if not a.is_cuda:
            raise ValueError("steam_b200: tensor arguments must be CUDA tensors")
        t = a
        if dtype is not None and t.dtype != dtype:
            t = t.to(dtype)
        if not t.is_contiguous():
            t = t.contiguous()
        elif copy:
            t = t.clone()
        return t, None
    host = np.asarray(a)
    if dtype is None:
        dtype = torch.float64 if host.dtype == np.float64 else torch.float32
    t = torch.from_numpy(np.ascontiguousarray(host)).to(device='cuda', dtype=dtype)
    return t, host


def torch_dtype(np_dtype):
    import torch
    return torch.float64 if np.dtype(np_dtype) == np.float64 else torch.float32


def to_host(t, out=None):
    """Copy a device tensor back; into ``out`` (a numpy array) when given.
    A contiguous ``out`` of the same dtype receives the copy directly (one DMA
    when its memory is pinned)."""
    import torch
    if out is not None:
        if (out.flags.c_contiguous and out.flags.writeable and out.shape == tuple(t.shape)
                and np.dtype(out.dtype) == np.dtype(str(t.dtype).replace('torch.', ''))):
            torch.from_numpy(out).copy_(t)
        else:
            out[...] = t.detach().cpu().numpy()
        return out
    return t.detach().cpu().numpy()
