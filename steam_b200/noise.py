"""World-keyed counter noise (steam/noise.py).

The draw at a world lattice site is a pure function of (class key, site):
Philox4x32-10 over counter (ix, iy, iz, key2) with key (key0, key1), its
words 0 and 1 mapped to the float32 lattice (r >> 8) * 2^-24.  Any region's
noise is therefore the exact restriction of the world's.  The generator runs
in ``steam_keyed_uniforms`` / ``steam_levy_field`` on the device; the index
bookkeeping below is host-side and small.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._device import is_tensor, to_host


def class_key(seed_sequence):
    """The 96-bit Philox key of one size class from its SeedSequence child
    (steam/noise.py:133-146)."""
    if not isinstance(seed_sequence, np.random.SeedSequence):
        seed_sequence = np.random.SeedSequence(seed_sequence)
    state = seed_sequence.generate_state(3, dtype=np.uint32)
    return (np.uint64(state[0]), np.uint64(state[1]), np.uint64(state[2]))


def center_indices(n, origin, world_n, factor, wrap):
    """Turbulon-centre cells of one axis as (local, world) index arrays
    (steam/noise.py:149-182): the divisibility test applies to the wrapped
    world index."""
    local = np.arange(int(n), dtype=np.int64)
    world = local + int(origin)
    if wrap:
        world = world % int(world_n)
    keep = (world % int(factor)) == 0
    return local[keep], world[keep]


def keyed_uniforms(world_ix, world_iy, world_iz, key0, key1, key2, lane0, lane1):
    """Fill two flat float32 lanes with the uniforms of a world index box, C
    order over (ix, iy, iz) (steam/noise.py:103-130).

    numpy lanes are filled in place (transfers inside the call); CUDA tensor
    index vectors and lanes stay on the device.
    """
    torch = _lib.require_cuda("keyed_uniforms")
    lib = _lib.load()
    on_device = is_tensor(lane0)
    idx = []
    for v in (world_ix, world_iy, world_iz):
        if is_tensor(v):
            idx.append(v.to(device='cuda', dtype=torch.int64).contiguous())
        else:
            idx.append(torch.as_tensor(np.ascontiguousarray(v, dtype=np.int64), device='cuda'))
    if int(idx[1].numel()) and (int(idx[1].min().item()) < 0 or
                                int(idx[1].max().item()) > 0xFFFFFFFF):
        raise ValueError("keyed_uniforms: world_iy must lie in [0, 2^32)")
    n = int(idx[0].numel() * idx[1].numel() * idx[2].numel())
    if on_device:
        l0, l1 = lane0, lane1
        if l0.dtype != torch.float32 or l1.dtype != torch.float32:
            raise TypeError("keyed_uniforms: lanes must be float32")
    else:
        l0 = torch.empty(n, dtype=torch.float32, device='cuda')
        l1 = torch.empty(n, dtype=torch.float32, device='cuda')
    if l0.numel() < n or l1.numel() < n:
        raise ValueError(f"keyed_uniforms: lanes hold fewer than nx*ny*nz = {n} values")
    _lib.check(lib.steam_keyed_uniforms(
        _lib.ptr(idx[0]), idx[0].numel(), _lib.ptr(idx[1]), idx[1].numel(),
        _lib.ptr(idx[2]), idx[2].numel(), int(key0) & 0xFFFFFFFF, int(key1) & 0xFFFFFFFF,
        int(key2) & 0xFFFFFFFF, _lib.ptr(l0), _lib.ptr(l1), _lib.stream()))
    if not on_device:
        lane0[:n] = to_host(l0)
        lane1[:n] = to_host(l1)
