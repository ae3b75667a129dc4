"""The reference's ``steam.streaming`` interface on the B200.

The reference streams a root run through host RAM in horizontal tiles
(steam/streaming.py:850-1447) because its fields outgrow a 16 GiB card and
host memory.  On a 180 GB B200 the cascade's fields stay resident in HBM
(a 2048 x 2048 x 256 root needs about 10.5 fields, 45 GB), so here the
"stream" is the output path: the final fields leave the device slab by slab
into a memory-mapped store on scratch disk, each slab copied into a
page-locked buffer on a second CUDA stream while the previous one is written
out, so the host never holds a whole field.

Kept from the reference: ``streamed_cascade_loop``'s signature and return
tuple, ``TilePlan`` / ``plan_tiling`` (the halo rule of
steam/streaming.py:672-796; the horizon is the whole cascade whenever it fits
the device), and a ``TileStore`` that stores fields z-major, (nz, nx, ny), as
(nx, ny, nz) views (steam/streaming.py:276-622), owns only its own subtree
and refuses to delete a directory without its manifest.  Resume after a crash
(``completed``) is not offered: nothing is paged mid-run, so there is no
half-finished state to resume.
"""

from __future__ import annotations

import json
import shutil
from pathlib import Path

import numpy as np

from . import _lib
from ._device import check_device

STORE_DIRNAME = "steam_b200_store"
STORE_SCHEMA = "steam_b200-tilestore-1"
PEAK_FIELDS = 10.5  # the cascade's concurrent peak in fields (steam/streaming.py:627)


class TilePlan:
    """Which classes stream, and over how many tiles (steam/streaming.py:635).

    ``horizon`` is the first class that would page through host memory; on the
    device path every class below it runs resident, and it equals the class
    count unless forced."""

    __slots__ = ('horizon', 'tiles', 'halo', 'peak_scratch_bytes')

    def __init__(self, horizon, tiles, halo, peak_scratch_bytes):
        self.horizon = int(horizon)
        self.tiles = dict(tiles)
        self.halo = tuple(int(h) for h in halo)
        self.peak_scratch_bytes = int(peak_scratch_bytes)

    def __repr__(self):
        return (f"TilePlan(horizon={self.horizon}, tiles={self.tiles}, "
                f"halo={self.halo}, scratch={self.peak_scratch_bytes / 1024**3:.2f} GiB)")


def _field_bytes(grids, index, elem=4):
    return int(grids['nx'][index]) * int(grids['ny'][index]) * int(grids['nz'][index]) * elem


def plan_tiling(grids, kernel_shape, budget_bytes=None, device='cuda', force=None,
                save_increments=False):
    """The plan for a root run.  Halo per side = the kernel's half width plus
    the advective stencil's one cell, per axis (steam/streaming.py:672-723).
    ``budget_bytes`` bounds the device memory of the cascade (default: the
    free HBM); a run that does not fit is refused up front with its numbers,
    as the reference refuses oversize work.  ``force`` = (horizon, tiles_x,
    tiles_y) is recorded as given."""
    if device not in (None, 'cuda') and not str(device).startswith('cuda'):
        raise ValueError(f"plan_tiling: steam_b200 plans for CUDA devices, got {device!r}")
    n_classes = len(grids['k'])
    kernel_shape = tuple(int(n) for n in kernel_shape)
    if len(kernel_shape) != 3:
        raise ValueError(f"kernel_shape must have 3 entries, got {kernel_shape}")
    halo = (kernel_shape[0] // 2 + 1, kernel_shape[1] // 2 + 1)
    last = n_classes - 1
    scratch = 3 * _field_bytes(grids, last) * (2 if save_increments else 1)
    if force is not None:
        horizon, tx, ty = (int(v) for v in force)
        tiles = {i: (tx, ty) for i in range(horizon, n_classes)}
        return TilePlan(horizon, tiles, halo, scratch)
    need = int(PEAK_FIELDS * _field_bytes(grids, last))
    if budget_bytes is None:
        torch = _lib.require_cuda("plan_tiling")
        budget_bytes = torch.cuda.mem_get_info()[0]
    if need > budget_bytes:
        raise MemoryError(f"plan_tiling: the finest class needs {need} bytes of device "
                          f"memory ({PEAK_FIELDS} fields of {_field_bytes(grids, last)} B); "
                          f"the budget is {int(budget_bytes)} bytes")
    return TilePlan(n_classes, {}, halo, scratch)


class TileStore:
    """Fields on scratch disk, one z-major .npy per (class, field), opened as
    (nx, ny, nz) memory-mapped views.  The store owns ``scratch_dir/<subdir>``
    and nothing else."""

    def __init__(self, scratch_dir, owned_root=None):
        self.scratch_dir = Path(scratch_dir)
        self.root = Path(owned_root) if owned_root is not None else \
            self.scratch_dir / STORE_DIRNAME
        self.root.mkdir(parents=True, exist_ok=True)
        manifest = self.root / "manifest.json"
        if not manifest.exists():
            if any(self.root.iterdir()):
                raise OSError(f"{self.root} is not empty and carries no {STORE_SCHEMA!r} "
                              f"manifest; refusing to adopt it")
            manifest.write_text(json.dumps({"schema": STORE_SCHEMA}))
        self._open = {}

    @property
    def directory(self):
        return self.root

    def read_manifest(self):
        try:
            m = json.loads((self.root / "manifest.json").read_text())
        except (OSError, ValueError):
            return None
        return m if m.get("schema") == STORE_SCHEMA else None

    def path(self, index, name):
        return self.root / f"c{int(index):03d}_{name}.npy"

    def exists(self, index, name):
        return self.path(index, name).exists()

    def create(self, index, name, shape, dtype=np.float32):
        """A new z-major file for an (nx, ny, nz) field; returns the raw
        (nz, nx, ny) memmap."""
        nx, ny, nz = (int(n) for n in shape)
        raw = np.lib.format.open_memmap(self.path(index, name), mode='w+', dtype=dtype,
                                        shape=(nz, nx, ny))
        self._open[(index, name)] = raw
        return raw

    def open(self, index, name):
        """The stored field as an (nx, ny, nz) view."""
        raw = self._open.get((index, name))
        if raw is None:
            raw = np.load(self.path(index, name), mmap_mode='r+')
            self._open[(index, name)] = raw
        return raw.transpose(1, 2, 0)

    def close(self, index, name):
        raw = self._open.pop((index, name), None)
        if raw is not None:
            raw.flush()

    def disk_bytes(self):
        return sum(p.stat().st_size for p in self.root.rglob('*') if p.is_file())

    def destroy(self):
        """Remove the store's own subtree, and nothing else."""
        for key in list(self._open):
            self.close(*key)
        if not self.root.exists():
            return
        if any(self.root.iterdir()) and self.read_manifest() is None:
            raise OSError(f"refusing to destroy {self.root}: it is not empty and carries no "
                          f"{STORE_SCHEMA!r} manifest")
        shutil.rmtree(self.root, ignore_errors=True)


def write_field(store, index, name, field_t, slab_levels=8):
    """Stream a device field into the store, z-major, through two page-locked
    slabs: the copy of slab k+1 (on a side stream) overlaps the disk write of
    slab k."""
    torch = _lib.require_cuda("TileStore")
    nx, ny, nz = (int(n) for n in field_t.shape)
    np_t = np.float64 if field_t.dtype == torch.float64 else np.float32
    raw = store.create(index, name, (nx, ny, nz), np_t)
    slab = max(1, min(int(slab_levels), nz))
    bufs = [torch.empty((slab, nx, ny), dtype=field_t.dtype, pin_memory=True)
            for _ in range(2)]
    zmaj = torch.empty((slab, nx, ny), dtype=field_t.dtype, device=field_t.device)
    lib = _lib.load()
    code = _lib.dtype_code(field_t)
    done = [torch.cuda.Event(), torch.cuda.Event()]
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    starts = list(range(0, nz, slab))

    def issue(k):
        z0 = starts[k]
        z1 = min(nz, z0 + slab)
        with torch.cuda.stream(side):
            # the (x, y, z) -> (z, x, y) reorder runs on the device; the copy
            # of slab k - 1 out of zmaj precedes this launch on the same stream
            _lib.check(lib.steam_slab_zmajor(code, nx, ny, nz, _lib.ptr(field_t), z0, z1 - z0,
                                             _lib.ptr(zmaj), _lib.stream()))
            bufs[k % 2][:z1 - z0].copy_(zmaj[:z1 - z0], non_blocking=True)
            done[k % 2].record(side)

    issue(0)
    for k in range(len(starts)):
        # slab k + 1 goes into the buffer the host finished reading at k - 1
        if k + 1 < len(starts):
            issue(k + 1)
        done[k % 2].synchronize()
        z0 = starts[k]
        z1 = min(nz, z0 + slab)
        raw[z0:z1] = bufs[k % 2][:z1 - z0].numpy()
    raw.flush()
    torch.cuda.current_stream().wait_stream(side)
    return raw.transpose(1, 2, 0)


def streamed_cascade_loop(h_profile, qt_profile, z_profile, grids, C_h_k, C_qt_k,
                          b_h_k, b_qt_k, aspect_k, h_min, h_max, qt_min, qt_max,
                          min_distance_to_ground, sparsity_factors, class_seeds, plan,
                          scratch_dir, n_scale_classes_per_dyad=1, flux_noise_scale=None,
                          turbulon_shape='mexican_hat', zero_bottom=True, zero_top=True,
                          device='cuda', comp_k=None, increment_store=None, completed=None,
                          _crash_hook=None, dtype=np.float32):
    """cascade_loop for a ROOT run with its fields delivered through a
    scratch store (steam/streaming.py:850-1447).

    Same arguments as the reference.  The cascade runs resident on the
    device; the final h', qt', F and any deficits are streamed into a
    ``TileStore`` under ``scratch_dir``.  Returns (h_perturbation,
    qt_perturbation, flux, deficit_h, deficit_qt, deficit_flux,
    final_grid_info, ledger, store): the fields are memory-mapped (nx, ny, nz)
    views on the store, deficits None where every class was well resolved.
    With ``increment_store`` (a TileStore) each class's applied increments
    are persisted into it.  The caller owns the store and must destroy() it.
    """
    from . import simulate as sim
    check_device(device, "streamed_cascade_loop")
    torch = _lib.require_cuda("streamed_cascade_loop")
    if completed:
        raise NotImplementedError("streamed_cascade_loop: resume is not offered on the device "
                                  "path (nothing is paged mid-run)")
    for name in ('padded_extent_x', 'padded_extent_y', 'padded_height'):
        values = np.asarray(grids[name])
        if not np.allclose(values, values[0]):
            raise ValueError(f"streamed_cascade_loop needs a root's grids (constant {name} "
                             f"across classes, so the regrid is a pure zoom); got a varying "
                             f"one, which means a nest's shrinking pad")
    if not isinstance(plan, TilePlan):
        raise TypeError(f"plan must be a TilePlan, got {type(plan).__name__}")
    store = TileStore(scratch_dir)
    inc_dir = None
    if increment_store is not None:
        inc_dir = increment_store.directory
    out = sim.cascade_loop(
        h_profile, qt_profile, z_profile, grids, C_h_k, C_qt_k, b_h_k, b_qt_k, aspect_k,
        h_min, h_max, qt_min, qt_max, min_distance_to_ground, sparsity_factors, class_seeds,
        n_scale_classes_per_dyad=n_scale_classes_per_dyad, flux_noise_scale=flux_noise_scale,
        turbulon_shape=turbulon_shape, zero_bottom=zero_bottom, zero_top=zero_top,
        device=device, increment_dir=inc_dir, comp_k=comp_k, dtype=dtype, resident=True)
    hp, qp, F, dh, dq, dF, final_grid, ledger = out
    final = len(grids['k']) - 1
    views = []
    for name, t in (('h_perturbation', hp), ('qt_perturbation', qp), ('flux', F),
                    ('h_deficit', dh), ('qt_deficit', dq), ('flux_deficit', dF)):
        views.append(None if t is None else write_field(store, final, name, t))
    if _crash_hook is not None:
        _crash_hook(final, 'class_done')
    del hp, qp, F, dh, dq, dF
    torch.cuda.synchronize()
    return (*views, final_grid, ledger, store)
