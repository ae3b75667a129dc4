"""Serving world-coordinate tiles of the flux field with continuous batching.

A ``TileWorld`` is one class of a STEAM world: its grid, its Philox key, its
turbulon kernel and its world ledger -- the flux advance's realized restore
factor, measured once over the whole world (the measure/apply split of
steam/ledger.py:115-142 and of the tiled driver steam/streaming.py:850-1447,
where per-class scalars are realized over the domain and applied per tile).
A tile request (world origin, cube size n) is computed from its own box: the
tile plus the kernel's halo of 6 cells per side (12 s + 1 = 13 taps at
sparsity 1; steam/streaming.py:707 uses the same 6 s + 1 halo), with the
world-keyed noise evaluated at world coordinates, so a tile equals the same
cells of the whole-world field bit for bit, alone or in any mix.

``TileServer`` admits requests as they arrive: a request starts when one of
its CUDA streams is free and the bytes of all requests in flight stay under a
device-memory budget (by default half of the HBM free at start); requests in
flight overlap on the device.  Each tile is downloaded into a page-locked
host buffer of its slot; latency is arrival to download complete.
"""

from __future__ import annotations

import ctypes
import gc
import time
from collections import deque

import numpy as np

from . import _lib
from . import simulate as sim
from . import utils as _utils

HALO = 6  # (13 - 1) / 2: the sparsity-1 turbulon kernel's half width


class TileWorld:
    """One class of a world: the finest class of a root run over
    ``shape`` (dx = dz = 100 m, turbulon size k = 200 m) with seed ``seed``."""

    def __init__(self, shape, seed=7, alpha=sim.FLUX_ALPHA, c1=0.1, n_per_dyad=1,
                 dtype=np.float32, min_distance_to_ground=1):
        torch = _lib.require_cuda("TileWorld")
        self.lib = _lib.load()
        self.shape = tuple(int(n) for n in shape)
        nx, ny, nz = self.shape
        self.np_t = np.dtype(dtype).type
        self.dtype = torch.float64 if self.np_t == np.float64 else torch.float32
        self.code = _lib.dtype_code(torch.empty(0, dtype=self.dtype))
        outer = nx * 100.0
        n_classes = int(round(np.log(outer / 200.0) / np.log(2.0))) + 1
        self.key = sim.class_key(np.random.SeedSequence(seed).spawn(n_classes)[-1])
        self.kernel = sim._turbulon_envelope(1, 0.5, 0.5, 0.5, dtype=np.float64)
        self.alpha = float(alpha)
        pcs = c1 / n_per_dyad ** (1.0 / alpha)
        self.pcs = float(self.np_t(pcs))
        self.shift = float(self.np_t(sim.levy_log_mean(alpha) * pcs ** alpha))
        self.n_zero = int(round(2 * min_distance_to_ground))
        self.factor, self.fill = self._world_ledger()

    def region(self, origin, box):
        r = _lib.Region()
        for a in range(3):
            r.shape[a] = int(box[a])
            r.origin[a] = int(origin[a])
            r.world[a] = int(self.shape[a])
            r.sparsity[a] = 1
            r.key[a] = int(self.key[a]) & 0xFFFFFFFF
        return r

    def advance(self, F, product, origin, box, sums, zero_bottom, zero_top, ws, stream):
        """F = max(F + T * (eps F), 0) on a box at a world origin (enqueued)."""
        lib = self.lib
        nx, ny, nz = box
        region = self.region(origin, box)
        _lib.check(lib.steam_flux_noise_async(
            self.code, ctypes.byref(region), self.alpha, self.pcs, self.shift, self.n_zero,
            int(zero_bottom), int(zero_top), _lib.ptr(F), _lib.ptr(product), None,
            _lib.ptr(sums), _lib.ptr(ws), ws.numel(), stream))
        plan = _utils.plan_convolution(self.kernel, box, self.np_t)
        _utils.run_plan_async(plan, product, F, None, _lib.STEAM_EPI_FLUX, None,
                              ctypes.c_void_p(sums.data_ptr() + 24), ws, stream)

    def workspace_bytes(self, box):
        lib = self.lib
        plan = _utils.plan_convolution(self.kernel, box, self.np_t)
        return max(lib.steam_flux_noise_workspace_bytes(),
                   _utils.plan_workspace_bytes(plan, self.code, box))

    def _world_ledger(self):
        """The restore factor realized over the whole world (one advance)."""
        torch = _lib.require_cuda("TileWorld")
        F = torch.ones(self.shape, dtype=self.dtype, device='cuda')
        product = torch.empty_like(F)
        sums = torch.zeros(8, dtype=torch.float64, device='cuda')
        ledger = torch.zeros(10, dtype=torch.float64, device='cuda')
        ws = torch.empty(self.workspace_bytes(self.shape), dtype=torch.uint8, device='cuda')
        stream = _lib.stream()
        self.advance(F, product, (0, 0, 0), self.shape, sums, True, True, ws, stream)
        cells = float(F.numel())
        _lib.check(self.lib.steam_flux_finish_async(
            self.code, F.numel(), _lib.ptr(F), _lib.ptr(sums),
            ctypes.c_void_p(sums.data_ptr() + 24), cells, _lib.ptr(ledger), stream))
        led = ledger.cpu().numpy()
        self.world_ledger = led
        self._world_F = F  # kept only while the caller asks for it (world_field)
        return float(led[8]), int(led[9])

    def world_field(self):
        """The whole-world advanced flux of the ledger measurement (device)."""
        return self._world_F

    def drop_world_field(self):
        self._world_F = None

    def box_depth(self, n):
        """Most levels a tile box of an n-cube spans (halo, plus the zeroed
        bottom/top bands pulled in whole)."""
        return min(self.shape[2], n + 2 * HALO + 2 * self.n_zero)

    def tile_box(self, origin, n):
        """(box origin, box shape, z offset of the tile in the box, zero flags)."""
        x0, y0, z0 = (int(v) for v in origin)
        nz = self.shape[2]
        if not (0 <= z0 and z0 + n <= nz):
            raise ValueError(f"tile z range [{z0}, {z0 + n}) outside [0, {nz})")
        bz0 = max(0, z0 - HALO)
        if bz0 < self.n_zero:  # the zeroed bottom levels sit at the box bottom
            bz0 = 0
        bz1 = min(nz, z0 + n + HALO)
        if bz1 > nz - self.n_zero:
            bz1 = nz
        return ((x0 - HALO) % self.shape[0], (y0 - HALO) % self.shape[1], bz0), \
            (n + 2 * HALO, n + 2 * HALO, bz1 - bz0), z0 - bz0, bz0 == 0, bz1 == nz


class _Slot:
    def __init__(self, world, max_n, torch):
        self.stream = torch.cuda.Stream()
        nbox = max_n + 2 * HALO
        zbox = world.box_depth(max_n)
        cap = nbox * nbox * zbox
        self.F = torch.empty(cap, dtype=world.dtype, device='cuda')
        self.product = torch.empty(cap, dtype=world.dtype, device='cuda')
        self.sums = torch.zeros(8, dtype=torch.float64, device='cuda')
        ws = max(world.workspace_bytes((nbox, nbox, zbox)), 1)
        self.ws = torch.empty(ws, dtype=torch.uint8, device='cuda')
        # the tile's cells, contiguous, then page-locked: both sized once here so
        # serving allocates nothing (a first allocation on a stream blocks the
        # host loop for tens of ms)
        self.out = torch.empty(max_n ** 3, dtype=world.dtype, device='cuda')
        self.host = torch.empty(max_n ** 3, dtype=world.dtype, pin_memory=True)
        self.event = torch.cuda.Event()
        self.request = None


class TileServer:
    """Continuous-batching tile server over ``n_slots`` CUDA streams."""

    def __init__(self, world, n_slots=4, max_n=256, budget_bytes=None):
        torch = _lib.require_cuda("TileServer")
        self.world = world
        self.max_n = int(max_n)
        self.slots = [_Slot(world, self.max_n, torch) for _ in range(n_slots)]
        if budget_bytes is None:
            free, _ = torch.cuda.mem_get_info()
            budget_bytes = free // 2
        self.budget = int(budget_bytes)
        self.in_flight_bytes = 0

    def request_bytes(self, n):
        nbox = n + 2 * HALO
        elem = 8 if self.world.np_t == np.float64 else 4
        return 2 * elem * nbox * nbox * self.world.box_depth(n) + elem * n ** 3

    def _launch(self, slot, req):
        import torch
        w = self.world
        origin, n = req['origin'], req['n']
        borig, box, zoff, zb, zt = w.tile_box(origin, n)
        cnt = box[0] * box[1] * box[2]
        F = slot.F[:cnt].view(box)
        product = slot.product[:cnt].view(box)
        with torch.cuda.stream(slot.stream):
            stream = _lib.stream()
            _lib.check(w.lib.steam_scale(w.code, cnt, _lib.ptr(F), 1.0, 1, stream))
            w.advance(F, product, borig, box, slot.sums, zb, zt, slot.ws, stream)
            # the world restore on the tile's cells only, into the contiguous buffer
            out = slot.out[:n ** 3]
            _lib.check(w.lib.steam_tile_extract(
                w.code, box[0], box[1], box[2], _lib.ptr(F), HALO, HALO, zoff, n, n, n,
                w.factor, w.fill, _lib.ptr(out), stream))
            slot.host[:n ** 3].copy_(out, non_blocking=True)
            slot.event.record(slot.stream)
        slot.request = req

    def check_request(self, req):
        """Refuse a request this server cannot hold, before it takes a slot."""
        n = int(req['n'])
        if not 1 <= n <= self.max_n:
            raise ValueError(f"tile size {n} outside [1, {self.max_n}] (the server's max_n)")
        self.world.tile_box(req['origin'], n)  # raises ValueError on a bad z range

    def tile(self, origin, n):
        """One tile, alone (synchronous); returns a host array."""
        slot = self.slots[0]
        req = {'origin': origin, 'n': int(n)}
        self.check_request(req)
        self._launch(slot, req)
        slot.event.synchronize()
        slot.request = None
        return slot.host[:n ** 3].view(n, n, n).numpy().copy()

    def serve(self, requests, keep=False):
        """Serve ``requests`` (dicts with 'arrival' seconds, 'origin', 'n'),
        admitting each at its arrival time as slots and budget allow.
        Returns the requests with 'start', 'done', 'latency' (seconds) and,
        with ``keep``, 'tile' (host array)."""
        # the host loop is the server's critical path: no collection pauses
        # while requests are in flight
        gc_was = gc.isenabled()
        gc.disable()
        try:
            return self._serve(requests, keep)
        finally:
            if gc_was:
                gc.enable()

    def _serve(self, requests, keep):
        for req in requests:
            self.check_request(req)
        pending = deque(sorted(requests, key=lambda r: r['arrival']))
        free = list(self.slots)
        busy = []
        t0 = time.perf_counter()
        out = []
        while pending or busy:
            now = time.perf_counter() - t0
            progressed = False
            while pending and pending[0]['arrival'] <= now and free:
                req = pending[0]
                need = self.request_bytes(req['n'])
                if busy and self.in_flight_bytes + need > self.budget:
                    break  # wait for memory to free up
                pending.popleft()
                slot = free.pop()
                req['start'] = now
                req['bytes'] = need
                try:
                    self._launch(slot, req)
                except BaseException:
                    free.append(slot)
                    raise
                self.in_flight_bytes += need
                busy.append(slot)
                progressed = True
            for slot in list(busy):
                if slot.event.query():
                    req = slot.request
                    req['done'] = time.perf_counter() - t0
                    req['latency'] = req['done'] - req['arrival']
                    if keep:
                        n = req['n']
                        req['tile'] = slot.host[:n ** 3].view(n, n, n).numpy().copy()
                    self.in_flight_bytes -= req['bytes']
                    slot.request = None
                    busy.remove(slot)
                    free.append(slot)
                    out.append(req)
                    progressed = True
            if not progressed and not busy and pending:
                # idle until the next arrival: sleep only when it is more than
                # 2 ms away (a sleep can overshoot on a loaded host); with
                # tiles in flight the loop polls without sleeping
                wait = pending[0]['arrival'] - now
                if wait > 2e-3:
                    time.sleep(wait - 1e-3)
        return out


def poisson_trace(world, rate, n_requests, seed=4, sizes=(32, 64, 128, 256),
                  weights=(0.4, 0.3, 0.2, 0.1), adjacent=True):
    """Poisson arrivals of cube tiles on the world lattice.  With ``adjacent``
    origins sit on a grid of the cube size, so neighbouring requests share
    halo cells."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n_requests))
    nx, ny, nz = world.shape
    reqs = []
    for i in range(n_requests):
        n = int(rng.choice(sizes, p=np.asarray(weights) / np.sum(weights)))
        n = min(n, nz)
        if adjacent:
            ox = int(rng.integers(0, max(1, nx // n))) * n
            oy = int(rng.integers(0, max(1, ny // n))) * n
            oz = int(rng.integers(0, max(1, nz // n))) * n
        else:
            ox, oy = int(rng.integers(0, nx)), int(rng.integers(0, ny))
            oz = int(rng.integers(0, nz - n + 1))
        reqs.append({'arrival': float(t[i]), 'origin': (ox, oy, min(oz, nz - n)), 'n': n})
    return reqs


def latency_summary(done):
    lat = np.array([r['latency'] for r in done])
    vox = sum(r['n'] ** 3 for r in done)
    span = max(r['done'] for r in done) - min(r['arrival'] for r in done)
    by = {}
    for n in sorted({r['n'] for r in done}):
        ln = np.array([r['latency'] for r in done if r['n'] == n])
        by[f"{n}^3"] = {"count": int(ln.size), "p50_ms": float(np.percentile(ln, 50) * 1e3),
                       "p99_ms": float(np.percentile(ln, 99) * 1e3)}
    return {"requests": len(done), "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "voxels_per_s": vox / span if span > 0 else None, "by_size": by}
