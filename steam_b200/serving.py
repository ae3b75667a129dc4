"""Serving world-coordinate tiles of the full class step with continuous batching.

A ``TileWorld`` is one class of a STEAM world -- the finest class (k = 200 m,
dx = dz = 100 m) of a root run over the world's shape with its seed and
parameters -- stepped once from rest (h' = qt' = 0, F = 1) over the whole
world: the flux advance, both scalar branches with the second convolution and
the bounded add, and the thermodynamic map to condensate.  What that step
realized over the whole world -- the flux restore and signed-amplitude
scale, the pattern's per-level sums, both bounded adds' per-level chains --
is its world ledger (the measure/apply split of steam/ledger.py:46-270 and of
the tiled driver steam/streaming.py:1139-1280), kept on the device.

A tile request (world origin, cube size n) is computed apply-only from a box
of the world: the tile plus a halo of 7 cells per side in x and y (the
kernel's half width 6 and one for the pattern's stencil: the kernel//2 + 1
rule of steam/streaming.py:707), and in z every level from the ground to
7 above the tile (the thermodynamic column march starts at the surface).
The box's step evaluates the world-keyed noise at world coordinates and
takes every realized scalar from the world ledger, so each field of the
tile (h', qt', F, qc, qi) equals the same cells of the world's step bit for
bit, alone or in any mix.

``TileServer`` admits requests as they arrive: a request starts when one of
its CUDA-stream slots is free and the bytes of all requests in flight stay
under a device-memory budget (by default half of the HBM free at start);
requests in flight overlap on the device.  Each tile's five fields land in a
page-locked host buffer of its slot with one copy; latency is arrival to
that copy's completion.  Every device buffer a request touches is sized and
allocated before the first request is admitted (``prepare``).
"""

from __future__ import annotations

import gc
import time
from collections import deque

import numpy as np

from . import _lib
from . import simulate as sim
from . import utils as _utils

HALO = 7   # the sparsity-1 kernel's half width (6) + the pattern stencil (1)
FIELDS = ('h', 'qt', 'flux', 'qc', 'qi')


class TileWorld:
    """One class of a world over ``shape`` (seed, alpha, C1, H, Hz), stepped
    once from rest; its world ledger stays on the device.  ``keep_fields``
    keeps the world's own step (for checking tiles against it)."""

    def __init__(self, shape, seed=7, alpha=sim.FLUX_ALPHA, c1=0.1, H=1.0 / 3.0,
                 Hz=5.0 / 9.0, dtype=np.float32, keep_fields=False):
        torch = _lib.require_cuda("TileWorld")
        from .ensemble import member_setup
        from .resident import ResidentClass
        self.lib = _lib.load()
        self.shape = tuple(int(n) for n in shape)
        self.np_t = np.dtype(dtype).type
        self.dtype = torch.float64 if self.np_t == np.float64 else torch.float32
        self.code = _lib.STEAM_F64 if self.np_t == np.float64 else _lib.STEAM_F32
        self.setup = member_setup(self.shape, seed, alpha, c1, H, Hz, self.np_t)
        self.kernel = sim._turbulon_envelope(1, 0.5, 0.5, 0.5, dtype=np.float64)
        rc = ResidentClass(self.setup, self.dtype)
        f = dict(dtype=self.dtype, device='cuda')
        h = torch.zeros(self.shape, **f)
        q = torch.zeros(self.shape, **f)
        F = torch.ones(self.shape, **f)
        diag = {k: torch.empty(self.shape, **f) for k in ("T", "qv", "qc", "qi", "p")}
        rc.step(h, q, F, diagnostics=diag)
        self.ledger = rc.class_ledger()   # raises if a persistent phase gave up
        self.block = rc.ledger.clone()    # the world ledger, device
        self.cells = rc.cells
        self.fields = ({'h': h, 'qt': q, 'flux': F, 'qc': diag['qc'], 'qi': diag['qi']}
                       if keep_fields else None)
        del rc, diag
        torch.cuda.empty_cache()

    def world_field(self, name='flux'):
        """A field of the world's own step (device; ``keep_fields`` only)."""
        if self.fields is None:
            raise RuntimeError("TileWorld: built without keep_fields")
        return self.fields[name]

    def drop_world_fields(self):
        self.fields = None

    def tile_box(self, origin, n):
        """(box origin, box shape, the tile's first level) of a tile: the
        tile plus HALO in x and y (wrapping in the world), and the levels
        from the ground to at least HALO above the tile.  The box's level
        count is a multiple of 4 exactly when the world's is: the kernels
        pick their vectorised forms by that, and the box must run the same
        arithmetic as the world to reproduce its bits; so does the parity of
        its row count."""
        x0, y0, z0 = (int(v) for v in origin)
        nx, ny, nz = self.shape
        if not (n >= 1 and 0 <= z0 and z0 + n <= nz):
            raise ValueError(f"tile z range [{z0}, {z0 + n}) outside [0, {nz})")
        bz = min(nz, z0 + n + HALO)
        if nz % 4 == 0:
            bz = min(nz, (bz + 3) // 4 * 4)
        elif bz % 4 == 0 and bz < nz:
            bz += 1
        # the box's row count has the world's parity (the packed convolution
        # takes even row counts only), one spare row past the halo if needed
        by = n + 2 * HALO
        if by % 2 != ny % 2:
            by += 1
        return ((x0 - HALO) % nx, (y0 - HALO) % ny, 0), (n + 2 * HALO, by, bz), z0

    def box_setup(self, box_shape):
        """The class set-up of a box of ``box_shape`` that starts at the
        ground: the world's per-level vectors for its levels (its origin is
        set per request)."""
        s = self.setup
        nzb = int(box_shape[2])
        return s._replace(
            shape=tuple(int(v) for v in box_shape), z=s.z[:nzb], h_mean=s.h_mean[:nzb],
            qt_mean=s.qt_mean[:nzb], C_h=s.C_h[:nzb], C_qt=s.C_qt[:nzb], b_h=s.b_h[:nzb],
            b_qt=s.b_qt[:nzb], aspect=s.aspect[:nzb],
            region=sim.NoiseRegion(s.region.key, (0, 0, 0), self.shape),
            plan=_utils.plan_convolution(self.kernel, box_shape, self.np_t),
            zero_bottom=True, zero_top=nzb == self.shape[2], window=None, deficit=None)

    def box_bytes(self, n):
        """Device bytes one request of an n-cube may hold: its box's state
        (3), work (3) and diagnostic (5) fields over full columns, and the
        tile's five fields."""
        elem = 8 if self.np_t == np.float64 else 4
        return elem * (11 * (n + 2 * HALO) * (n + 2 * HALO + 1) * self.shape[2] + 5 * n ** 3)


class _Slot:
    """A CUDA stream with buffers for the largest box and tile."""

    def __init__(self, world, max_n, torch):
        self.stream = torch.cuda.Stream()
        nb = max_n + 2 * HALO
        cap = nb * (nb + 1) * world.shape[2]
        f = dict(dtype=world.dtype, device='cuda')
        self.buf = {k: torch.empty(cap, **f)
                    for k in ('h', 'qt', 'F', 'product', 'W', 'inc', 'T', 'qv', 'qc', 'qi', 'p')}
        self.out = torch.empty(5 * max_n ** 3, **f)
        self.host = torch.empty(5 * max_n ** 3, dtype=world.dtype, pin_memory=True)
        self.event = torch.cuda.Event()
        self.request = None
        self.classes = {}  # box shape -> (ResidentClass, ReplayBlock)

    def views(self, box):
        cnt = box[0] * box[1] * box[2]
        return {k: v[:cnt].view(box) for k, v in self.buf.items()}


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
        return self.world.box_bytes(int(n))

    def check_request(self, req):
        """Refuse a request this server cannot hold, before it takes a slot."""
        n = int(req['n'])
        if not 1 <= n <= self.max_n:
            raise ValueError(f"tile size {n} outside [1, {self.max_n}] (the server's max_n)")
        self.world.tile_box(req['origin'], n)  # raises ValueError on a bad z range

    def _class_for(self, slot, box):
        hit = slot.classes.get(box)
        if hit is None:
            import torch
            from .resident import ResidentClass
            w = self.world
            with torch.cuda.stream(slot.stream):
                rc = ResidentClass(w.box_setup(box), w.dtype)
                rep = rc.replay_block(w.block, w.cells, w.shape[2])
                _lib.WORKSPACE.get(rc.workspace_bytes())  # the slot stream's scratch
            slot.stream.synchronize()
            hit = (rc, rep)
            slot.classes[box] = hit
        return hit

    def prepare(self, requests):
        """Build, on every slot, the box classes (their per-level vectors,
        convolution plans and replay blocks) the requests will need, so that
        serving allocates nothing."""
        boxes = {self.world.tile_box(r['origin'], int(r['n']))[1] for r in requests}
        for slot in self.slots:
            for box in boxes:
                self._class_for(slot, box)

    def _launch(self, slot, req):
        import torch
        w = self.world
        origin, n = req['origin'], int(req['n'])
        borig, box, z0 = w.tile_box(origin, n)
        rc, rep = self._class_for(slot, box)
        v = slot.views(box)
        cnt = box[0] * box[1] * box[2]
        lib, code = w.lib, w.code
        with torch.cuda.stream(slot.stream):
            stream = _lib.stream()
            # the world's rest state on the box
            _lib.check(lib.steam_scale(code, cnt, _lib.ptr(v['h']), 0.0, 1, stream))
            _lib.check(lib.steam_scale(code, cnt, _lib.ptr(v['qt']), 0.0, 1, stream))
            _lib.check(lib.steam_scale(code, cnt, _lib.ptr(v['F']), 1.0, 1, stream))
            rc.set_origin(borig, w.shape)
            diag = {k: v[k] for k in ("T", "qv", "qc", "qi", "p")}
            rc.step(v['h'], v['qt'], v['F'], diagnostics=diag, replay=rep,
                    work=(v['product'], v['W'], v['inc']), copy_ledger=False)
            n3 = n ** 3
            for i, key in enumerate(('h', 'qt', 'F', 'qc', 'qi')):
                _lib.check(lib.steam_tile_extract(
                    code, box[0], box[1], box[2], _lib.ptr(v[key]), HALO, HALO, z0, n, n, n,
                    1.0, 0, _lib.ptr(slot.out[i * n3:(i + 1) * n3]), stream))
            slot.host[:5 * n3].copy_(slot.out[:5 * n3], non_blocking=True)
            slot.event.record(slot.stream)
        slot.request = req

    def _fields(self, slot, n):
        n3 = n ** 3
        flat = slot.host[:5 * n3].numpy()
        return {name: flat[i * n3:(i + 1) * n3].reshape(n, n, n).copy()
                for i, name in enumerate(FIELDS)}

    def tile(self, origin, n):
        """One tile, alone (synchronous); returns {field: host array}."""
        slot = self.slots[0]
        req = {'origin': origin, 'n': int(n)}
        self.check_request(req)
        self.prepare([req])
        self._launch(slot, req)
        slot.event.synchronize()
        slot.request = None
        return self._fields(slot, int(n))

    def serve(self, requests, keep=False):
        """Serve ``requests`` (dicts with 'arrival' seconds, 'origin', 'n'),
        admitting each at its arrival time as slots and budget allow.
        Returns the requests with 'start', 'done', 'latency' (seconds) and,
        with ``keep``, 'tile' ({field: host array})."""
        for req in requests:
            self.check_request(req)
        self.prepare(requests)
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
                        req['tile'] = self._fields(slot, int(req['n']))
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
    """p50/p99 latency (arrival to host), overall and per size, and the tile
    voxels served per second; ``offered_voxels_per_s``, the tile voxels the
    arrivals asked for per second, beside it: when it exceeds the served
    rate the device is saturated and the queue sets the latency."""
    lat = np.array([r['latency'] for r in done])
    vox = sum(r['n'] ** 3 for r in done)
    span = max(r['done'] for r in done) - min(r['arrival'] for r in done)
    arrivals = sorted(r['arrival'] for r in done)
    a_span = arrivals[-1] - arrivals[0]
    offered = vox / a_span if a_span > 0 else None
    by = {}
    for n in sorted({r['n'] for r in done}):
        ln = np.array([r['latency'] for r in done if r['n'] == n])
        by[f"{n}^3"] = {"count": int(ln.size), "p50_ms": float(np.percentile(ln, 50) * 1e3),
                       "p99_ms": float(np.percentile(ln, 99) * 1e3)}
    return {"requests": len(done), "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "voxels_per_s": vox / span if span > 0 else None,
            "offered_voxels_per_s": offered, "by_size": by}
