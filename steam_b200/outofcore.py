"""Out-of-core class step: a class whose fields live in host memory.

The tiled driver of steam/streaming.py:850-1447 -- measure, reduce, apply --
for one size class on the device, with the class's state (h', qt', F) in
(page-locked) host arrays and only tiles of it on the device at a time.  A
tile is a block of columns over every level, plus a halo of HALO = 7
columns per side (the kernel's half width and the pattern stencil's one:
steam/streaming.py:707), wrapping in x and y.  Each pass streams the tiles
through two device buffer sets on three CUDA streams -- uploads, compute,
downloads -- so tile k + 1 goes up while tile k computes and tile k - 1
comes down (steam/utils.py:377-405 streams its FFT blocks to the host the
same way):

1. flux measure: noise, multiplier product and flux convolution on each
   box; the new flux of the tile's own columns goes to the host, and the
   tile's sums (entering, |noise|, realized, clip count, over its own
   columns) to a per-tile record;
2. the records reduce in tile order on the host into the flux ledger; each
   tile's new flux is restored on the device with it (the resident step's
   restore kernel), and the pattern's per-level sums of both scalars are
   measured per tile;
3. the per-level sums reduce into the pattern ledger; the second
   convolution of each scalar runs per box with that normalisation and the
   increment of the tile's columns goes to the host;
4. the bounded add solves per slab of levels over every column of them
   (its statistics are per level, so a slab of levels is a complete
   problem), reading the perturbation and increment slabs from the host and
   writing the perturbation back;
5. thermodynamics per tile of columns (no halo: a column is independent).

Every realized scalar is measured over the whole class, so the result is
the resident step's up to the order of the double-precision sums (tile
records reduce in tile order, the device's block partials in theirs).
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from . import simulate as sim
from . import utils as _utils
from .ledger import (BoundedAddLedger, ClassLedger, FluxAdvanceLedger, MeanReduction,
                     PatternLedger)

HALO = 7


def _tiles(n, t):
    return [(a, min(t, n - a)) for a in range(0, n, t)]


class _Pipe:
    """Three streams and two buffer sets: uploads of tile k + 1 overlap the
    compute of tile k and the downloads of tile k - 1."""

    def __init__(self, torch):
        self.torch = torch
        self.up = torch.cuda.Stream()
        self.comp = torch.cuda.Stream()
        self.down = torch.cuda.Stream()
        self.freed = [None, None]  # download finished with buffer set s

    def run(self, items, upload, compute, download):
        torch = self.torch
        main = torch.cuda.current_stream()
        for s in (self.up, self.comp, self.down):
            s.wait_stream(main)
        for k, item in enumerate(items):
            b = k & 1
            with torch.cuda.stream(self.up):
                if self.freed[b] is not None:
                    self.up.wait_event(self.freed[b])
                upload(b, item)
                ev_up = torch.cuda.Event()
                ev_up.record(self.up)
            with torch.cuda.stream(self.comp):
                self.comp.wait_event(ev_up)
                compute(b, item)
                ev_c = torch.cuda.Event()
                ev_c.record(self.comp)
            with torch.cuda.stream(self.down):
                self.down.wait_event(ev_c)
                download(b, item)
                ev_d = torch.cuda.Event()
                ev_d.record(self.down)
                self.freed[b] = ev_d
        for s in (self.up, self.comp, self.down):
            main.wait_stream(s)
        self.freed = [None, None]


def host_scratch(shape, dtype):
    """The page-locked host arrays a streamed class step of ``shape`` works
    in (the new flux and both increments), for reuse across calls."""
    import torch
    tdt = torch.float64 if np.dtype(dtype) == np.float64 else torch.float32
    return {k: torch.empty(tuple(shape), dtype=tdt, pin_memory=True).numpy()
            for k in ('F_new', 'h', 'qt')}


def streamed_class_step(h, qt, flux, setup, tile=(256, 256), slab_levels=32,
                        diagnostics=('qc', 'qi'), out=None, surface_pressure=101325.0,
                        scratch=None):
    """One class step (flux advance, both scalar branches, thermodynamics) on
    HOST arrays h', qt', F of ``setup.shape`` (updated in place), with at
    most a tile of columns plus its halo, or a slab of levels, on the device
    at a time.  Page-locked arrays let every copy run asynchronously;
    ``scratch`` (see ``host_scratch``) holds the step's own host arrays,
    allocated page-locked per call otherwise.  Returns ({diagnostic: host
    array}, ClassLedger)."""
    torch = _lib.require_cuda("streamed_class_step")
    from .resident import N_RESCALE, ResidentClass
    lib = _lib.load()
    cs = setup
    nx, ny, nz = (int(n) for n in cs.shape)
    for name, a in (('h', h), ('qt', qt), ('flux', flux)):
        if tuple(np.shape(a)) != (nx, ny, nz) or not isinstance(a, np.ndarray) \
                or not a.flags.c_contiguous:
            raise ValueError(f"streamed_class_step: {name} must be a C-contiguous "
                             f"{(nx, ny, nz)} numpy array")
    if cs.window is not None or cs.deficit is not None:
        raise NotImplementedError("streamed_class_step: windows and compensation deficits "
                                  "run resident")
    np_t = h.dtype.type
    if qt.dtype != h.dtype or flux.dtype != h.dtype or np_t not in (np.float32, np.float64):
        raise ValueError("streamed_class_step: h, qt, flux must share a float dtype")
    tdt = torch.float64 if np_t == np.float64 else torch.float32
    code = _lib.STEAM_F64 if np_t == np.float64 else _lib.STEAM_F32
    elem = np.dtype(np_t).itemsize
    dev = torch.device('cuda', torch.cuda.current_device())
    f64 = dict(dtype=torch.float64, device=dev)
    # per-level device vectors of the class (the resident step's own)
    rc = ResidentClass(cs, tdt, autotune=False)
    tx, ty = min(int(tile[0]), nx), min(int(tile[1]), ny)
    # an axis one tile covers needs no halo (the box is the whole period);
    # otherwise the tile plus both halos must fit in the period
    hx = 0 if tx >= nx else HALO
    hy = 0 if ty >= ny else HALO
    if tx + 2 * hx > nx or ty + 2 * hy > ny:
        raise ValueError(f"streamed_class_step: tile {tx} x {ty} plus its halo of {HALO} "
                         f"does not fit the period {nx} x {ny}; use a larger tile")
    xt, yt = _tiles(nx, tx), _tiles(ny, ty)
    items = [(x0, bx, y0, by) for (x0, bx) in xt for (y0, by) in yt]
    index = {item: k for k, item in enumerate(items)}
    bxm, bym = tx + 2 * hx, ty + 2 * hy
    cap = bxm * bym * nz
    bufs = [{k: torch.empty(cap, dtype=tdt, device=dev)
             for k in ('F', 'h', 'qt', 'P', 'W', 'I')} for _ in range(2)]
    sums = [torch.zeros(8 + 4 * nz, **f64) for _ in range(2)]
    ntile = len(items)
    rec = torch.zeros((ntile, 8 + 4 * nz), dtype=torch.float64, pin_memory=True)
    pipe = _Pipe(torch)
    lo_hi = {'h': cs.bounds[0:2], 'qt': cs.bounds[2:4]}
    host = {'F': flux, 'h': h, 'qt': qt}
    plans = {}

    def box(item):
        x0, bx, y0, by = item
        return (bx + 2 * hx, by + 2 * hy, nz), ((x0 - hx) % nx, (y0 - hy) % ny)

    def view(b, key, shape):
        return bufs[b][key][:shape[0] * shape[1] * shape[2]].view(shape)

    def plan(shape):
        p = plans.get(shape)
        if p is None:
            p = _utils.plan_convolution(cs.plan.kernel, shape, np_t)
            _utils.prepare_plan(p, dev, tdt)
            plans[shape] = p
        return p

    def upload_box(b, item, keys):
        shape, (ox, oy) = box(item)
        for k in keys:
            _lib.check(lib.steam_box_h2d(elem, host[k].ctypes.data, nx, ny, nz, ox, oy, 0,
                                         shape[0], shape[1], nz, _lib.ptr(view(b, k, shape)),
                                         _lib.stream()))

    def region(item):
        shape, (ox, oy) = box(item)
        return sim._region_struct(sim.NoiseRegion(cs.region.key, (ox, oy, 0), (nx, ny, nz)),
                                  shape, cs.sparsity)

    def window(item):
        x0, bx, y0, by = item
        return (hx, hx + bx, hy, hy + by)

    def noise(b, item, sums_ptr):
        shape, _ = box(item)
        r = region(item)
        ws = _lib.WORKSPACE.get(lib.steam_flux_noise_workspace_bytes())
        _lib.check(lib.steam_flux_noise_async(
            code, ctypes.byref(r), rc.alpha, rc.pcs, rc.shift, int(cs.n_zero),
            int(bool(cs.zero_bottom)), int(bool(cs.zero_top)), _lib.ptr(view(b, 'F', shape)),
            _lib.ptr(view(b, 'P', shape)), _lib.window_arg(window(item)), sums_ptr,
            _lib.ptr(ws), ws.numel(), _lib.stream()))

    def off(t, n):
        return ctypes.c_void_p(t.data_ptr() + 8 * int(n))

    # ---- pass 1: flux measure ------------------------------------------------
    if scratch is None:
        scratch = host_scratch((nx, ny, nz), np_t)
    F_new = scratch['F_new']

    def p1_up(b, item):
        upload_box(b, item, ('F',))

    def p1_comp(b, item):
        shape, _ = box(item)
        noise(b, item, off(sums[b], 0))
        # the convolution stored, then the flux epilogue with the clip
        # counted over the tile's own columns
        _utils.run_plan_async(plan(shape), view(b, 'P', shape), view(b, 'W', shape), None,
                              _lib.STEAM_EPI_STORE_WIDE, None, None)
        ws = _lib.WORKSPACE.get(lib.steam_flux_clip_workspace_bytes(*shape))
        _lib.check(lib.steam_flux_clip_async(code, *shape, _lib.ptr(view(b, 'F', shape)),
                                             _lib.ptr(view(b, 'W', shape)),
                                             _lib.window_arg(window(item)), off(sums[b], 3),
                                             _lib.ptr(ws), ws.numel(), _lib.stream()))

    def p1_down(b, item):
        shape, _ = box(item)
        x0, bx, y0, by = item
        k = index[item]
        rec[k, :5].copy_(sums[b][:5], non_blocking=True)
        _lib.check(lib.steam_box_d2h(elem, _lib.ptr(view(b, 'F', shape)), *shape, hx, hy, 0,
                                     bx, by, nz, F_new.ctypes.data, nx, ny, nz, x0, y0, 0,
                                     _lib.stream()))

    pipe.run(items, p1_up, p1_comp, p1_down)
    torch.cuda.synchronize()
    r = rec.numpy()
    ns_g = torch.tensor([r[:, 0].sum(), r[:, 1].sum(), r[:, 2].sum()], **f64)
    cs_g = torch.tensor([r[:, 3].sum(), r[:, 4].sum()], **f64)
    cells = float(nx * ny * nz)
    # the flux ledger as the resident step's restore kernel writes it: entry 7
    # is the signed amplitude's scale 1/mean|eps| rounded to the dtype
    ns_h, cs_h = ns_g.cpu().numpy(), cs_g.cpu().numpy()
    mean_abs = ns_h[1] / (ns_h[2] if ns_h[2] > 1.0 else 1.0)
    s_scale = float(np_t(1.0 / mean_abs)) if mean_abs > 0.0 else 1.0
    fl = torch.tensor([ns_h[0], cells, ns_h[1], ns_h[2], cs_h[0], cells, cs_h[1], s_scale,
                       0.0, 0.0], **f64)

    # ---- pass 2: measure both patterns (the entering flux makes the product) ----
    def p2_up(b, item):
        upload_box(b, item, ('F', 'h', 'qt'))

    def pattern(b, item, name, level_sums_ptr, win):
        shape, _ = box(item)
        lo, hi = lo_hi[name]
        ws = _lib.WORKSPACE.get(lib.steam_scalar_pattern_workspace_bytes(*shape))
        _lib.check(lib.steam_scalar_pattern_async(
            code, *shape, _lib.ptr(view(b, name, shape)), _lib.ptr(rc.vecs[name]),
            _lib.ptr(view(b, 'P', shape)), off(fl, 7), float(cs.dx), float(cs.dy),
            _lib.dvec(rc.z), 1, float(lo), float(hi), _lib.ptr(view(b, 'W', shape)),
            _lib.window_arg(win), level_sums_ptr, _lib.ptr(ws), ws.numel(), _lib.stream()))

    def p2_comp(b, item):
        noise(b, item, off(sums[b], 0))
        pattern(b, item, 'h', off(sums[b], 8), window(item))
        pattern(b, item, 'qt', off(sums[b], 8 + 2 * nz), window(item))

    def p2_down(b, item):
        k = index[item]
        rec[k, 8:].copy_(sums[b][8:], non_blocking=True)

    pipe.run(items, p2_up, p2_comp, p2_down)
    torch.cuda.synchronize()
    r = rec.numpy()
    ps_h = r[:, 8:8 + 2 * nz].sum(axis=0)
    ps_q = r[:, 8 + 2 * nz:8 + 4 * nz].sum(axis=0)
    ps_dev = {'h': torch.as_tensor(ps_h, **f64).contiguous(),
              'qt': torch.as_tensor(ps_q, **f64).contiguous()}
    cl = ClassLedger()
    flv = fl.cpu().numpy()
    cl.flux = FluxAdvanceLedger(MeanReduction(flv[0], int(flv[1])),
                                MeanReduction(flv[2], int(flv[3])),
                                MeanReduction(flv[4], int(flv[5])), int(flv[6]))
    cl.pattern['h'] = PatternLedger(ps_h[:nz].copy(), ps_h[nz:].astype(np.int64))
    cl.pattern['qt'] = PatternLedger(ps_q[:nz].copy(), ps_q[nz:].astype(np.int64))

    # ---- pass 3: second convolutions ------------------------------------------
    inc = {'h': scratch['h'], 'qt': scratch['qt']}
    for name in ('h', 'qt'):
        def p3_up(b, item, name=name):
            upload_box(b, item, ('F', name))

        def p3_comp(b, item, name=name):
            shape, _ = box(item)
            noise(b, item, off(sums[b], 0))
            pattern(b, item, name, off(sums[b], 8), None)
            _lib.check(lib.steam_pattern_norm_async(code, nz, _lib.ptr(ps_dev[name]),
                                                    _lib.ptr(rc.mul[name]),
                                                    _lib.ptr(rc.pre[name]), _lib.stream()))
            _utils.run_plan_async(plan(shape), view(b, 'W', shape), view(b, 'I', shape),
                                  rc.pre[name], _lib.STEAM_EPI_STORE, None, None)

        def p3_down(b, item, name=name):
            shape, _ = box(item)
            x0, bx, y0, by = item
            _lib.check(lib.steam_box_d2h(elem, _lib.ptr(view(b, 'I', shape)), *shape, hx,
                                         hy, 0, bx, by, nz, inc[name].ctypes.data, nx, ny,
                                         nz, x0, y0, 0, _lib.stream()))

        pipe.run(items, p3_up, p3_comp, p3_down)
    torch.cuda.synchronize()
    bufs = None

    # ---- pass 4: bounded adds on slabs of whole levels -------------------------
    dz = max(1, min(int(slab_levels), nz))
    slab = [{k: torch.empty(nx * ny * dz, dtype=tdt, device=dev) for k in ('p', 'd')}
            for _ in range(2)]
    W = BoundedAddLedger.record_doubles(N_RESCALE)
    for name, mean in (('h', cs.h_mean), ('qt', cs.qt_mean)):
        lo, hi = lo_hi[name]
        led = np.zeros((nz, W))
        slabs = [(z0, min(dz, nz - z0)) for z0 in range(0, nz, dz)]
        for k, (z0, n) in enumerate(slabs):
            b = k & 1
            pv = slab[b]['p'][:nx * ny * n].view(nx, ny, n)
            dv = slab[b]['d'][:nx * ny * n].view(nx, ny, n)
            s = _lib.stream()
            _lib.check(lib.steam_box_h2d(elem, host[name].ctypes.data, nx, ny, nz, 0, 0, z0, nx,
                                         ny, n, _lib.ptr(pv), s))
            _lib.check(lib.steam_box_h2d(elem, inc[name].ctypes.data, nx, ny, nz, 0, 0, z0, nx,
                                         ny, n, _lib.ptr(dv), s))
            out_led = sim.bounded_add_device(pv, np.asarray(mean)[z0:z0 + n], dv, lo, hi,
                                             n_rescale=N_RESCALE)
            led[z0:z0 + n] = out_led.to_device()
            _lib.check(lib.steam_box_d2h(elem, _lib.ptr(pv), nx, ny, n, 0, 0, 0, nx, ny, n,
                                         host[name].ctypes.data, nx, ny, nz, 0, 0, z0, s))
        torch.cuda.current_stream().synchronize()
        cl.bounded_add[name] = BoundedAddLedger.from_device(led, N_RESCALE)
    slab = inc = None

    # ---- pass 5: the flux restore and thermodynamics per tile of columns ---------
    names = tuple(diagnostics or ())
    out = {} if out is None else out
    for k in names:
        if k not in out:
            out[k] = np.empty_like(h)
    tb = [{k: torch.empty(tx * ty * nz, dtype=tdt, device=dev)
           for k in ('F', 'h', 'qt', 'T', 'qv', 'qc', 'qi', 'p')} for _ in range(2)]

    def tv(b, k, item):
        _, bx, _, by = item
        return tb[b][k][:bx * by * nz].view(bx, by, nz)

    def p5_up(b, item):
        x0, bx, y0, by = item
        for k, src in (('F', F_new), ('h', h), ('qt', qt)):
            if k != 'F' and not names:
                continue
            _lib.check(lib.steam_box_h2d(elem, src.ctypes.data, nx, ny, nz, x0, y0, 0, bx, by,
                                         nz, _lib.ptr(tv(b, k, item)), _lib.stream()))

    def p5_comp(b, item):
        x0, bx, y0, by = item
        # the resident step's restore kernel with the class's sums
        _lib.check(lib.steam_flux_finish_async(code, bx * by * nz, _lib.ptr(tv(b, 'F', item)),
                                               _lib.ptr(ns_g), _lib.ptr(cs_g), cells, None,
                                               _lib.stream()))
        if names:
            _lib.check(lib.steam_thermo_async(
                code, bx, by, nz, _lib.ptr(tv(b, 'h', item)), _lib.ptr(tv(b, 'qt', item)),
                _lib.ptr(rc.prof), 1, _lib.dvec(rc.bounds), float(surface_pressure), None,
                *(_lib.ptr(tv(b, k, item)) for k in ('T', 'qv', 'qc', 'qi', 'p')),
                _lib.stream()))

    def p5_down(b, item):
        x0, bx, y0, by = item
        for k, dst in (('F', flux),) + tuple((k, out[k]) for k in names):
            _lib.check(lib.steam_box_d2h(elem, _lib.ptr(tv(b, k, item)), bx, by, nz, 0, 0, 0,
                                         bx, by, nz, dst.ctypes.data, nx, ny, nz, x0, y0, 0,
                                         _lib.stream()))

    pipe.run(items, p5_up, p5_comp, p5_down)
    torch.cuda.synchronize()
    return {k: out[k] for k in names}, cl
