"""Resident, asynchronous form of one size class.

``run_class`` in ``simulate`` reads every realized scalar back to the host
between stages, as the reference's stage functions do.  This module runs the
same class step (steam/simulate.py:1903-2029, plus the thermodynamic map of
steam/thermodynamics.py:25-123) with every scalar kept in device memory: the
flux restore factor, the product norm, the pattern's level means and the
bounded add's whole demean/rescale/shift solve are decided by small device
kernels between the field sweeps.  A step therefore enqueues all of its work
without waiting on the GPU; its ledger is copied back asynchronously and read
only when asked for.

``ResidentClass`` holds what a class needs on the device across steps: the
per-level vectors, the work fields (product, pattern, increment) and the
ledger block.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from . import utils as _utils
from .ledger import (BoundedAddLedger, ClassLedger, FluxAdvanceLedger, MeanReduction,
                     PatternLedger)

N_RESCALE = 10


def _off(t, n_doubles):
    """Device pointer ``n_doubles`` float64 elements into tensor ``t``."""
    return ctypes.c_void_p(t.data_ptr() + 8 * int(n_doubles))


class ResidentClass:
    """Device-resident constants, work fields and ledger block of one class.

    ``setup`` is a ``simulate.ClassSetup``; its convolution plan may be of
    any kind (separable, FFT or direct)."""

    def __init__(self, setup, dtype=None, autotune=True):
        torch = _lib.require_cuda("resident class step")
        from . import simulate as sim
        self.lib = _lib.load()
        self.setup = setup
        self.dtype = dtype if dtype is not None else torch.float32
        self.np_t = np.float64 if self.dtype == torch.float64 else np.float32
        self.code = _lib.STEAM_F64 if self.dtype == torch.float64 else _lib.STEAM_F32
        nx, ny, nz = setup.shape
        self.shape = (nx, ny, nz)
        dev = torch.device('cuda', torch.cuda.current_device())
        f64 = dict(dtype=torch.float64, device=dev)
        z = np.asarray(setup.z, dtype=np.float64)
        self.z = z
        self.vecs, self.mean, self.mul, self.pre = {}, {}, {}, {}
        for name, mean, C, b in (('h', setup.h_mean, setup.C_h, setup.b_h),
                                 ('qt', setup.qt_mean, setup.C_qt, setup.b_qt)):
            vec = torch.empty(6 * nz, dtype=self.dtype, device=dev)
            _lib.check(self.lib.steam_scalar_pattern_vectors(
                self.code, nz, _lib.dvec(mean), _lib.dvec(z), _lib.dvec(setup.aspect),
                _lib.dvec(b), _lib.ptr(vec), _lib.stream()))
            self.vecs[name] = vec
            self.mean[name] = torch.as_tensor(np.asarray(mean, np.float64), **f64).contiguous()
            self.mul[name] = torch.as_tensor(np.asarray(C, np.float32).astype(np.float64),
                                             **f64).contiguous()
            self.pre[name] = torch.empty(2 * nz, dtype=self.dtype, device=dev)
        dz = np.zeros(nz)
        dz[:-1] = np.diff(z)
        prof = np.concatenate([z, dz, np.asarray(setup.h_mean, np.float64),
                               np.asarray(setup.qt_mean, np.float64)])
        self.prof = torch.as_tensor(prof, **f64).contiguous()
        h_min, h_max, qt_min, qt_max = setup.bounds
        self.bounds = [float(self.np_t(v)) for v in (h_min, h_max, qt_min, qt_max)]
        # ledger block: noise sums [3] | conv sums [2] | flux ledger [10] |
        # pattern sums h, qt [2][nz] each | bounded-add ledger h, qt [nz][W]
        # each (W = BoundedAddLedger.record_doubles(N_RESCALE))
        W = BoundedAddLedger.record_doubles(N_RESCALE)
        self.ba_width = W
        self.o_ns, self.o_cs, self.o_fl = 0, 3, 5
        self.o_ps = {'h': 15, 'qt': 15 + 2 * nz}
        self.o_ba = {'h': 15 + 4 * nz, 'qt': 15 + 4 * nz + W * nz}
        n_led = 15 + 4 * nz + 2 * W * nz
        self.ledger = torch.zeros(n_led, **f64)
        self.ledger_host = torch.empty(n_led, dtype=torch.float64, pin_memory=True)
        self.ledger_ready = torch.cuda.Event()
        self.work = None
        self.io = None
        # flux-noise constants (steam/simulate.py:2135-2143)
        alpha = setup.alpha
        pcs = setup.flux_noise_scale / setup.n_per_dyad ** (1.0 / alpha)
        shift = sim.levy_log_mean(alpha) * pcs ** alpha
        self.alpha = alpha
        self.pcs = float(self.np_t(pcs))
        self.shift = float(self.np_t(shift))
        self.region = sim._region_struct(setup.region, self.shape, setup.sparsity)
        w = setup.window
        cols = nx * ny if w is None else (w[1] - w[0]) * (w[3] - w[2])
        self.cells = float(cols * nz)
        from . import utils as _utils
        _utils.prepare_plan(setup.plan, dev, self.dtype)
        if autotune and nx * ny * nz >= (1 << 28) and setup.plan.kind == 'separable':
            # a field this large amortises timing its convolution's tile
            # lengths once (the tile never changes a result)
            from .ensemble import autotune_conv
            autotune_conv(setup, self.dtype)

    def _work(self, like):
        import torch
        if self.work is None or self.work[0].dtype != like.dtype:
            self.work = tuple(torch.empty_like(like) for _ in range(3))
        return self.work

    def workspace_bytes(self):
        """Scratch one step takes from the stream's workspace."""
        lib, code = self.lib, self.code
        nx, ny, nz = self.shape
        return max(lib.steam_flux_noise_workspace_bytes(),
                   _utils.plan_workspace_bytes(self.setup.plan, code, self.shape),
                   lib.steam_scalar_pattern_workspace_bytes(nx, ny, nz),
                   lib.steam_bounded_add_workspace_bytes(nz, N_RESCALE),
                   lib.steam_bounded_add_replay_workspace_bytes(nz, N_RESCALE))

    def set_origin(self, origin, world_shape):
        """Place this class's box at ``origin`` of a world of ``world_shape``
        (the world-keyed noise is evaluated at world coordinates)."""
        from . import simulate as sim
        cs = self.setup
        region = sim.NoiseRegion(cs.region.key, tuple(int(v) for v in origin),
                                 tuple(int(v) for v in world_shape))
        self.region = sim._region_struct(region, self.shape, cs.sparsity)

    def replay_block(self, world_block, world_cells, world_nz):
        """This class's ledger layout filled from the ledger block of a class
        over more levels (``world_nz``; the same layout there): the flux
        sums, and the per-level pattern sums and bounded-add chains of this
        class's levels, which are the world's first nz.  For a box of the
        world that starts at its ground; the result is what ``step(...,
        replay=)`` reads."""
        import torch
        nz, W = self.shape[2], self.ba_width
        if world_nz < nz:
            raise ValueError(f"replay: the world has {world_nz} levels, this class {nz}")
        blk = torch.zeros_like(self.ledger)
        blk[:15] = world_block[:15]
        for name in ('h', 'qt'):
            w0 = 15 if name == 'h' else 15 + 2 * world_nz
            o = self.o_ps[name]
            blk[o:o + nz] = world_block[w0:w0 + nz]
            blk[o + nz:o + 2 * nz] = world_block[w0 + world_nz:w0 + world_nz + nz]
            wb = 15 + 4 * world_nz + (0 if name == 'h' else W * world_nz)
            blk[self.o_ba[name]:self.o_ba[name] + W * nz] = world_block[wb:wb + W * nz]
        return ReplayBlock(blk, float(world_cells))

    def step(self, hp, qp, F, diagnostics=None, surface_pressure=101325.0, ready=None,
             done=None, before_thermo=(), copy_ledger=True, replay=None, work=None):
        """Enqueue one class step on the resident fields (mutated in place)
        and, with ``diagnostics`` (a dict of tensors T, qv, qc, qi, p), the
        composition + thermodynamics.  Returns without waiting on the GPU.

        ``ready`` maps 'h' / 'qt' to CUDA events the step waits for before it
        first reads that field (an upload still in flight on another
        stream); ``done``, a dict, receives events recorded when F, h, qt and
        the diagnostics are final; the thermodynamics waits for the events in
        ``before_thermo`` (copies still reading the diagnostic buffers).
        ``copy_ledger=False`` leaves the ledger block on the device (a caller
        that copies it on its own stream); ``done['end']`` then marks the
        step's end.

        ``replay`` (a ``ReplayBlock``, see ``replay_block``) makes the step
        apply-only: the flux restore and the signed-amplitude scale come from
        its flux sums and cell count, the second convolution's per-level
        normalisation from its pattern sums, and each bounded add replays its
        recorded chain -- no realized scalar of this field is used, so a box
        cut from a larger field gives that field's values on every cell far
        enough from the box's sides (the kernel's support plus the pattern
        stencil).  ``work``: three field-shaped tensors (the product, the
        pattern and the increment) to use instead of this class's own."""
        import torch
        for t in (hp, qp, F):
            if tuple(t.shape) != self.shape or t.dtype != self.dtype or not t.is_contiguous():
                raise ValueError("resident class step: fields must be contiguous "
                                 f"{self.shape} {self.dtype} CUDA tensors")
        product, W, inc = self._work(F) if work is None else work
        self.enqueue_flux(F, product, replay)
        if done is not None:
            done['F'] = torch.cuda.Event()
            done['F'].record()
        # the two scalars
        for name, pert in (('h', hp), ('qt', qp)):
            if ready is not None and name in ready:
                torch.cuda.current_stream().wait_event(ready[name])
            self.enqueue_increment(name, pert, product, W, inc, replay)
            self.enqueue_bounded_add(name, pert, inc, replay)
            if done is not None:
                done[name] = torch.cuda.Event()
                done[name].record()
        if diagnostics is not None:
            for ev in before_thermo:
                torch.cuda.current_stream().wait_event(ev)
            self.enqueue_thermo(hp, qp, diagnostics, surface_pressure)
            if done is not None:
                done['diag'] = torch.cuda.Event()
                done['diag'].record()
        if copy_ledger:
            self.ledger_host.copy_(self.ledger, non_blocking=True)
            self.ledger_ready.record()
        elif done is not None:
            done['end'] = torch.cuda.Event()
            done['end'].record()
        return self

    # ---- the step's stages, each enqueued on the current stream -------------
    # (``step`` runs them in order; a batched ensemble interleaves them across
    # its members and runs the bounded adds of all members as one group)

    def _ws(self):
        ws = _lib.WORKSPACE.get(self.workspace_bytes())
        return ws, _lib.ptr(ws), ws.numel()

    def enqueue_flux(self, F, product, replay=None):
        """Flux advance: noise x F into ``product``, the flux convolution
        with its clip and window sum, the restore to the entering mean."""
        cs = self.setup
        ws, _, _ = self._ws()
        self.enqueue_noise(F, product)
        _utils.run_plan_async(cs.plan, product, F, None, _lib.STEAM_EPI_FLUX, cs.window,
                              _off(self.ledger, self.o_cs), ws, _lib.stream())
        self.enqueue_flux_finish(F, replay)

    def enqueue_noise(self, F, product):
        """The flux noise: product = eps F and the entering sums."""
        lib, cs, code = self.lib, self.setup, self.code
        ws, wsp, wsn = self._ws()
        _lib.check(lib.steam_flux_noise_async(
            code, ctypes.byref(self.region), self.alpha, self.pcs, self.shift, int(cs.n_zero),
            int(bool(cs.zero_bottom)), int(bool(cs.zero_top)), _lib.ptr(F), _lib.ptr(product),
            _lib.window_arg(cs.window), _off(self.ledger, self.o_ns), wsp, wsn, _lib.stream()))

    def enqueue_flux_finish(self, F, replay=None):
        """The restore of F to its entering mean (after the flux convolution)."""
        L = self.ledger
        src = L if replay is None else replay.block
        cells = self.cells if replay is None else replay.cells
        _lib.check(self.lib.steam_flux_finish_async(
            self.code, F.numel(), _lib.ptr(F), _off(src, self.o_ns), _off(src, self.o_cs),
            cells, _off(L, self.o_fl), _lib.stream()))

    def enqueue_increment(self, name, pert, product, W, inc, replay=None):
        """Scalar ``name``'s pattern into ``W``, its per-level normalisation
        and the second convolution into ``inc``."""
        cs = self.setup
        ws, _, _ = self._ws()
        self.enqueue_pattern(name, pert, product, W, replay)
        _utils.run_plan_async(cs.plan, W, inc, self.pre[name], _lib.STEAM_EPI_STORE,
                              cs.window, None, ws, _lib.stream())

    def enqueue_pattern(self, name, pert, product, W, replay=None):
        """Scalar ``name``'s pattern into ``W`` and its per-level
        normalisation (the second convolution's input scaling)."""
        lib, cs, code = self.lib, self.setup, self.code
        nx, ny, nz = self.shape
        stream = _lib.stream()
        L = self.ledger
        src = L if replay is None else replay.block
        ws, wsp, wsn = self._ws()
        lo, hi = self._bounds(name)
        _lib.check(lib.steam_scalar_pattern_async(
            code, nx, ny, nz, _lib.ptr(pert), _lib.ptr(self.vecs[name]), _lib.ptr(product),
            _off(L, self.o_fl + 7), float(cs.dx), float(cs.dy), _lib.dvec(self.z), 1,
            float(lo), float(hi), _lib.ptr(W), _lib.window_arg(cs.window),
            _off(L, self.o_ps[name]), wsp, wsn, stream))
        _lib.check(lib.steam_pattern_norm_async(
            code, nz, _off(src, self.o_ps[name]), _lib.ptr(self.mul[name]),
            _lib.ptr(self.pre[name]), stream))

    def conv_problem(self, src, out, pre=None, flux=False):
        """A convolution of this class as one field of a grouped launch
        (``steam_conv_problem_t``): the flux convolution (``flux``: its sums
        go to this class's ledger) or a second convolution with ``pre``."""
        nx, ny, nz = self.shape
        p = _lib.ConvProblem()
        p.nx, p.ny, p.nz = nx, ny, nz
        p.in_ = src.data_ptr()
        p.out = out.data_ptr()
        p.pre = None if pre is None else pre.data_ptr()
        w = self.setup.window
        p.has_window = 0 if w is None else 1
        if w is not None:
            p.window = _lib.Window(*[int(v) for v in w])
        p.sums = self.ledger.data_ptr() + 8 * int(self.o_cs) if flux else None
        return p

    def enqueue_bounded_add(self, name, pert, inc, replay=None):
        """Scalar ``name``'s bounded amplitude-preserving add of ``inc``
        (solved, or replayed from ``replay``'s chain)."""
        lib, cs, code = self.lib, self.setup, self.code
        nx, ny, nz = self.shape
        stream = _lib.stream()
        ws, wsp, wsn = self._ws()
        lo, hi = self._bounds(name)
        if replay is None:
            _lib.check(lib.steam_bounded_add_async(
                code, nx, ny, nz, _lib.ptr(pert), _lib.ptr(self.mean[name]), _lib.ptr(inc),
                float(lo), float(hi), _lib.window_arg(cs.window), N_RESCALE, 0,
                _off(self.ledger, self.o_ba[name]), wsp, wsn, stream))
        else:
            _lib.check(lib.steam_bounded_add_replay_async(
                code, nx, ny, nz, _lib.ptr(pert), _lib.ptr(self.mean[name]), _lib.ptr(inc),
                float(lo), float(hi), N_RESCALE, 0, _off(replay.block, self.o_ba[name]),
                wsp, wsn, stream))

    def bounded_add_problem(self, name, pert, inc):
        """Scalar ``name``'s bounded add as one field of a grouped solve
        (``steam_ba_problem_t``); its record goes to this class's ledger."""
        nx, ny, nz = self.shape
        lo, hi = self._bounds(name)
        p = _lib.BAProblem()
        p.nx, p.ny, p.nz = nx, ny, nz
        p.pert = pert.data_ptr()
        p.increment = inc.data_ptr()
        p.mean = self.mean[name].data_ptr()
        p.phi_min, p.phi_max = float(lo), float(hi)
        w = self.setup.window
        p.has_window = 0 if w is None else 1
        if w is not None:
            p.window = _lib.Window(*[int(v) for v in w])
        p.ledger = self.ledger.data_ptr() + 8 * int(self.o_ba[name])
        return p

    def enqueue_thermo(self, hp, qp, diagnostics, surface_pressure=101325.0):
        """Composition with the mean profiles, the bounds and the
        thermodynamic map into ``diagnostics`` (T, qv, qc, qi, p)."""
        nx, ny, nz = self.shape
        d = diagnostics
        _lib.check(self.lib.steam_thermo_async(
            self.code, nx, ny, nz, _lib.ptr(hp), _lib.ptr(qp), _lib.ptr(self.prof), 1,
            _lib.dvec(self.bounds), float(surface_pressure), None, _lib.ptr(d["T"]),
            _lib.ptr(d["qv"]), _lib.ptr(d["qc"]), _lib.ptr(d["qi"]), _lib.ptr(d["p"]),
            _lib.stream()))

    def _bounds(self, name):
        h_min, h_max, qt_min, qt_max = self.setup.bounds
        return (h_min, h_max) if name == 'h' else (qt_min, qt_max)

    def host_step(self, h, qt, flux, diagnostics=('qc', 'qi'), out=None,
                  surface_pressure=101325.0, wait=True):
        """One class step on host arrays, with the transfers pipelined.

        h, qt, flux (numpy, updated in place) are uploaded on one copy
        stream in the order the step needs them (F first; h and qt while the
        flux advance runs), and each result is downloaded on a second copy
        stream as soon as it is final (F while h and qt are still going up and
        the scalars run, h while qt runs, qt and the diagnostics last), so the
        two directions of the link run at the same time and both overlap
        compute.  ``out`` maps diagnostic names to host arrays to fill;
        page-locked arrays (e.g. ``torch.empty(..., pin_memory=True).numpy()``)
        let every copy run asynchronously at full PCIe bandwidth.  Returns the
        diagnostics.

        ``wait=False`` returns a ``PendingHostStep`` at once, without waiting
        for the downloads: a following call on the same arrays orders itself
        after them (each upload waits for the download of the same array, the
        thermodynamics for the previous diagnostic downloads), so the uploads
        of step k + 1 overlap the downloads of step k.  Only for host arrays
        the copies can fill directly (C-contiguous, of the step's dtype);
        others make the call wait.  The step's ledger comes with the pending
        step (``result()[1]``), not from ``class_ledger``."""
        import torch
        shape = self.shape
        for name, a in (('h', h), ('qt', qt), ('flux', flux)):
            if tuple(np.shape(a)) != shape:
                raise ValueError(f"field_step: {name} has shape {np.shape(a)}, expected {shape}")
        if self.io is None:
            self.io = {k: torch.empty(shape, dtype=self.dtype, device='cuda')
                       for k in ('h', 'qt', 'F', 'T', 'qv', 'qc', 'qi', 'p')}
            self.up_stream = torch.cuda.Stream()
            self.down_stream = torch.cuda.Stream()
            self.downloaded = None
        io, up, cp = self.io, self.up_stream, self.down_stream
        prev = self.downloaded
        main = torch.cuda.current_stream()
        src = {k: torch.from_numpy(np.ascontiguousarray(a, dtype=self.np_t))
               for k, a in (('F', flux), ('h', h), ('qt', qt))}
        up.wait_stream(main)  # the previous step's compute is done with the buffers
        ready = {}
        with torch.cuda.stream(up):
            for k in ('F', 'h', 'qt'):
                if prev is not None:
                    up.wait_event(prev[k])  # its download of this array is complete
                io[k].copy_(src[k], non_blocking=True)
                ready[k] = torch.cuda.Event()
                ready[k].record(up)
        main.wait_event(ready['F'])
        done = {}
        diag_dev = {k: io[k] for k in ('T', 'qv', 'qc', 'qi', 'p')} if diagnostics else None
        before = (prev['diag'],) if prev is not None and 'diag' in prev else ()
        # the main stream carries compute only: every device-to-host copy,
        # the ledger's included, goes on the download stream
        self.step(io['h'], io['qt'], io['F'], diagnostics=diag_dev,
                  surface_pressure=surface_pressure, ready=ready, done=done,
                  before_thermo=before, copy_ledger=False)
        ledger = torch.empty(self.ledger.numel(), dtype=torch.float64, pin_memory=True)
        if out is None:
            out = {}
        host_out = {}
        for k in (diagnostics or ()):
            if k in out:
                host_out[k] = torch.from_numpy(out[k])
            else:
                host_out[k] = torch.empty(shape, dtype=self.dtype, pin_memory=True)
        dl = {}
        with torch.cuda.stream(cp):
            for k, host in (('F', flux), ('h', h), ('qt', qt)):
                cp.wait_event(done[k])
                t = torch.from_numpy(host) if isinstance(host, np.ndarray) and \
                    host.dtype == self.np_t and host.flags.c_contiguous else None
                if t is not None:
                    t.copy_(io[k], non_blocking=True)
                else:
                    host_out['_' + k] = torch.empty(shape, dtype=self.dtype, pin_memory=True)
                    host_out['_' + k].copy_(io[k], non_blocking=True)
                dl[k] = torch.cuda.Event()
                dl[k].record(cp)
            if diagnostics:
                cp.wait_event(done['diag'])
                for k in diagnostics:
                    host_out[k].copy_(io[k], non_blocking=True)
                dl['diag'] = torch.cuda.Event()
                dl['diag'].record(cp)
            cp.wait_event(done['end'])
            ledger.copy_(self.ledger, non_blocking=True)
            ledger_ready = torch.cuda.Event()
            ledger_ready.record(cp)
        self.downloaded = dl
        pending = PendingHostStep(self, (('F', flux), ('h', h), ('qt', qt)), host_out,
                                  tuple(diagnostics or ()), ledger, ledger_ready)
        staged = any(k.startswith('_') for k in host_out)
        if wait or staged:
            return pending.result()[0] if wait else pending.wait_now()
        return pending

    def class_ledger(self, cl=None, wait=True):
        """The step's ledger as a ``ClassLedger``.  ``wait``: wait for the
        step's ledger copy first; a caller that replayed the step from a CUDA
        graph (whose event records do not reach this event) synchronises the
        device itself and passes False."""
        if wait:
            self.ledger_ready.synchronize()
        n = ctypes.c_int32(0)
        _lib.check(self.lib.steam_take_wait_errors(ctypes.byref(n)))
        if n.value:
            raise RuntimeError(f"resident class step: {n.value} convolution blocks gave up "
                               "waiting for their slab copies; the step's fields are invalid")
        return self.parse_ledger(self.ledger_host.numpy().copy(), cl)

    def parse_ledger(self, v, cl=None):
        """A ``ClassLedger`` from a host copy of the step's ledger block."""
        nz = self.shape[2]
        fl = v[self.o_fl:self.o_fl + 10]
        cl = ClassLedger() if cl is None else cl
        cl.flux = FluxAdvanceLedger(MeanReduction(fl[0], int(fl[1])),
                                    MeanReduction(fl[2], int(fl[3])),
                                    MeanReduction(fl[4], int(fl[5])), int(fl[6]))
        for name in ('h', 'qt'):
            ps = v[self.o_ps[name]:self.o_ps[name] + 2 * nz]
            cl.pattern[name] = PatternLedger(ps[:nz].copy(), ps[nz:].astype(np.int64))
            cl.bounded_add[name] = BoundedAddLedger.from_device(
                v[self.o_ba[name]:self.o_ba[name] + self.ba_width * nz], N_RESCALE)
            if cl.bounded_add[name].n_sweeps < 0:
                raise RuntimeError(f"resident class step: the {name} bounded add's "
                                   f"persistent phase timed out at a grid barrier")
        return cl


class ReplayBlock:
    """A ledger block in a ResidentClass's layout plus the cell count its
    flux sums were taken over: the realized scalars an apply-only step
    uses."""

    __slots__ = ('block', 'cells')

    def __init__(self, block, cells):
        self.block = block
        self.cells = float(cells)


class PendingHostStep:
    """A host step whose downloads may still be in flight (``host_step`` with
    ``wait=False``).  ``result()`` waits for them and returns (diagnostics,
    ClassLedger) of this step."""

    def __init__(self, rc, fields, host_out, names, ledger, ledger_ready):
        self._rc = rc
        self._fields = fields
        self._host_out = host_out
        self._names = names
        self._ledger = ledger
        self._ledger_ready = ledger_ready
        self._done = None

    def _finish(self):
        if self._done is None:
            self._rc.down_stream.synchronize()
            self._rc.up_stream.synchronize()
            for k, host in self._fields:
                if '_' + k in self._host_out:
                    host[...] = self._host_out['_' + k].numpy()
            diag = {k: self._host_out[k].numpy() for k in self._names}
            self._ledger_ready.synchronize()
            self._done = (diag, self._rc.parse_ledger(self._ledger.numpy().copy()))
        return self._done

    def wait_now(self):
        """Finish now (the call that staged a host array needs its results
        written back before anything else reads them) and return self."""
        self._finish()
        return self

    def result(self):
        return self._finish()


_CACHE = {}


def resident_for(setup, dtype):
    """The cached ResidentClass of ``setup`` on the current device."""
    import torch
    key = (id(setup), dtype, torch.cuda.current_device())
    hit = _CACHE.get(key)
    if hit is not None and hit.setup is setup:
        return hit
    if len(_CACHE) > 64:
        _CACHE.clear()
    rc = ResidentClass(setup, dtype)
    _CACHE[key] = rc
    return rc
