"""Batched ensembles: many independent members in one captured launch graph.

A member is one class step of its own world (its shape, seed, alpha, C1, H,
Hz): the finest class of a root run over the member's domain, run by a
``ResidentClass`` on device fields.  ``Ensemble`` spreads the members over a
few CUDA streams and captures one step of all of them into a single CUDA
graph: a replay then issues the whole step with one launch call.  The step
runs stage by stage: every member's flux noise (spread over the streams),
ONE grouped flux convolution over all members (``steam_conv_group_async``:
every member its own block range of one packed-kernel launch, the same bits
as its own launch), every member's flux restore and h pattern, one grouped h
convolution, ONE grouped bounded add of h (``steam_bounded_add_group_async``:
one launch per stage of the solve, each persistent phase a cooperative launch
whose blocks split into per-member teams with their own grid barriers) on a
side stream beside every member's qt pattern and the grouped qt convolution,
one grouped bounded add of qt, and every member's thermodynamics.  Members of
uneven sizes fill the GPU side by side.

``autotune_conv`` is the tile-shape autotuner: for a field shape it times the
fused convolution over its CTA tile heights (32 or 64 rows for the packed
float32 kernel) and x-chunk lengths (planes per CTA; short chunks give small
members enough CTAs, long ones amortise the halo) and installs the fastest
for that shape.  Neither changes the result.
"""

from __future__ import annotations

import ctypes
import time

import numpy as np

from . import _lib
from . import simulate as sim
from . import utils as _utils
from . import resident as _resident
from .resident import ResidentClass

CHUNKS = (16, 32, 64, 128, 256, 384, 512)
_TUNED = {}


def member_setup(shape, seed, alpha=1.8, c1=0.1, H=1.0 / 3.0, Hz=5.0 / 9.0,
                 dtype=np.float32, spheroscale=1000.0):
    """The ClassSetup of a member: the finest class (k = 200 m, dx = dz =
    100 m) of a root run over ``shape`` with the member's parameters.  Hz
    enters through the canonical vertical scale k_z = l_s (k / l_s)^Hz of the
    advective weight's aspect ratio."""
    nx, ny, nz = (int(n) for n in shape)
    height = nz * 100.0
    zp = np.arange(int(height / 50.0) + 1) * 50.0
    hp = (340e3 - 20e3 * zp / zp[-1]).astype(np.float32)
    qp = (0.018 - 0.016 * zp / zp[-1]).astype(np.float32)
    sph = np.full(zp.size, spheroscale)
    k = 200.0
    outer = max(nx, ny) * 100.0
    grids = sim._compute_all_grids(np.array([k]), nx * 100.0, ny * 100.0, height, (1, 1, 1),
                                   sph, zp)
    got = (int(grids['nx'][0]), int(grids['ny'][0]), int(grids['nz'][0]))
    if got != (nx, ny, nz):
        raise ValueError(f"member shape {shape} is not a class grid (got {got})")
    kzl = sim._k_z('piecewise_isotropic_below_spheroscale', outer, sph)
    C_h = sim._compute_normalization(hp, zp, kzl, np.array([k]), outer, grids,
                                     hurst_horizontal=H)[0]
    C_q = sim._compute_normalization(qp, zp, kzl, np.array([k]), outer, grids,
                                     hurst_horizontal=H)[0]
    b_h = sim._bound_buffers([C_h], 1, H)[0]
    b_q = sim._bound_buffers([C_q], 1, H)[0]
    aspect = np.full(nz, spheroscale * (k / spheroscale) ** Hz / k, np.float32)
    n_classes = int(round(np.log(outer / 200.0) / np.log(2.0))) + 1
    key = sim.class_key(np.random.SeedSequence(seed).spawn(n_classes)[-1])
    return sim.make_class_setup(
        grids, 0, h_profile=hp, qt_profile=qp, z_profile=zp, C_h=C_h, C_qt=C_q, b_h=b_h,
        b_qt=b_q, aspect=aspect, bounds=(315 * 1004.0, 355 * 1004.0, 0.0, 0.03), key=key,
        flux_noise_scale=c1, flux_alpha=alpha, dtype=dtype)


def autotune_conv(setup, dtype, chunks=CHUNKS, repeats=3):
    """Time the fused convolution of ``setup``'s kernel on its shape over its
    CTA tile shapes -- for float32 fields the packed kernel's tile height (32
    or 64 rows) -- and x-chunk lengths (0: the kernel's own wave model), and
    install the fastest pair; returns {(rows, chunk): ms}.  Neither changes a
    result."""
    torch = _lib.require_cuda("autotune_conv")
    lib = _lib.load()
    shape = tuple(int(n) for n in setup.shape)
    key = (shape, dtype)
    if key in _TUNED:
        return _TUNED[key]
    plan = setup.plan
    if plan.kind != 'separable':
        return {}
    f = torch.randn(shape, dtype=dtype, device='cuda')
    out = torch.empty_like(f)
    rows_set = (32, 64) if dtype == torch.float32 else (32,)
    times = {}
    for rows in rows_set:
        _lib.check(lib.steam_conv_set_tile_rows(*shape, int(rows)))
        for c in (0,) + tuple(chunks):
            if c > 2 * shape[0]:
                continue
            _lib.check(lib.steam_conv_set_xchunk(*shape, int(c)))
            _utils.run_plan(plan, f, out)  # warm
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(repeats):
                _utils.run_plan(plan, f, out)
            e1.record()
            e1.synchronize()
            times[(rows, c)] = e0.elapsed_time(e1) / repeats
    rows, best = min(times, key=times.get)
    _lib.check(lib.steam_conv_set_tile_rows(*shape, int(rows)))
    _lib.check(lib.steam_conv_set_xchunk(*shape, int(best)))
    _TUNED[key] = times
    return times


class Member:
    """One ensemble member: its setup, resident class step and device fields."""

    def __init__(self, shape, seed, alpha=1.8, c1=0.1, H=1.0 / 3.0, Hz=5.0 / 9.0,
                 dtype=np.float32, init_seed=None):
        torch = _lib.require_cuda("ensemble member")
        self.params = dict(shape=tuple(int(n) for n in shape), seed=int(seed), alpha=alpha,
                           c1=c1, H=H, Hz=Hz)
        self.setup = member_setup(shape, seed, alpha, c1, H, Hz, dtype)
        tdt = torch.float64 if np.dtype(dtype) == np.float64 else torch.float32
        self.rc = ResidentClass(self.setup, tdt)
        g = torch.Generator(device='cuda')
        g.manual_seed(int(seed if init_seed is None else init_seed))
        self.h0 = 600.0 * torch.randn(shape, generator=g, device='cuda', dtype=tdt)
        self.q0 = 0.0006 * torch.randn(shape, generator=g, device='cuda', dtype=tdt)
        self.F0 = 1.0 + 0.1 * torch.rand(shape, generator=g, device='cuda', dtype=tdt)
        self.h, self.q, self.F = self.h0.clone(), self.q0.clone(), self.F0.clone()
        self.diag = {k: torch.empty_like(self.h) for k in ("T", "qv", "qc", "qi", "p")}

    @property
    def voxels(self):
        nx, ny, nz = self.params['shape']
        return nx * ny * nz

    def reset(self):
        self.h.copy_(self.h0)
        self.q.copy_(self.q0)
        self.F.copy_(self.F0)

    def step(self):
        self.rc.step(self.h, self.q, self.F, diagnostics=self.diag)

    def buffers(self):
        """The member's work fields for a stage-by-stage step: the product,
        the pattern, and one increment per scalar (both bounded adds of the
        ensemble run after all members' increments are in)."""
        import torch
        product, W, inc_h = self.rc._work(self.F)
        if getattr(self, 'inc_qt', None) is None:
            self.inc_qt = torch.empty_like(inc_h)
        return product, W, inc_h, self.inc_qt


class Ensemble:
    """Members spread over ``n_streams`` streams; one step of all of them
    either issued eagerly or replayed from a captured CUDA graph.  Each step
    starts from the members' initial state (the reset copies are part of it),
    so every step does the same work."""

    def __init__(self, members, n_streams=4, tune=True, grouped=True):
        torch = _lib.require_cuda("Ensemble")
        self.members = list(members)
        self.grouped = False
        self.groups = {}
        self.streams = [torch.cuda.Stream() for _ in range(max(1, int(n_streams)))]
        # largest members first, dealt round-robin, so the streams carry
        # similar work
        order = sorted(range(len(self.members)), key=lambda i: -self.members[i].voxels)
        self.lanes = [[] for _ in self.streams]
        for j, i in enumerate(order):
            self.lanes[j % len(self.streams)].append(self.members[i])
        self.tuning = {}
        if tune:
            for m in self.members:
                key = m.params['shape']
                if key not in self.tuning:
                    self.tuning[key] = autotune_conv(m.setup, m.rc.dtype)
        self.graph = None
        # a first eager step on every stream builds each member's work fields
        # and its stream's workspace before anything is captured
        self.step_eager()
        torch.cuda.synchronize()
        self.conv_groups = {}
        self.thermo_group = None
        self.side_stream = torch.cuda.Stream()
        if grouped:
            self.groups = self._prepare_groups()
            self.grouped = bool(self.groups)
            if self.grouped:
                self.conv_groups = self._prepare_conv_groups()
                self.thermo_group = self._prepare_thermo_group()
                self.step_eager()
                torch.cuda.synchronize()

    def _prepare_conv_groups(self):
        """One grouped launch per convolution stage (flux, h, qt) over every
        member, when all members share the filters and the packed kernel
        takes their layout; otherwise the members' convolutions stay
        per-member launches."""
        import torch
        lib = _lib.load()
        plan0 = self.members[0].setup.plan
        if plan0.kind != 'separable' or self.members[0].rc.code != _lib.STEAM_F32:
            return {}
        k0 = np.asarray(plan0.kernel)
        for m in self.members:
            pl = m.setup.plan
            if pl.kind != 'separable' or not np.array_equal(np.asarray(pl.kernel), k0):
                return {}
        groups = {}
        for stage in ('flux', 'h', 'qt'):
            probs = []
            for m in self.members:
                product, W, inc_h, inc_qt = m.buffers()
                if stage == 'flux':
                    probs.append(m.rc.conv_problem(product, m.F, flux=True))
                else:
                    inc = inc_h if stage == 'h' else inc_qt
                    probs.append(m.rc.conv_problem(W, inc, pre=m.rc.pre[stage]))
            arr = (_lib.ConvProblem * len(probs))(*probs)
            nbytes = lib.steam_conv_group_workspace_bytes(len(probs), arr)
            ws = torch.empty(int(nbytes), dtype=torch.uint8, device='cuda')
            epi = _lib.STEAM_EPI_FLUX if stage == 'flux' else _lib.STEAM_EPI_STORE
            rc = lib.steam_conv_group_prepare(
                ctypes.byref(plan0.spec), plan0.z_taps, plan0.y_taps, plan0.x_taps, len(probs),
                arr, epi, _lib.ptr(ws), int(nbytes))
            if rc != 0:
                for w, _ in groups.values():
                    lib.steam_conv_group_release(_lib.ptr(w))
                return {}
            groups[stage] = (ws, arr)
        return groups

    def _prepare_thermo_group(self):
        """Every member's thermodynamics as one launch (the members' dtype is
        common: the grouped bounded adds require it)."""
        import torch
        lib = _lib.load()
        probs = []
        for m in self.members:
            nx, ny, nz = m.rc.shape
            p = _lib.ThermoProblem()
            p.nx, p.ny, p.nz = nx, ny, nz
            p.h, p.qt, p.prof = _lib.ptr(m.h), _lib.ptr(m.q), _lib.ptr(m.rc.prof)
            p.compose = 1
            for j, b in enumerate(m.rc.bounds):
                p.bounds[j] = float(b)
            p.surface_pressure = 101325.0
            p.ps_field = None
            p.T, p.qv, p.qc = (_lib.ptr(m.diag[k]) for k in ("T", "qv", "qc"))
            p.qi, p.p = _lib.ptr(m.diag["qi"]), _lib.ptr(m.diag["p"])
            probs.append(p)
        arr = (_lib.ThermoProblem * len(probs))(*probs)
        nbytes = lib.steam_thermo_group_workspace_bytes(len(probs), arr)
        ws = torch.empty(int(nbytes), dtype=torch.uint8, device='cuda')
        _lib.check(lib.steam_thermo_group_prepare(self.members[0].rc.code, len(probs), arr,
                                                  _lib.ptr(ws), int(nbytes)))
        return (ws, arr)

    def _prepare_groups(self):
        """One grouped bounded add per scalar over every member (members
        whose layout the grouped solve does not take -- nz % 4 != 0 or
        unaligned fields -- keep the per-member path for the whole step)."""
        import torch
        lib = _lib.load()
        groups = {}
        if any(m.rc.code != self.members[0].rc.code or m.voxels == 0 or
               m.params['shape'][2] % 4 for m in self.members):
            return {}
        code = self.members[0].rc.code
        for name in ('h', 'qt'):
            probs = []
            for m in self.members:
                _, _, inc_h, inc_qt = m.buffers()
                pert, inc = (m.h, inc_h) if name == 'h' else (m.q, inc_qt)
                probs.append(m.rc.bounded_add_problem(name, pert, inc))
            arr = (_lib.BAProblem * len(probs))(*probs)
            nbytes = lib.steam_bounded_add_group_workspace_bytes(code, len(probs), arr,
                                                                 _resident.N_RESCALE)
            ws = torch.empty(int(nbytes), dtype=torch.uint8, device='cuda')
            _lib.check(lib.steam_bounded_add_group_prepare(
                code, len(probs), arr, _resident.N_RESCALE, _lib.ptr(ws), int(nbytes)))
            groups[name] = (ws, arr)
        return groups

    def __del__(self):
        # the library keys a prepared group by its workspace's address: forget
        # it before the workspace memory can be reused
        try:
            self.release()
        except Exception:
            pass

    def release(self):
        """Forget the grouped solves' device state (the graph too)."""
        if (not getattr(self, 'groups', None) and not getattr(self, 'conv_groups', None) and
                getattr(self, 'thermo_group', None) is None):
            return
        lib = _lib.load()
        for ws, _ in getattr(self, 'groups', {}).values():
            lib.steam_bounded_add_group_release(_lib.ptr(ws))
        for ws, _ in getattr(self, 'conv_groups', {}).values():
            lib.steam_conv_group_release(_lib.ptr(ws))
        if getattr(self, 'thermo_group', None) is not None:
            lib.steam_thermo_group_release(_lib.ptr(self.thermo_group[0]))
        self.groups = {}
        self.conv_groups = {}
        self.thermo_group = None
        self.grouped = False
        self.graph = None

    def _fan(self, fn):
        """fn(member) for every member on the members' streams, joined back
        to the current stream."""
        import torch
        main = torch.cuda.current_stream()
        for s in self.streams:
            s.wait_stream(main)
        for s, lane in zip(self.streams, self.lanes):
            with torch.cuda.stream(s):
                for m in lane:
                    fn(m)
        for s in self.streams:
            main.wait_stream(s)

    def _issue_grouped(self):
        """One ensemble step stage by stage: every member's flux noise (over
        the streams), ONE grouped flux convolution, every member's flux
        restore and h pattern, one grouped h convolution, ONE grouped bounded
        add of h over all members (on a side stream, beside the next two
        stages), every member's qt pattern, one grouped qt convolution, one
        grouped bounded add of qt, every member's thermodynamics.  (Without conv groups each member runs its own
        convolutions inside the fanned stages.)"""
        lib = _lib.load()
        cg = self.conv_groups

        def conv(stage):
            _lib.check(lib.steam_conv_group_async(_lib.ptr(cg[stage][0]), _lib.stream()))

        def ba(name):
            _lib.check(lib.steam_bounded_add_group_async(_lib.ptr(self.groups[name][0]),
                                                         _lib.stream()))

        if cg:
            def noise(m):
                m.reset()
                product, _, _, _ = m.buffers()
                m.rc.enqueue_noise(m.F, product)

            def finish_h(m):
                product, W, _, _ = m.buffers()
                m.rc.enqueue_flux_finish(m.F)
                m.rc.enqueue_pattern('h', m.h, product, W)

            def pattern_q(m):
                product, W, _, _ = m.buffers()
                m.rc.enqueue_pattern('qt', m.q, product, W)

            import torch
            main = torch.cuda.current_stream()
            self._fan(noise)
            conv('flux')
            self._fan(finish_h)
            conv('h')
            # h's bounded add on a side stream while the qt patterns and the
            # qt convolution run (they read qt', the product and W, never h')
            side = self.side_stream
            side.wait_stream(main)
            with torch.cuda.stream(side):
                ba('h')
            self._fan(pattern_q)
            conv('qt')
            ba('qt')
            main.wait_stream(side)
        else:
            def first(m):
                m.reset()
                product, W, inc_h, _ = m.buffers()
                m.rc.enqueue_flux(m.F, product)
                m.rc.enqueue_increment('h', m.h, product, W, inc_h)

            def second(m):
                product, W, _, inc_qt = m.buffers()
                m.rc.enqueue_increment('qt', m.q, product, W, inc_qt)

            self._fan(first)
            ba('h')
            self._fan(second)
            ba('qt')

        if self.thermo_group is not None:
            _lib.check(lib.steam_thermo_group_async(_lib.ptr(self.thermo_group[0]),
                                                    _lib.stream()))
            for m in self.members:
                m.rc.ledger_host.copy_(m.rc.ledger, non_blocking=True)
                m.rc.ledger_ready.record()
            return

        def third(m):
            m.rc.enqueue_thermo(m.h, m.q, m.diag)
            m.rc.ledger_host.copy_(m.rc.ledger, non_blocking=True)
            m.rc.ledger_ready.record()

        self._fan(third)

    @property
    def voxels(self):
        return sum(m.voxels for m in self.members)

    def _issue(self):
        import torch
        if self.grouped:
            self._issue_grouped()
            return
        main = torch.cuda.current_stream()
        for s in self.streams:
            s.wait_stream(main)
        for s, lane in zip(self.streams, self.lanes):
            with torch.cuda.stream(s):
                for m in lane:
                    m.reset()
                    m.step()
        for s in self.streams:
            main.wait_stream(s)

    def step_eager(self):
        self._issue()

    def capture(self):
        """Capture one step of every member into a CUDA graph."""
        import torch
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        cap = torch.cuda.Stream()
        with torch.cuda.graph(g, stream=cap, capture_error_mode="thread_local"):
            self._issue()
        torch.cuda.synchronize()
        self.graph = g
        return g

    def step_graph(self):
        if self.graph is None:
            self.capture()
        self.graph.replay()

    def check(self):
        """Wait for the device and read every member's ledger; raises if a
        member's step failed (a persistent phase that timed out at a grid
        barrier).  Returns the members' ``ClassLedger``s."""
        import torch
        torch.cuda.synchronize()
        return [m.rc.class_ledger(wait=False) for m in self.members]

    def throughput(self, steps=5, graph=True):
        """Mvoxels/s over ``steps`` ensemble steps (device time)."""
        import torch
        run = self.step_graph if graph else self.step_eager
        run()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record()
        for _ in range(steps):
            run()
        e1.record()
        e1.synchronize()
        host = time.perf_counter() - t0
        ms = e0.elapsed_time(e1)
        return {"mvoxels_per_s": self.voxels * steps / (ms / 1e3) / 1e6,
                "ms_per_step": ms / steps, "host_ms_per_step": 1e3 * host / steps}


def config_members(n_members, seed=3, smallest=(64, 64, 64), largest=(256, 256, 128),
                   dtype=np.float32):
    """Members with sizes log-uniform between two shapes (x = y, nz at most
    the largest's), and alpha ~ U[1.5, 1.95], C1 ~ U[0.05, 0.2],
    H ~ U[0.2, 0.5], Hz ~ U[0.5, 0.6]; member seeds 1000 + j."""
    rng = np.random.default_rng(seed)
    lo = np.log(np.prod(smallest))
    hi = np.log(np.prod(largest))
    out = []
    for j in range(n_members):
        v = np.exp(rng.uniform(lo, hi))
        # a box with x = y = 2 nz (capped), sizes on multiples of 16
        nz = int(min(largest[2], max(smallest[2], round((v / 4) ** (1 / 3) / 16) * 16)))
        nxy = int(max(smallest[0], min(largest[0], round(np.sqrt(v / nz) / 16) * 16)))
        out.append(Member((nxy, nxy, nz), 1000 + j, alpha=rng.uniform(1.5, 1.95),
                          c1=rng.uniform(0.05, 0.2), H=rng.uniform(0.2, 0.5),
                          Hz=rng.uniform(0.5, 0.6), dtype=dtype))
    return out


def plain_fp64_throughput(members, steps=1):
    """Mvoxels/s of the plain FP64 drop-in on the same members: each member's
    class step stage by stage (every realized scalar read back to the host
    between stages, as the reference's stage functions do) in float64, plus
    the thermodynamic map, one member after another."""
    import torch
    from .ledger import ClassLedger
    from .thermodynamics import recover_diagnostics_device
    work = []
    for m in members:
        p = m.params
        setup = member_setup(p['shape'], p['seed'], p['alpha'], p['c1'], p['H'], p['Hz'],
                             dtype=np.float64)
        h0, q0, F0 = (t.double() for t in (m.h0, m.q0, m.F0))
        work.append((setup, h0, q0, F0))
    voxels = sum(m.voxels for m in members)

    def run():
        for setup, h0, q0, F0 in work:
            h, q, F = h0.clone(), q0.clone(), F0.clone()
            sim.run_class(h, q, F, None, None, None, setup, ClassLedger(), resident=False)
            hlo, hhi, qlo, qhi = setup.bounds
            recover_diagnostics_device(h, q, setup.z, 101325.0, h_mean=setup.h_mean,
                                       qt_mean=setup.qt_mean, bounds=[hlo, hhi, qlo, qhi])

    run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        run()
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    return {"mvoxels_per_s": voxels * steps / (ms / 1e3) / 1e6, "ms_per_step": ms / steps}


def main(argv=None):
    """``python -m steam_b200.ensemble --members N --steps K``: build the
    configuration's members (``config_members``), an ``Ensemble`` over four
    streams (no autotuning), run K eager steps and print the device time."""
    import argparse
    import torch
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--members", type=int, default=256)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--streams", type=int, default=4)
    ap.add_argument("--f64", action="store_true")
    args = ap.parse_args(argv)
    members = config_members(args.members, dtype=np.float64 if args.f64 else np.float32)
    ens = Ensemble(members, n_streams=args.streams, tune=False)
    res = ens.throughput(steps=args.steps, graph=False)
    ens.check()
    print({"members": len(members), "voxels": ens.voxels, "grouped": ens.grouped, **res})
    ens.release()
    torch.cuda.synchronize()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
